"""bench.py's reference arm on the CPU, launched the way multi-GPU runs are
launched (torchrun, two ranks, rendezvous on 127.0.0.1): rank 0 alone prints
one JSON line of the contract and both ranks exit 0."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_reference_arm_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "1",
           "--particles", "2e5", "--nbins", "1024", "--reference-seconds", "1"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["steps"] == 2
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["metric"] == "particle-turns/s (plain)" and d["unit"] == "particle-turns/s"
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["particles"] == 200_000 and d["config"]["nbins"] == 1024


def test_reference_arm_never_loads_the_gpu_library(monkeypatch, capsys):
    """The CPU arm builds its ring in plain Python and runs the oracle only."""
    sys.path.insert(0, ROOT)
    import bench
    from haissinskijulia_b200 import _lib

    def refuse():
        raise AssertionError("the reference arm loaded the GPU library")
    monkeypatch.setattr(_lib, "load", refuse)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--steps", "1",
                                      "--warmup", "0", "--particles", "5e4", "--nbins", "512",
                                      "--turns-per-step", "3", "--reference-seconds", "0.2"])
    bench.main()
    d = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["config"]["turns_per_step"] == 3


def test_plain_python_ring_equals_the_library_ring():
    """bench.ring_structs restates rings.benchmark_ring and hj_wake_resonator
    field for field."""
    sys.path.insert(0, ROOT)
    import bench
    from haissinskijulia_b200 import benchmark_ring
    p, w, sz, sE = bench.ring_structs(16384)
    cfg = benchmark_ring(n_turns=1, nbins=16384)
    pc, wc = cfg.params.to_c(), cfg.wake.to_c()
    for f, _ in pc._fields_:
        if f != "_pad":
            assert getattr(p, f) == getattr(pc, f), f
    for f, _ in wc._fields_:
        assert getattr(w, f) == getattr(wc, f), f
    assert (sz, sE) == (cfg.sigma_z, cfg.sigma_E)


def test_sharded_arm_plan_under_torchrun():
    """bench.py --gpus 2 shards one bunch of 2 x particles over the ranks: rank
    r owns [r n, (r + 1) n) of 2n (the argument handling of the multi-GPU arm,
    launched as the driver launches it; --plan-only does no GPU work)."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--gpus", "2", "--steps", "2", "--warmup", "1", "--particles", "1e8", "--plan-only"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["parallelism"] == "shard"
    assert d["plan"] == [
        {"rank": 0, "n_local": 100_000_000, "first_particle": 0, "n_global": 200_000_000},
        {"rank": 1, "n_local": 100_000_000, "first_particle": 100_000_000,
         "n_global": 200_000_000}]


def test_gpus_must_match_the_world_size():
    out = subprocess.run([sys.executable, "bench.py", "--gpus", "2", "--plan-only"], cwd=ROOT,
                         capture_output=True, text=True, timeout=120)
    assert out.returncode != 0 and "WORLD_SIZE=1" in (out.stderr + out.stdout)
