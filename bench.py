#!/usr/bin/env python
"""Benchmark of the B200 tracking path: particle-turns/s of the plain single-bunch
method at scale (1e8 Float64 macroparticles, 16384 bins, the benchmark ring with
its broadband-resonator wake, every physics switch on).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one turn of the whole bunch.  `value` is device-timed (CUDA events on
the bunch's stream, max over ranks) with the state resident in HBM; `e2e` is the
public longitudinal_evolve call with pinned host buffers, host<->device copies
inside the timed region.  `--impl reference` times the CPU oracle (the plain-C
restatement of the reference's turn loop, OpenMP over all host cores) on the
same workload, rank 0 only.  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-turns/s (plain)"
UNIT = "particle-turns/s"
BYTES_PER_PARTICLE_TURN = 32   # read + write z and ΔE, Float64
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--particles", type=float, default=1e8)
    ap.add_argument("--nbins", type=int, default=16384)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--layout", type=int, default=-1,
                    help="thread layout of the fused pass (-1 = library default)")
    ap.add_argument("--e2e-calls", type=int, default=1,
                    help="timed longitudinal_evolve calls (after one warm-up call)")
    ap.add_argument("--e2e-turns", type=int, default=10000,
                    help="turns per call: the at-scale configuration's 10,000")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="bounded CPU work of the cpu_baseline leg")
    ap.add_argument("--reference-seconds", type=float, default=90.0,
                    help="bounded CPU work of the --impl reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-sweep", action="store_true",
                    help="skip the batched-sweep / serving measurements (single GPU only)")
    ap.add_argument("--sweep-turns", type=int, default=5000)
    ap.add_argument("--sweep-plain-points", type=int, default=8,
                    help="points of the sweep also run one after another on the plain path")
    ap.add_argument("--serve-requests", type=int, default=40)
    ap.add_argument("--scan-points", type=int, default=32,
                    help="parameter-scan points (0: no scan measurement)")
    ap.add_argument("--scan-samples", type=int, default=20)
    ap.add_argument("--scan-sequential-points", type=int, default=4)
    return ap.parse_args()


def workload(n: int, B: int) -> dict:
    return {
        "workload": f"plain single bunch at scale: {n:.0e} Float64 macroparticles, {B} bins, "
                    "4 GeV benchmark ring, resonator wake (Rs=10kOhm, Q=1, fr=20GHz, 1e10 e-), "
                    "RF+QE(Philox)+SR+drift+wake+E0 update every turn; moments and line density "
                    "logged on the device every 100 turns",
        "particles": n,
        "nbins": B,
        "turns_per_step": 1,
        "l2": (f"state ({16 * n / 1e6:.0f} MB, 16 B/particle) exceeds the 126 MB L2; "
               "no flush between turns") if 16 * n > 126e6 else
              (f"state ({16 * n / 1e6:.1f} MB) fits the 126 MB L2: a small case, "
               "not the measured workload"),
    }


def measured_hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic_per_particle_turn():
    """DRAM bytes per particle-turn of the particle pass from the committed ncu
    summary (profiles/), or None."""
    for f in sorted((ROOT / "profiles").glob("*.md")):
        m = re.search(r"dram_bytes_per_particle_turn:\s*([0-9.eE+-]+)", f.read_text())
        if m:
            return float(m.group(1)), f.name
    return None, None


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"hj_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "power_w_median": statistics.median(power) if power else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_oracle_rate(n: int, B: int, seconds: float, seed: int, threads: int):
    """Particle-turns/s of the CPU oracle on an n-particle bunch of the benchmark
    workload: whole turns until `seconds` of CPU work (at least one turn)."""
    from haissinskijulia_b200 import benchmark_ring, synthetic_bunch
    from oracle import Oracle
    cfg = benchmark_ring(n_turns=1, nbins=B)
    orc = Oracle(threads=threads)
    p = synthetic_bunch(n, cfg.sigma_z, cfg.sigma_E, seed)
    z, dE = p.coordinates.z, p.coordinates.dE
    st = orc.state(z, dE, cfg.params.to_c(), cfg.wake.to_c(), B, None, seed=seed)
    turns = 0
    t0 = time.perf_counter()
    while True:
        st.turn(None)
        turns += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    st.close()
    return n * turns / el, turns, el


def run_reference(args) -> None:
    """--impl reference: the CPU oracle of the reference's loop, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n_full, B = int(args.particles), args.nbins
    cores = cpu_cores()
    from haissinskijulia_b200 import benchmark_ring, synthetic_bunch
    from oracle import Oracle
    orc = Oracle(threads=cores)
    # size the per-step sample so warmup + steps fit the CPU budget
    probe, _, _ = cpu_oracle_rate(min(n_full, 1_000_000), B, 0.5, args.seed, cores)
    total_steps = args.steps + args.warmup
    n = int(min(n_full, max(100_000, args.reference_seconds * probe / max(total_steps, 1))))
    cfg = benchmark_ring(n_turns=1, nbins=B)
    p = synthetic_bunch(n, cfg.sigma_z, cfg.sigma_E, args.seed)
    st = orc.state(p.coordinates.z, p.coordinates.dE, cfg.params.to_c(), cfg.wake.to_c(), B,
                   None, seed=args.seed)
    for _ in range(args.warmup):
        st.turn(None)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st.turn(None)
    el = time.perf_counter() - t0
    value = n * args.steps / el
    sample = (f"{n} of the {n_full:.0e} particles per step (one turn each, {B} bins), "
              f"oracle/oracle.c (plain-C restatement of longitudinal_evolve!, OpenMP)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload(n_full, B),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def measure_sweeps(ctx, args) -> dict:
    """The ragged 256-point sweep (batched vs plain point by point), the
    32-bunch intensity scan and a served request stream, host wall clock
    around each (admission, turns, retirement and result read-back included)."""
    import numpy as np
    from haissinskijulia_b200.sweep import (autotune, intensity_scan, request_stream,
                                            run_batched, run_plain, serve, serve_plain,
                                            sweep_points)
    T = args.sweep_turns
    pts = sweep_points(256, turns=T)
    t0 = time.perf_counter()
    tun = autotune(ctx, pts, trial_turns=32, sample=64)
    t_tune = time.perf_counter() - t0
    t0 = time.perf_counter()
    bat = run_batched(ctx, pts, tuning=tun, block_turns=500)
    t_bat = time.perf_counter() - t0
    k = max(1, min(args.sweep_plain_points, len(pts)))
    idx = list(range(0, len(pts), len(pts) // k))[:k]
    t0 = time.perf_counter()
    pla = run_plain(ctx, [pts[i] for i in idx])
    t_pla = time.perf_counter() - t0
    rel = 0.0
    for j, i in enumerate(idx):
        a, b = bat[i].result, pla[j].result
        for key in ("E0", "sigma_E", "sigma_z"):
            x, y = getattr(a, key), getattr(b, key)
            rel = max(rel, abs(x - y) / abs(y))
    pt = sum(p.n * p.turns for p in pts)
    out = {
        "config": f"256 points: V ~ U[3,7] MV, population log-U[1e9,1e11], particles "
                  f"log-U[1e4,2e6] (total {sum(p.n for p in pts):.3e}), {T} turns, 4096 bins, "
                  "own seed; bunches generated on the device",
        "batched_solves_per_s": len(pts) / t_bat, "batched_seconds": t_bat,
        "batched_particle_turns_per_s": pt / t_bat,
        "plain_solves_per_s": k / t_pla, "plain_seconds": t_pla,
        "plain_sample": f"{k} of the 256 points (every {len(pts) // k}th), all {T} turns each, "
                        "one after another on the plain resident path",
        "speedup_vs_plain": (len(pts) / t_bat) / (k / t_pla),
        "max_rel_diff_vs_plain": rel,
        "tuning": {"particles_per_block": tun.chunk, "layout": tun.layout,
                   "graph_turns": tun.graph_turns, "autotune_seconds": t_tune},
        "timing": "host wall clock: admission, every turn, retirement",
    }
    scan = intensity_scan(turns=T)
    t0 = time.perf_counter()
    tun_i = autotune(ctx, scan, trial_turns=32, sample=len(scan))
    t_tune_i = time.perf_counter() - t0
    t0 = time.perf_counter()
    run_batched(ctx, scan, tuning=tun_i, block_turns=500)
    t_scan = time.perf_counter() - t0
    out["intensity_scan"] = {
        "config": f"32 bunches x 1e6 particles, populations log-spaced 1e9-1e11, {T} turns, "
                  "8192 bins, one batch",
        "solves_per_s": len(scan) / t_scan, "seconds": t_scan,
        "particle_turns_per_s": sum(p.n * p.turns for p in scan) / t_scan,
        "tuning": {"particles_per_block": tun_i.chunk, "layout": tun_i.layout,
                   "graph_turns": tun_i.graph_turns, "autotune_seconds": t_tune_i}}
    if args.serve_requests > 0:
        reqs = request_stream(args.serve_requests)
        rep = serve(ctx, reqs, tuning=tun)
        sm = rep.summary()
        sm["config"] = (f"{args.serve_requests} requests, Poisson arrivals at 50/s, V ~ U[3,7] "
                        "MV, population log-U[1e9,1e11], particles log-U[1e4,4e6], turns "
                        "U[1000,20000], bins in {2048,4096,8192}; admission by footprint "
                        "(8 GB budget), 200-turn blocks")
        sm["particle_turns_per_s"] = sm["particle_turns"] / sm["wall_s"]
        pl = serve_plain(ctx, reqs).summary()
        sm["plain"] = {"solves_per_s": pl["solves_per_s"], "p50_latency_s": pl["p50_latency_s"],
                       "p99_latency_s": pl["p99_latency_s"], "wall_s": pl["wall_s"],
                       "how": "the same requests one at a time on the plain resident path, "
                              "first come first served (measured service times)"}
        sm["speedup_vs_plain"] = sm["solves_per_s"] / pl["solves_per_s"]
        out["serving"] = sm
    if args.scan_points > 0:
        out["parameter_scan"] = measure_scan(ctx, args)
    return out


def measure_scan(ctx, args) -> dict:
    """scan_parameter (src/parameter_sensitivity/scan.jl) over RF voltage with
    the emittance figure of merit and derivative samples: every run in one
    batch, against the same runs one after another on a sample of points."""
    import numpy as np
    from haissinskijulia_b200 import Particles, benchmark_ring
    from haissinskijulia_b200.sensitivity import (EmittanceFoM, VoltageTransform,
                                                  scan_parameter, scan_parameter_sequential)
    n, P, S = 100_000, args.scan_points, args.scan_samples
    cfg = benchmark_ring(n_turns=100, nbins=n // 10)
    rng = np.random.default_rng(args.seed)
    parts = Particles(rng.normal(0.0, cfg.sigma_z, n), rng.normal(0.0, cfg.sigma_E, n))
    values = np.linspace(3e6, 7e6, P)
    kw = dict(ctx=ctx, n_samples=S, seed=args.seed, return_runs=True)
    times = []
    for _ in range(2):            # the first scan also fills the context's block cache
        t0 = time.perf_counter()
        _, fb, gb, _, runs = scan_parameter(VoltageTransform(), EmittanceFoM(), values, parts,
                                            cfg.params, block_turns=32, graph_turns=32, **kw)
        times.append(time.perf_counter() - t0)
    t_bat = times[-1]
    k = max(1, min(args.scan_sequential_points, P))
    idx = list(range(0, P, max(P // k, 1)))[:k]
    t0 = time.perf_counter()
    _, fs, gs, _, _ = scan_parameter_sequential(VoltageTransform(), EmittanceFoM(),
                                                values[idx], parts, cfg.params, **kw)
    t_seq = time.perf_counter() - t0
    rel = float(np.max(np.abs(fb[idx] - fs) / np.abs(fs)))
    return {
        "config": f"{P} RF voltages in [3, 7] MV, EmittanceFoM, {S} derivative samples per "
                  f"point ({1 + 2 * S} runs per point, {len(runs)} in all); 1e5 particles, "
                  "1e4 bins (the reference's nbins = n/10), 100-turn point runs, 10-turn "
                  "derivative runs",
        "batched_points_per_s": P / t_bat, "batched_seconds": t_bat,
        "batched_seconds_first_scan": times[0],
        "sequential_points_per_s": k / t_seq, "sequential_seconds": t_seq,
        "sequential_sample": f"{k} of the {P} points, all their runs one after another on "
                             "the plain resident path",
        "speedup_vs_sequential": (P / t_bat) / (k / t_seq),
        "max_rel_diff_fom": rel,
        "timing": "host wall clock: admission, every turn, retirement, figures of merit",
    }


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from haissinskijulia_b200 import (Context, Particles, ResidentBunch, benchmark_ring,
                                      create_simulation_buffers, longitudinal_evolve)
    from haissinskijulia_b200 import build as hjbuild
    hjbuild.build()

    n, B, K, W = int(args.particles), args.nbins, args.steps, args.warmup
    cfg = benchmark_ring(n_turns=K, nbins=B)
    ctx = Context(local)
    ctx.set_pass_layout(args.layout)
    stream = torch.cuda.current_stream()
    gen = torch.Generator(device="cuda").manual_seed(args.seed + 7919 * rank)
    z = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) * cfg.sigma_z
    dE = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) * cfg.sigma_E
    bunch = ResidentBunch(ctx, z.data_ptr(), dE.data_ptr(), n, cfg.params, B, wake=cfg.wake,
                          seed=args.seed + rank, stream=stream.cuda_stream)
    # moments and line density logged on the device every 100 turns
    bunch.set_log(100, capacity=(K + W) // 100 + 1, density=True)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    bunch.advance(W)
    barrier()
    bunch.set_profiling(True)
    clocks = ClockSampler(local)
    clocks.start()
    t_wall0 = time.perf_counter()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    bunch.advance(K)
    ev1.record(stream)
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    clock_info = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    prof = bunch.read_profile()
    log = bunch.read_log()
    res = bunch.finish()
    bunch.close()
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = n * K * world / (ms / 1e3)

    # roofline of the dominant kernel (the fused particle pass)
    pass_ms = prof["pass_ms"] / max(prof["turns"], 1)
    bins_ms = prof["bins_ms"] / max(prof["turns"], 1)
    achieved = BYTES_PER_PARTICLE_TURN * n / (pass_ms / 1e3) / 1e9
    peak, peak_kind = measured_hbm_peak()
    tr, tr_src = profiled_traffic_per_particle_turn()
    roofline = {"bound": "hbm", "kernel": "k_track_pass", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6.65 TB/s",
                "traffic": (tr * n) if tr else None,
                "traffic_source": tr_src,
                "algorithmic_bytes": BYTES_PER_PARTICLE_TURN * n,
                "pass_ms": pass_ms, "bins_ms": bins_ms,
                "pass_share": prof["pass_ms"] / max(prof["pass_ms"] + prof["bins_ms"], 1e-30)}

    # e2e through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        del z, dE
        torch.cuda.empty_cache()
        E = args.e2e_turns
        params = cfg.params.replace(n_turns=E)
        zh = torch.empty(n, dtype=torch.float64, pin_memory=True)
        eh = torch.empty(n, dtype=torch.float64, pin_memory=True)
        g = torch.Generator().manual_seed(args.seed + rank)
        z0 = torch.randn(n, dtype=torch.float64, generator=g) * cfg.sigma_z
        e0 = torch.randn(n, dtype=torch.float64, generator=g) * cfg.sigma_E
        buf = create_simulation_buffers(n, B, ctx=ctx)
        times = []
        for c in range(args.e2e_calls + 1):          # first call warms the allocator
            zh.copy_(z0)
            eh.copy_(e0)
            p = Particles(zh.numpy(), eh.numpy())
            assert p.coordinates.z.ctypes.data == zh.data_ptr()
            barrier()
            t0 = time.perf_counter()
            longitudinal_evolve(p, params, buf, wake=cfg.wake, seed=args.seed + c)
            times.append(time.perf_counter() - t0)
        t_e2e = max(times[1:]) if len(times) > 1 else times[0]
        if world > 1:
            t = torch.tensor([t_e2e], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e2e = float(t.item())
        e2e = {"value": n * E * world / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 16 * n,
               "d2h_bytes_per_step": 16 * n, "turns_per_step": E,
               "seconds_per_step": t_e2e, "api": "haissinskijulia_b200.longitudinal_evolve -> hj_evolve"}

    sweep = None
    if world == 1 and not args.no_sweep:
        sweep = measure_sweeps(ctx, args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = cpu_cores()
        rate, turns, el = cpu_oracle_rate(n, B, args.cpu_seconds, args.seed, cores)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{turns} whole turn(s) of the same {n:.0e}-particle, {B}-bin bunch "
                         f"({el:.1f} s) by oracle/oracle.c (plain-C restatement, OpenMP)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload(n, B), parallelism="replicas" if world > 1 else "single GPU"),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "sweep": sweep,
            "gpu_launches": prof["launches"], "clocks": clock_info,
            "wall_seconds_timed": t_wall,
            "turn_log": {"every": 100, "records": int(log.shape[0]),
                         "content": "turn, E0, sigma_z, sigma_E, mean z, mean dE, wake current, "
                                    f"particles in bins + {B} bin counts, written on the device",
                         "last": {"turn": float(log[-1, 0]), "E0": float(log[-1, 1]),
                                  "sigma_z": float(log[-1, 2]), "sigma_E": float(log[-1, 3])}
                         if log.shape[0] else None},
            "final": {"sigma_E": res.sigma_E, "sigma_z": res.sigma_z, "E0": res.E0},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
