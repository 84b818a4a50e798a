#!/usr/bin/env python
"""Benchmark of the B200 tracking path: particle-turns/s of the plain single-bunch
method at scale (1e8 Float64 macroparticles, 16384 bins, the benchmark ring with
its broadband-resonator wake, every physics switch on).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is 100 turns of the whole bunch, ending with the turn-log record
(moments and line density) the at-scale configuration asks for every 100
turns.  `value` is device-timed (CUDA events on the bunch's stream, max over
ranks) with the state resident in HBM; `e2e` is the public longitudinal_evolve
call with pinned host buffers, host<->device copies inside the timed region.
`--impl reference` times the CPU oracle (the plain-C restatement of the
reference's turn loop, OpenMP over all host cores) on the same workload, rank
0 only, without loading the GPU library.  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import math
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
LOG_EVERY = 100                # turns between turn-log records (one per step)
# DRAM bytes (read + write) per particle-turn of k_track_pass from one ncu
# capture, by bin count: (bytes, the profile summary that holds the capture).
PASS_DRAM_BYTES = {16384: (31.45, "profiles/k_track_pass_full_2e7_b16384.md")}


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--particles", type=float, default=1e8)
    ap.add_argument("--nbins", type=int, default=16384)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--turns-per-step", type=int, default=LOG_EVERY,
                    help="turns of one step (the last one writes the turn-log record)")
    ap.add_argument("--multi", choices=["shard", "replicas"], default="shard",
                    help="N > 1: one bunch sharded over the ranks with one all-reduce of the "
                         "bin exchange per turn (default), or independent replicas")
    ap.add_argument("--shard-one-rank", action="store_true",
                    help="under torchrun with one rank: run the sharded arm (N > 1) over a "
                         "one-rank NCCL group, so that its code path runs on one GPU")
    ap.add_argument("--plan-only", action="store_true",
                    help="print the ranks' shard plan (rank 0) and exit; no GPU work")
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
    ap.add_argument("--sweep-plain-points", type=int, default=32,
                    help="points of the sweep (a stratified sample) also run one after "
                         "another on the plain path")
    ap.add_argument("--serve-requests", type=int, default=200,
                    help="requests per offered load of the served stream (0: no serving)")
    ap.add_argument("--serve-rates", default="5,10,20,50",
                    help="offered loads (requests/s) of the served stream")
    ap.add_argument("--scan-points", type=int, default=32,
                    help="parameter-scan points (0: no scan measurement)")
    ap.add_argument("--scan-samples", type=int, default=20)
    ap.add_argument("--scan-sequential-points", type=int, default=4)
    return ap.parse_args()


def workload(n: int, B: int, turns_per_step: int = LOG_EVERY, logged: bool = True) -> dict:
    return {
        "workload": f"plain single bunch at scale: {n:.0e} Float64 macroparticles, {B} bins, "
                    "4 GeV benchmark ring, resonator wake (Rs=10kOhm, Q=1, fr=20GHz, 1e10 e-), "
                    "RF+QE(Philox)+SR+drift+wake+E0 update every turn"
                    + ("; moments and line density logged on the device every 100 turns"
                       if logged else ""),
        "particles": n,
        "nbins": B,
        "turns_per_step": turns_per_step,
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


class ClockSampler:
    """nvidia-smi clock/throttle samples every 100 ms; mark() brackets the
    timed region so that only its samples are summarised."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.marks = []
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"hj_clocks_{os.getpid()}.csv"

    def start(self):
        """Starts the sampler and waits (up to 5 s) for its first sample."""
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.device)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 5.0 and self._lines() == 0 and self.proc.poll() is None:
            time.sleep(0.05)

    def _lines(self) -> int:
        try:
            return len(self.path.read_text().splitlines())
        except Exception:
            return 0

    def mark(self):
        self.marks.append(self._lines())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)              # the sample that closes the timed region
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        lines = self.path.read_text().splitlines()
        lo, hi = (self.marks[0], self.marks[1] + 1) if len(self.marks) >= 2 else (0, len(lines))
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in lines[lo:hi]:
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
                "samples": len(sm), "reasons": sorted(reasons),
                "window": "samples every 100 ms between the start and the end of the timed region"}


def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def ring_structs(B: int):
    """The benchmark ring's (hj_params, hj_wake) in plain Python, so that the
    CPU legs never load the GPU library: the values of rings.benchmark_ring
    (E0 = 4 GeV, h = 360 at 500 MHz, V = 5 MV, α_c = 3e-4, U0 = 0.5 MeV,
    5000-turn damping) and the resonator mapping of hj_wake_resonator
    (Rs = 10 kΩ, Q = 1, f_r = 20 GHz, 1e10 electrons, bins over ±6σ_z)."""
    from haissinskijulia_b200._lib import HjParams, HjWake
    E0, U0, V, c = 4e9, 0.5e6, 5e6, 299792458.0
    p = HjParams()
    p.E0, p.mass, p.voltage, p.harmonic = E0, 0.51099895069e6, V, 360
    p.radius = 4 * 8.85e-5 * (E0 / 1e9) ** 3 * 5000.0
    p.pipe_radius, p.alpha_c, p.phi_s, p.freq_rf = 2.5e-4, 3e-4, math.pi - math.asin(U0 / V), 500e6
    p.n_turns = 1
    p.use_wakefield = p.update_eta = p.update_E0 = p.SR_damping = p.use_excitation = 1
    wr = 6.283185307179586 * 20e9
    alpha = wr / 2.0
    wbar = math.sqrt(wr * wr - alpha * alpha)
    w = HjWake()
    w.wake_factor, w.wake_sqrt, w.ctau, w.sin_coef = 2.0 * alpha * 1e4, wbar / c, c / alpha, alpha / wbar
    w.population, w.half_width_sigmas, w.delta_std = 1e10, 6.0, 0.15
    return p, w, 4e-3, 1e-3 * E0


def cpu_oracle_rate(n: int, B: int, seconds: float, seed: int, threads: int, tps: int = 1):
    """Particle-turns/s of the CPU oracle on an n-particle bunch of the benchmark
    workload: whole blocks of `tps` turns until `seconds` of CPU work (at least one)."""
    from oracle import Oracle
    params, wake, sigma_z, sigma_E = ring_structs(B)
    orc = Oracle(threads=threads)
    rng = np.random.Generator(np.random.Philox(seed))
    z, dE = rng.normal(0.0, sigma_z, n), rng.normal(0.0, sigma_E, n)
    st = orc.state(z, dE, params, wake, B, None, seed=seed)
    turns = 0
    t0 = time.perf_counter()
    while True:
        for _ in range(tps):
            st.turn(None)
        turns += tps
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    st.close()
    return n * turns / el, turns, el


def run_reference(args) -> None:
    """--impl reference: the CPU oracle of the reference's loop, rank 0 only,
    on the same ring, wake and step (100 turns) as the GPU arm, over a bounded
    sample of the bunch's particles."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import Oracle
    n_full, B, tps = int(args.particles), args.nbins, args.turns_per_step
    cores = cpu_cores()
    orc = Oracle(threads=cores)
    # size the per-step sample so warmup + steps fit the CPU budget
    probe, _, _ = cpu_oracle_rate(min(n_full, 1_000_000), B, 0.5, args.seed, cores)
    total_turns = (args.steps + args.warmup) * tps
    n = int(min(n_full, max(20_000, args.reference_seconds * probe / max(total_turns, 1))))
    params, wake, sigma_z, sigma_E = ring_structs(B)
    rng = np.random.Generator(np.random.Philox(args.seed))
    z, dE = rng.normal(0.0, sigma_z, n), rng.normal(0.0, sigma_E, n)
    st = orc.state(z, dE, params, wake, B, None, seed=args.seed)
    for _ in range(args.warmup * tps):
        st.turn(None)
    t0 = time.perf_counter()
    for _ in range(args.steps * tps):
        st.turn(None)
    el = time.perf_counter() - t0
    value = n * args.steps * tps / el
    sample = (f"{n} of the {n_full:.0e} particles, {tps} turns per step, {B} bins: "
              "oracle/oracle.c (plain-C restatement of longitudinal_evolve!, OpenMP)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload(n_full, B, tps),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _max_rel_diff(a_solves, b_solves) -> float:
    rel = 0.0
    for a, b in zip(a_solves, b_solves):
        for key in ("E0", "sigma_E", "sigma_z"):
            x, y = getattr(a.result, key), getattr(b.result, key)
            rel = max(rel, abs(x - y) / abs(y))
    return rel


def stratified_sample(points, k: int):
    """k points, one from each of k equal strata of the points sorted by
    particle count (the middle one of each), so that the sample's particle
    counts follow the whole sweep's distribution."""
    order = sorted(range(len(points)), key=lambda i: points[i].n)
    size = len(order) / k
    return sorted(order[int((j + 0.5) * size)] for j in range(k))


def measure_sweeps(ctx, args) -> dict:
    """The ragged 256-point sweep (batched vs plain point by point on a
    stratified sample), the 32-bunch intensity scan (batched vs all 32 bunches
    one after another) and served request streams at several offered loads
    (batched vs one at a time), host wall clock around each (admission,
    turns, retirement and result read-back included)."""
    from haissinskijulia_b200.sweep import (autotune, intensity_scan, plain_service,
                                            plain_timeline, request_stream, run_batched,
                                            run_plain, serve, sweep_points)
    T = args.sweep_turns
    pts = sweep_points(256, turns=T)
    t0 = time.perf_counter()
    tun = autotune(ctx, pts, trial_turns=32, sample=64)
    t_tune = time.perf_counter() - t0
    t0 = time.perf_counter()
    bat = run_batched(ctx, pts, tuning=tun, block_turns=500)
    t_bat = time.perf_counter() - t0
    k = max(1, min(args.sweep_plain_points, len(pts)))
    idx = stratified_sample(pts, k)
    t0 = time.perf_counter()
    pla = run_plain(ctx, [pts[i] for i in idx])
    t_pla = time.perf_counter() - t0
    pt = sum(p.n * p.turns for p in pts)
    # the sample's particle-turns scaled to the whole sweep
    sample_pt = sum(pts[i].n * pts[i].turns for i in idx)
    plain_est_s = t_pla * pt / sample_pt
    out = {
        "config": f"256 points: V ~ U[3,7] MV, population log-U[1e9,1e11], particles "
                  f"log-U[1e4,2e6] (total {sum(p.n for p in pts):.3e}), {T} turns, 4096 bins, "
                  "own seed; bunches generated on the device",
        "batched_solves_per_s": len(pts) / t_bat, "batched_seconds": t_bat,
        "batched_particle_turns_per_s": pt / t_bat,
        "plain_solves_per_s": k / t_pla, "plain_seconds": t_pla,
        "plain_sample": f"{k} of the 256 points, one from each of {k} strata of equal size by "
                        f"particle count (mean {np.mean([pts[i].n for i in idx]):.3e} particles "
                        f"against {np.mean([p.n for p in pts]):.3e} for all 256), all {T} "
                        "turns each, one after another on the plain resident path",
        "plain_seconds_scaled_to_256_by_particle_turns": plain_est_s,
        "speedup_vs_plain": (len(pts) / t_bat) / (k / t_pla),
        "speedup_vs_plain_by_particle_turns": plain_est_s / t_bat,
        "max_rel_diff_vs_plain": _max_rel_diff([bat[i] for i in idx], pla),
        "tuning": {"particles_per_block": tun.chunk, "layout": tun.layout,
                   "graph_turns": tun.graph_turns, "autotune_seconds": t_tune},
        "timing": "host wall clock: admission, every turn, retirement",
    }
    scan = intensity_scan(turns=T)
    t0 = time.perf_counter()
    tun_i = autotune(ctx, scan, trial_turns=32, sample=len(scan))
    t_tune_i = time.perf_counter() - t0
    t0 = time.perf_counter()
    sbat = run_batched(ctx, scan, tuning=tun_i, block_turns=500)
    t_scan = time.perf_counter() - t0
    t0 = time.perf_counter()
    spla = run_plain(ctx, scan)
    t_scan_plain = time.perf_counter() - t0
    out["intensity_scan"] = {
        "config": f"32 bunches x 1e6 particles, populations log-spaced 1e9-1e11, {T} turns, "
                  "8192 bins, one batch",
        "solves_per_s": len(scan) / t_scan, "seconds": t_scan,
        "particle_turns_per_s": sum(p.n * p.turns for p in scan) / t_scan,
        "plain_solves_per_s": len(scan) / t_scan_plain, "plain_seconds": t_scan_plain,
        "plain_how": "all 32 bunches one after another on the plain resident path",
        "speedup_vs_plain": t_scan_plain / t_scan,
        "max_rel_diff_vs_plain": _max_rel_diff(sbat, spla),
        "tuning": {"particles_per_block": tun_i.chunk, "layout": tun_i.layout,
                   "graph_turns": tun_i.graph_turns, "autotune_seconds": t_tune_i}}
    if args.serve_requests > 0:
        rates = [float(r) for r in args.serve_rates.split(",") if r]
        base = request_stream(args.serve_requests, rate=rates[0])
        service = plain_service(ctx, base)             # the same requests at every rate
        loads = []
        for rate in rates:
            reqs = request_stream(args.serve_requests, rate=rate)
            assert [(p.n, p.turns, p.seed) for p in reqs] == [(p.n, p.turns, p.seed) for p in base]
            sm = serve(ctx, reqs, tuning=tun).summary()
            sm["offered_rate_per_s"] = rate
            sm["particle_turns_per_s"] = sm["particle_turns"] / sm["wall_s"]
            pl = plain_timeline(reqs, service).summary()
            sm["plain"] = {"solves_per_s": pl["solves_per_s"],
                           "p50_latency_s": pl["p50_latency_s"],
                           "p99_latency_s": pl["p99_latency_s"], "wall_s": pl["wall_s"]}
            sm["speedup_vs_plain"] = sm["solves_per_s"] / pl["solves_per_s"]
            loads.append(sm)
        out["serving"] = {
            "config": f"{args.serve_requests} requests per offered load, Poisson arrivals, V ~ "
                      "U[3,7] MV, population log-U[1e9,1e11], particles log-U[1e4,4e6], turns "
                      "U[1000,20000], bins in {2048,4096,8192}; admission by footprint (8 GB "
                      "budget), 200-turn blocks; the same requests at every rate",
            "plain_how": "the same requests one at a time on the plain resident path, first "
                         "come first served, each taking its measured service time",
            "plain_service_seconds_total": float(sum(s.finished for s in service)),
            "loads": loads}
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


def shard_plan(rank: int, world: int, n_per_rank: int) -> dict:
    """Weak scaling: every rank holds n_per_rank particles of one bunch of
    world * n_per_rank; rank r owns particles [r n, (r + 1) n), whose Philox
    draws are those of the same particles of the whole bunch."""
    return {"rank": rank, "n_local": n_per_rank, "first_particle": rank * n_per_rank,
            "n_global": world * n_per_rank}


def run_plan(args) -> None:
    """--plan-only: the shard plan of every rank, gathered on rank 0."""
    import datetime
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    plan = shard_plan(rank, world, int(args.particles))
    plans = [plan]
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        plans = [None] * world
        dist.all_gather_object(plans, plan)
    if rank == 0:
        print(json.dumps({"n_gpus": world, "parallelism": args.multi if world > 1 else
                          "single GPU", "plan": plans}), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_sharded(args, ctx, cfg, stream, rank, world, local, clocks) -> None:
    """N > 1: one bunch of N x particles sharded over the ranks.  Per turn each
    rank runs the fused pass on its particles (hj_bunch_pass), the two
    exchange buffers (bin counts and cell deposits, 3B + 2 u64; the four sums)
    are summed over the ranks with NCCL all-reduces on the bunch's stream, and
    every rank runs the same bins step (hj_bunch_bins).  Timed with CUDA events
    on that stream, max over ranks."""
    import torch
    import torch.distributed as dist
    from haissinskijulia_b200 import BinGrid, ShardedBunch
    n, B, K, W, tps = int(args.particles), args.nbins, args.steps, args.warmup, args.turns_per_step
    plan = shard_plan(rank, world, n)
    grid = BinGrid.make(cfg.sigma_z, B, cfg.wake.half_width_sigmas)    # the same on every rank
    gen = torch.Generator(device="cuda").manual_seed(args.seed + 7919 * rank)
    z = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) * cfg.sigma_z
    dE = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) * cfg.sigma_E
    sb = ShardedBunch(ctx, z.data_ptr(), dE.data_ptr(), n, plan["first_particle"],
                      plan["n_global"], cfg.params, grid, wake=cfg.wake, seed=args.seed,
                      stream=stream.cuda_stream)
    counts, sums = sb.buffers()
    pass_events = []

    def turn(profile: bool):
        if profile:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
        sb.pass_()
        if profile:
            b.record(stream)
            pass_events.append((a, b))
        dist.all_reduce(counts)
        dist.all_reduce(sums)
        sb.bins()

    for _ in range(W * tps):
        turn(False)
    torch.cuda.synchronize()
    dist.barrier()
    clocks.mark()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(K * tps):
        turn(True)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks.mark()
    clock_info = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    pass_ms = sum(a.elapsed_time(b) for a, b in pass_events) / len(pass_events)
    res = sb.global_result()
    sb.finish()
    sb.close()
    del z, dE, counts, sums
    t = torch.tensor([ms, pass_ms], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, pass_ms = float(t[0].item()), float(t[1].item())
    value = plan["n_global"] * K * tps / (ms / 1e3)

    # secondary: independent replicas (no exchange), 2 steps
    from haissinskijulia_b200 import ResidentBunch
    zr = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) * cfg.sigma_z
    er = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) * cfg.sigma_E
    rb = ResidentBunch(ctx, zr.data_ptr(), er.data_ptr(), n, cfg.params, B, wake=cfg.wake,
                       seed=args.seed + rank, stream=stream.cuda_stream)
    rb.advance(tps)
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    rb.advance(2 * tps)
    e1.record(stream)
    torch.cuda.synchronize()
    rb.finish()
    rb.close()
    del zr, er
    tr = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    dist.all_reduce(tr, op=dist.ReduceOp.MAX)
    replicas = {"value": n * world * 2 * tps / (float(tr.item()) / 1e3), "unit": UNIT,
                "turns": 2 * tps, "how": "one independent bunch per rank, no exchange"}

    # e2e: host shards in pinned memory, copied in, tracked with the exchange, copied out
    e2e = None
    if not args.no_e2e:
        torch.cuda.empty_cache()
        E = args.e2e_turns
        zh = torch.empty(n, dtype=torch.float64, pin_memory=True)
        eh = torch.empty(n, dtype=torch.float64, pin_memory=True)
        g = torch.Generator().manual_seed(args.seed + rank)
        zh.copy_(torch.randn(n, dtype=torch.float64, generator=g) * cfg.sigma_z)
        eh.copy_(torch.randn(n, dtype=torch.float64, generator=g) * cfg.sigma_E)
        times = []
        for c in range(2):                               # the first call warms up
            torch.cuda.synchronize()
            dist.barrier()
            t0 = time.perf_counter()
            zd = zh.to("cuda", non_blocking=True)
            ed = eh.to("cuda", non_blocking=True)
            s2 = ShardedBunch(ctx, zd.data_ptr(), ed.data_ptr(), n, plan["first_particle"],
                              plan["n_global"], cfg.params, grid, wake=cfg.wake,
                              seed=args.seed + c, stream=stream.cuda_stream)
            c2, m2 = s2.buffers()
            for _ in range(E):
                s2.pass_()
                dist.all_reduce(c2)
                dist.all_reduce(m2)
                s2.bins()
            s2.finish()
            zh.copy_(zd)
            eh.copy_(ed)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            s2.close()
            del zd, ed, c2, m2
        te = torch.tensor([times[-1]], dtype=torch.float64, device="cuda")
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
        t_e2e = float(te.item())
        e2e = {"value": plan["n_global"] * E / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 16 * n, "turns_per_step": E,
               "seconds_per_step": t_e2e,
               "api": "haissinskijulia_b200.ShardedBunch (hj_bunch_create_shard, hj_bunch_pass, "
                      "NCCL all-reduce, hj_bunch_bins) per rank, host shards copied in and out"}
    if rank == 0:
        peak, peak_kind = measured_hbm_peak()
        achieved = BYTES_PER_PARTICLE_TURN * n / (pass_ms / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload(plan["n_global"], B, tps, logged=False),
                           parallelism=f"shard{world}",
                           particles_per_rank=n,
                           exchange="per turn: NCCL SUM all-reduce of the 3B+2 u64 bin "
                                    "exchange and of the 4 double sums (replaces the "
                                    "reference's MPI Allreduce/Scatterv/Gatherv/Bcast)",
                           turn_log="none in the sharded arm"),
            "roofline": {"bound": "hbm", "kernel": "k_track_pass", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "traffic": None, "algorithmic_bytes": BYTES_PER_PARTICLE_TURN * n,
                         "pass_ms": pass_ms, "max_over_ranks": True},
            "cpu_baseline": None, "e2e": e2e, "replicas": replicas,
            "gpu_launches": 4 * K * tps, "clocks": clock_info,
            "final": {"sigma_E": res.sigma_E, "sigma_z": res.sigma_z, "E0": res.E0},
        }
        print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    sharded = args.multi == "shard" and (world > 1 or args.shard_one_rank)
    if world > 1 or sharded:
        import datetime
        os.environ.setdefault("NCCL_DEBUG", "INFO")     # init lines show the rank count
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from haissinskijulia_b200 import (Context, Particles, ResidentBunch, benchmark_ring,
                                      create_simulation_buffers, longitudinal_evolve)
    from haissinskijulia_b200 import build as hjbuild
    hjbuild.build()

    n, B, K, W = int(args.particles), args.nbins, args.steps, args.warmup
    tps = args.turns_per_step
    cfg = benchmark_ring(n_turns=K * tps, nbins=B)
    ctx = Context(local)
    ctx.set_pass_layout(args.layout)
    stream = torch.cuda.current_stream()
    if sharded:
        clocks = ClockSampler(local)
        clocks.start()
        run_sharded(args, ctx, cfg, stream, rank, world, local, clocks)
        dist.barrier()
        dist.destroy_process_group()
        return
    gen = torch.Generator(device="cuda").manual_seed(args.seed + 7919 * rank)
    z = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) * cfg.sigma_z
    dE = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) * cfg.sigma_E
    bunch = ResidentBunch(ctx, z.data_ptr(), dE.data_ptr(), n, cfg.params, B, wake=cfg.wake,
                          seed=args.seed + rank, stream=stream.cuda_stream)
    # moments and line density logged on the device every 100 turns: each
    # step ends with one record
    bunch.set_log(LOG_EVERY, capacity=(K + W) * tps // LOG_EVERY + 1, density=True)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    bunch.advance(W * tps)
    barrier()
    bunch.set_profiling(True)
    clocks.mark()
    t_wall0 = time.perf_counter()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(K):
        bunch.advance(tps)
    ev1.record(stream)
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    clocks.mark()
    clock_info = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    prof = bunch.read_profile()
    log = bunch.read_log()
    res = bunch.finish()
    bunch.close()

    # the same pass with the opt-in single-precision excitation normals
    # (layout 23), for the cost of the default Float64 normals: 2 steps
    fast = None
    if args.layout == -1:
        ctx.set_pass_layout(23)
        fb = ResidentBunch(ctx, z.data_ptr(), dE.data_ptr(), n, cfg.params, B, wake=cfg.wake,
                           seed=args.seed + rank + 1, stream=stream.cuda_stream)
        fb.advance(tps)
        fb.set_profiling(True)
        fb.advance(2 * tps)
        fp = fb.read_profile()
        fb.finish()
        fb.close()
        ctx.set_pass_layout(args.layout)
        fpass = fp["pass_ms"] / max(fp["turns"], 1)
        fast = {"layout": 23, "pass_ms": fpass,
                "frac": BYTES_PER_PARTICLE_TURN * n / (fpass / 1e3) / 1e9 / measured_hbm_peak()[0],
                "turns": fp["turns"],
                "what": "k_track_pass with single-precision Box-Muller normals (opt-in layout "
                        "23) instead of the default Float64 ones, CUDA events, same bunch"}
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = n * K * tps * world / (ms / 1e3)

    # roofline of the dominant kernel (the fused particle pass)
    pass_ms = prof["pass_ms"] / max(prof["turns"], 1)
    bins_ms = prof["bins_ms"] / max(prof["turns"], 1)
    achieved = BYTES_PER_PARTICLE_TURN * n / (pass_ms / 1e3) / 1e9
    peak, peak_kind = measured_hbm_peak()
    tr, tr_src = PASS_DRAM_BYTES.get(B, (None, None))
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
            "config": dict(workload(n, B, tps),
                           parallelism="replicas" if world > 1 else "single GPU"),
            "roofline": roofline, "roofline_fast_normals": fast, "cpu_baseline": cpu,
            "e2e": e2e, "sweep": sweep,
            "gpu_launches": prof["launches"], "clocks": clock_info,
            "wall_seconds_timed": t_wall,
            "turn_log": {"every": LOG_EVERY, "records": int(log.shape[0]),
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
    if args.plan_only:
        run_plan(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
