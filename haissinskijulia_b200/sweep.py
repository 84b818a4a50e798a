"""Parameter sweeps and served solves over batches of bunches.

The reference scans parameters one point after another
(src/parameter_sensitivity/scan.jl:182-184, each point a full
longitudinal_evolve!).  Here every point is a bunch of its own (particles,
RF voltage, intensity, bins, seed, turns) and all live points advance
together in a Batch: one batched particle pass, one histogram merge and one
batched bins step per turn, turn blocks replayed from a CUDA graph.

* `sweep_points` / `intensity_scan`: the ragged 256-point sweep and the
  32-bunch intensity scan, seeded.
* `run_batched`: admits points as slots and pool space free up, advances in
  blocks of K turns, retires finished points.
* `run_plain`: the same points one after another on the plain resident path
  (the baseline the batch is measured against).
* `autotune`: times candidate (particles per block, pass layout with the
  width of the shared-memory bin counters -- the histogram privatisation --,
  K) on a sample of the workload and keeps the fastest.
* `serve_plain`: the same stream one request at a time on the plain path
  (first come first served), the baseline of `serve`; `plain_service` and
  `plain_timeline` split it so that one set of measured service times serves
  every arrival rate of the same requests.
* `serve`: a request stream with arrival times; requests are admitted by
  device-memory footprint (16 B per particle plus bin tables) while others
  run, and per-request latency percentiles are reported with solves/s.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from .api import Batch, Context, HaissinskiError, ResidentBunch, gaussian_bunch
from . import _lib
from .rings import RingConfig, benchmark_ring


@dataclass
class Point:
    """One solve: a bunch of n particles of a ring, run for `turns` turns."""
    n: int
    voltage: float
    population: float
    nbins: int
    turns: int
    seed: int
    arrival: float = 0.0          # seconds after the stream starts (served solves)

    def ring(self) -> RingConfig:
        return benchmark_ring(n_turns=self.turns, nbins=self.nbins, population=self.population,
                              voltage=self.voltage)

    def spreads(self):
        """Initial spreads: σ_z = 4 mm, σ_E/E = 1e-3 (independent Gaussians,
        generated on the device from the point's seed)."""
        cfg = self.ring()
        return cfg.sigma_z, cfg.sigma_E

    def footprint(self) -> int:
        """Device bytes while resident: 16 B per particle plus the bin tables."""
        return 16 * self.n + 400 * self.nbins + (1 << 16)


@dataclass
class Solve:
    point: Point
    result: object
    z: Optional[np.ndarray] = None
    dE: Optional[np.ndarray] = None
    admitted: float = 0.0
    finished: float = 0.0


def _log_uniform(rng, lo, hi, size=None):
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size))


def sweep_points(n_points: int = 256, seed: int = 2024, turns: int = 5000,
                 nbins: int = 4096, n_lo: float = 1e4, n_hi: float = 2e6) -> List[Point]:
    """The ragged sweep: V ~ U[3, 7] MV, population log-uniform in [1e9, 1e11]
    electrons, particles log-uniform in [n_lo, n_hi], own seed per point."""
    rng = np.random.default_rng(seed)
    v = rng.uniform(3e6, 7e6, n_points)
    pop = _log_uniform(rng, 1e9, 1e11, n_points)
    n = np.round(_log_uniform(rng, n_lo, n_hi, n_points)).astype(np.int64)
    return [Point(int(n[i]), float(v[i]), float(pop[i]), nbins, turns, seed * 1000 + i)
            for i in range(n_points)]


def intensity_scan(n_bunches: int = 32, n: int = 1_000_000, turns: int = 5000,
                   nbins: int = 8192, seed: int = 7) -> List[Point]:
    """32 bunches of 1e6 particles, populations log-spaced over [1e9, 1e11]."""
    pops = np.logspace(9, 11, n_bunches)
    return [Point(n, 5e6, float(p), nbins, turns, seed * 1000 + i) for i, p in enumerate(pops)]


def request_stream(n_requests: int, rate: float = 50.0, seed: int = 11,
                   n_hi: float = 4e6) -> List[Point]:
    """Served solves: Poisson arrivals at `rate`/s, V ~ U[3, 7] MV, population
    log-uniform [1e9, 1e11], particles log-uniform [1e4, n_hi], turns
    uniform [1000, 20000], bins in {2048, 4096, 8192}."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    out = []
    for i in range(n_requests):
        out.append(Point(int(round(_log_uniform(rng, 1e4, n_hi))), float(rng.uniform(3e6, 7e6)),
                         float(_log_uniform(rng, 1e9, 1e11)), int(rng.choice([2048, 4096, 8192])),
                         int(rng.integers(1000, 20001)), seed * 100000 + i, float(t[i])))
    return out


@dataclass
class Tuning:
    chunk: int = 65536
    layout: int = -1
    graph_turns: int = 16
    resident: bool = False      # resident blocks on a chunk queue, or one block per chunk


def run_batched(ctx: Context, points: List[Point], *, pool_particles: Optional[int] = None,
                max_bunches: Optional[int] = None, tuning: Tuning = Tuning(),
                block_turns: int = 64, copy_out: bool = False) -> List[Solve]:
    """All points through one Batch: admit while there is room, advance in
    blocks, take finished points, admit the rest.  Returns the solves in the
    order of `points`."""
    max_b = max(p.nbins for p in points)
    pool = pool_particles or sum(p.n + 4 for p in points)
    slots = max_bunches or len(points)
    bt = Batch(ctx, pool, slots, max_b, chunk=tuning.chunk, layout=tuning.layout,
               graph_turns=tuning.graph_turns, resident=tuning.resident)
    pending = list(range(len(points)))
    live: Dict[int, int] = {}
    out: List[Optional[Solve]] = [None] * len(points)
    t0 = time.perf_counter()
    try:
        while pending or live:
            while pending:
                i = pending[0]
                p = points[i]
                cfg = p.ring()
                try:
                    bid = bt.add_gaussian(p.n, cfg.sigma_z, cfg.sigma_E, p.seed, cfg.params,
                                          p.nbins, wake=cfg.wake, seed=p.seed, turns=p.turns)
                except HaissinskiError as e:
                    if e.status == _lib.HJ_ERR_FULL and live:
                        break
                    raise
                live[bid] = i
                out[i] = Solve(p, None, admitted=time.perf_counter() - t0)
                pending.pop(0)
            bt.advance(block_turns)
            for bid in bt.poll():
                i = live.pop(bid)
                z, dE, r = bt.take(bid, copy_out=copy_out)
                s = out[i]
                s.result, s.z, s.dE = r, z, dE
                s.finished = time.perf_counter() - t0
    finally:
        bt.close()
    return out


def run_plain(ctx: Context, points: List[Point], copy_out: bool = False) -> List[Solve]:
    """The points one after another on the plain resident path."""
    import torch
    out = []
    t0 = time.perf_counter()
    for p in points:
        cfg = p.ring()
        dz = torch.empty(p.n, dtype=torch.float64, device="cuda")
        de = torch.empty_like(dz)
        gaussian_bunch(ctx, p.seed, p.n, cfg.sigma_z, cfg.sigma_E, dz.data_ptr(), de.data_ptr())
        a = time.perf_counter() - t0
        b = ResidentBunch(ctx, dz.data_ptr(), de.data_ptr(), p.n, cfg.params, p.nbins,
                          wake=cfg.wake, seed=p.seed)
        b.advance(p.turns)
        r = b.finish()
        b.close()
        s = Solve(p, r, admitted=a)
        if copy_out:
            s.z, s.dE = dz.cpu().numpy(), de.cpu().numpy()
        s.finished = time.perf_counter() - t0
        out.append(s)
    return out


def wave_chunks(points: List[Point], num_sms: int, waves=(1, 2, 4)) -> List[int]:
    """Particles per block that split the whole workload into `waves` full
    waves of `num_sms` blocks (rounded up to a multiple of 4)."""
    total = sum(p.n for p in points)
    out = []
    for w in waves:
        c = -(-total // (num_sms * w))
        c = min(max((c + 3) // 4 * 4, 4096), (1 << 20) - 8)   # a block counts < 2^20
        out.append(int(c))
    return out


def autotune(ctx: Context, points: List[Point], *, trial_turns: int = 64,
             chunks=None, layouts=(8, 9, 13), graph_turns=(8, 32),
             sample: int = 64) -> Tuning:
    """Times each candidate (particles per block, pass layout, graph turns) on
    up to `sample` of the points for `trial_turns` turns after a warm-up and
    returns the fastest.  Default block sizes: 16K, 64K, 256K particles and,
    when the trial runs the whole workload, those that fill one, two or four
    waves of the GPU with it (on a sample they would be sized for the sample)."""
    if chunks is None:
        chunks = [16384, 65536, 262144]
        if len(points) <= sample:
            import torch
            dev = torch.cuda.current_device()
            sms = torch.cuda.get_device_properties(dev).multi_processor_count
            chunks = sorted(set(chunks + wave_chunks(points, sms)))
    pts = points[:sample]
    pool = sum(p.n + 4 for p in pts)
    best, best_t = Tuning(), float("inf")
    data = [(p, p.ring()) for p in pts]
    for c in chunks:
        for L in layouts:
            for K in graph_turns:
                bt = Batch(ctx, pool, len(pts), max(p.nbins for p in pts), chunk=c, layout=L,
                           graph_turns=K)
                try:
                    for p, cfg in data:
                        bt.add_gaussian(p.n, cfg.sigma_z, cfg.sigma_E, p.seed, cfg.params,
                                        p.nbins, wake=cfg.wake, seed=p.seed,
                                        turns=10 * trial_turns)
                    bt.advance(K)
                    bt.poll()
                    t0 = time.perf_counter()
                    bt.advance(trial_turns)
                    bt.poll()
                    el = time.perf_counter() - t0
                finally:
                    bt.close()
                if el < best_t:
                    best, best_t = Tuning(c, L, K), el
    return best


@dataclass
class ServeReport:
    solves: List[Solve] = field(default_factory=list)
    wall: float = 0.0

    def latencies(self) -> np.ndarray:
        return np.array([s.finished - s.point.arrival for s in self.solves])

    def summary(self) -> dict:
        lat = self.latencies()
        return {"requests": len(self.solves), "solves_per_s": len(self.solves) / self.wall,
                "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)), "wall_s": self.wall,
                "particle_turns": float(sum(s.point.n * s.point.turns for s in self.solves))}


def serve(ctx: Context, requests: List[Point], *, memory_budget: int = 8 << 30,
          max_bunches: int = 256, tuning: Tuning = Tuning(), block_turns: int = 200,
          max_nbins: int = 8192) -> ServeReport:
    """Continuous batching of a request stream.  A request becomes admissible
    at its arrival time (wall clock from the start) and is admitted when its
    footprint fits the memory budget and a slot is free; admitted requests
    run together, each for its own number of turns; finished ones are retired
    between turn blocks and their slots reused.  Latency = finish - arrival."""
    pool = memory_budget // 16
    bt = Batch(ctx, pool, max_bunches, max_nbins, chunk=tuning.chunk, layout=tuning.layout,
               graph_turns=tuning.graph_turns, resident=tuning.resident)
    waiting = list(range(len(requests)))
    live: Dict[int, int] = {}
    used = 0
    rep = ServeReport()
    done: Dict[int, Solve] = {}
    t0 = time.perf_counter()
    try:
        while waiting or live:
            now = time.perf_counter() - t0
            while waiting and requests[waiting[0]].arrival <= now:
                i = waiting[0]
                p = requests[i]
                if used + p.footprint() > memory_budget and live:
                    break
                cfg = p.ring()
                try:
                    bid = bt.add_gaussian(p.n, cfg.sigma_z, cfg.sigma_E, p.seed, cfg.params,
                                          p.nbins, wake=cfg.wake, seed=p.seed, turns=p.turns)
                except HaissinskiError as e:
                    if e.status == _lib.HJ_ERR_FULL and live:
                        break
                    raise
                used += p.footprint()
                live[bid] = i
                done[i] = Solve(p, None, admitted=time.perf_counter() - t0)
                waiting.pop(0)
            if not live:
                time.sleep(max(0.0, min(0.01, requests[waiting[0]].arrival - now)))
                continue
            bt.advance(block_turns)
            for bid in bt.poll():
                i = live.pop(bid)
                _, _, r = bt.take(bid, copy_out=False)
                s = done[i]
                s.result = r
                s.finished = time.perf_counter() - t0
                used -= s.point.footprint()
        rep.wall = time.perf_counter() - t0
    finally:
        bt.close()
    rep.solves = [done[i] for i in sorted(done)]
    return rep


def plain_service(ctx: Context, requests: List[Point]) -> List[Solve]:
    """Each request solved alone on the plain resident path; Solve.finished
    is its measured service time (bunch generation, turns, result)."""
    return [run_plain(ctx, [p])[0] for p in requests]


def plain_timeline(requests: List[Point], service: List[Solve]) -> ServeReport:
    """First come first served on one plain solver: a request starts when it
    has arrived and the previous one has finished, and takes its measured
    service time (latency = finish - arrival on that timeline; no idle time is
    spent waiting for arrivals)."""
    rep = ServeReport()
    clock = 0.0
    for k in sorted(range(len(requests)), key=lambda q: requests[q].arrival):
        p, s = requests[k], service[k]
        start = max(clock, p.arrival)
        clock = start + s.finished
        rep.solves.append(Solve(p, s.result, admitted=start, finished=clock))
    rep.wall = clock
    return rep


def serve_plain(ctx: Context, requests: List[Point]) -> ServeReport:
    """The same request stream served one request at a time on the plain
    resident path (plain_service, then plain_timeline)."""
    return plain_timeline(requests, plain_service(ctx, requests))


def time_batch_turns(ctx: Context, points: List[Point], turns: int, tuning: Tuning) -> float:
    """Seconds per turn of all `points` live in one Batch (after a warm-up of
    one graph block); the points are given enough turns not to finish."""
    bt = Batch(ctx, sum(p.n + 4 for p in points), len(points), max(p.nbins for p in points),
               chunk=tuning.chunk, layout=tuning.layout, graph_turns=tuning.graph_turns,
               resident=tuning.resident)
    try:
        for p in points:
            cfg = p.ring()
            bt.add_gaussian(p.n, cfg.sigma_z, cfg.sigma_E, p.seed, cfg.params, p.nbins,
                            wake=cfg.wake, seed=p.seed, turns=10 * turns + 10 * tuning.graph_turns)
        bt.advance(max(tuning.graph_turns, 1))
        bt.poll()
        t0 = time.perf_counter()
        bt.advance(turns)
        bt.poll()
        return (time.perf_counter() - t0) / turns
    finally:
        bt.close()


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="Time batched turns of the 256-point sweep")
    ap.add_argument("--turns", type=int, default=64)
    ap.add_argument("--chunk", type=int, default=65536)
    ap.add_argument("--layout", type=int, default=-1)
    ap.add_argument("--graph-turns", type=int, default=8)
    ap.add_argument("--resident", type=int, default=0)
    args = ap.parse_args()
    s = time_batch_turns(Context(0), sweep_points(256), args.turns,
                         Tuning(args.chunk, args.layout, args.graph_turns, bool(args.resident)))
    print(f"{s * 1e3:.3f} ms per batched turn of the 256-point sweep")
