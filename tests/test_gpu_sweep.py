"""Sweeps and served solves (haissinskijulia_b200.sweep) on small workloads.

* run_batched against run_plain (one point after another on the resident
  path): every point's E0, σ_E and σ_z within 1e-12;
* serve(): requests that arrive while others run are admitted into the same
  batch, and each request's result is bit-identical to the same request
  solved alone;
* serve_plain(): the same stream one request at a time on the plain path
  gives every request's result within 1e-12 of serve()'s, on a first come
  first served timeline.
"""
import pytest

from haissinskijulia_b200.sweep import (Tuning, request_stream, run_batched, run_plain, serve,
                                        serve_plain, sweep_points)

pytestmark = pytest.mark.gpu


def _same(a, b, rel):
    for k in ("E0", "sigma_E", "sigma_z"):
        assert getattr(a, k) == pytest.approx(getattr(b, k), rel=rel), k
    assert abs(a.mean_z - b.mean_z) <= rel * a.sigma_z
    assert abs(a.mean_dE - b.mean_dE) <= rel * a.sigma_E


def test_batched_sweep_matches_plain_points(gpu_ctx):
    pts = sweep_points(10, seed=3, turns=60, nbins=1024, n_lo=1e3, n_hi=2e5)
    batched = run_batched(gpu_ctx, pts, max_bunches=4, tuning=Tuning(16384, -1, 8),
                          block_turns=25)
    plain = run_plain(gpu_ctx, pts)
    for b, p in zip(batched, plain):
        assert b.point is p.point and b.result is not None
        _same(b.result, p.result, 1e-12)


def test_served_requests_match_their_solo_runs(gpu_ctx):
    reqs = request_stream(8, rate=400.0, seed=5, n_hi=3e4)
    for r in reqs:                      # short runs so the test stays small
        r.turns = 150 + (r.seed % 7) * 20
        r.nbins = [512, 1024, 2048][r.seed % 3]
    rep = serve(gpu_ctx, reqs, memory_budget=64 << 20, max_bunches=4,
                tuning=Tuning(16384, -1, 8), block_turns=40, max_nbins=2048)
    s = rep.summary()
    assert s["requests"] == len(reqs) and s["p99_latency_s"] >= s["p50_latency_s"] > 0
    # at least one request was admitted while another was on the GPU
    assert any(b.admitted < a.finished and b.admitted > a.admitted
               for a in rep.solves for b in rep.solves)
    for sv in rep.solves:
        alone = run_batched(gpu_ctx, [sv.point], tuning=Tuning(16384, -1, 8), block_turns=40)[0]
        assert (alone.result.E0, alone.result.sigma_E, alone.result.sigma_z) == \
            (sv.result.E0, sv.result.sigma_E, sv.result.sigma_z)


def test_plain_serving_matches_batched_serving(gpu_ctx):
    reqs = request_stream(6, rate=400.0, seed=9, n_hi=3e4)
    for r in reqs:
        r.turns = 120 + (r.seed % 5) * 20
        r.nbins = [512, 1024][r.seed % 2]
    rep = serve(gpu_ctx, reqs, memory_budget=64 << 20, max_bunches=4,
                tuning=Tuning(16384, -1, 8), block_turns=40, max_nbins=1024)
    plain = serve_plain(gpu_ctx, reqs)
    s = plain.summary()
    assert s["requests"] == len(reqs) and s["p99_latency_s"] >= s["p50_latency_s"] > 0
    by_point = {id(sv.point): sv for sv in rep.solves}
    prev = 0.0
    for pv in plain.solves:             # first come first served: finishes in arrival order
        assert pv.admitted >= pv.point.arrival and pv.finished > pv.admitted >= prev
        prev = pv.finished
        _same(by_point[id(pv.point)].result, pv.result, 1e-12)
