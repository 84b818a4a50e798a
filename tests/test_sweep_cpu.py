"""Host logic of haissinskijulia_b200.sweep on the CPU: the seeded workloads,
the block sizes autotune tries, the serving report, and the first come first
served timeline of serve_plain with the solves replaced by a fake of fixed
service times."""
import math

import numpy as np
import pytest

from haissinskijulia_b200 import sweep
from haissinskijulia_b200.sweep import (Point, ServeReport, Solve, intensity_scan,
                                        request_stream, sweep_points, wave_chunks)


def test_sweep_points_are_seeded_and_in_range():
    a = sweep_points(256)
    assert a == sweep_points(256)
    assert len({p.seed for p in a}) == 256
    for p in a:
        assert 3e6 <= p.voltage <= 7e6 and 1e9 <= p.population <= 1e11
        assert 1e4 <= p.n <= 2e6 and p.nbins == 4096 and p.turns == 5000
    n = np.array([p.n for p in a])
    # log-uniform particles: the median sits near the geometric mean of the range
    assert abs(math.log(np.median(n)) - 0.5 * math.log(1e4 * 2e6)) < 0.5
    assert sweep_points(8, seed=1) != sweep_points(8, seed=2)


def test_intensity_scan_is_log_spaced():
    pts = intensity_scan()
    pops = np.array([p.population for p in pts])
    assert len(pts) == 32 and all(p.n == 1_000_000 and p.nbins == 8192 for p in pts)
    assert pops[0] == pytest.approx(1e9) and pops[-1] == pytest.approx(1e11)
    assert np.allclose(np.diff(np.log(pops)), math.log(100) / 31)


def test_request_stream_is_seeded_and_in_range():
    r = request_stream(40)
    assert r == request_stream(40)
    t = np.array([p.arrival for p in r])
    assert np.all(np.diff(t) > 0) and t[0] > 0
    for p in r:
        assert 1e4 <= p.n <= 4e6 and p.nbins in (2048, 4096, 8192)
        assert 1000 <= p.turns <= 20000 and 3e6 <= p.voltage <= 7e6
    long = request_stream(4000, rate=50.0)
    gaps = np.diff([p.arrival for p in long])
    assert abs(gaps.mean() - 1 / 50) < 5 * gaps.std() / math.sqrt(gaps.size)


@pytest.mark.parametrize("total", [10, 4096 * 148, 10**8, 10**10])
def test_wave_chunks_are_legal_block_sizes(total):
    pts = [Point(total, 5e6, 1e10, 4096, 10, 1)]
    for w, c in zip((1, 2, 4), wave_chunks(pts, 148)):
        assert c % 4 == 0 and 4096 <= c <= (1 << 20) - 8
        if 4096 < c < (1 << 20) - 8:                 # unclamped: fills the waves
            assert c * 148 * w >= total > (c - 4) * 148 * w


def test_footprint_counts_particles_and_bins():
    p = Point(1000, 5e6, 1e10, 2048, 10, 1)
    assert p.footprint() == 16 * 1000 + 400 * 2048 + (1 << 16)


def test_serve_report_summary():
    rep = ServeReport()
    for i, (arr, fin) in enumerate([(0.0, 1.0), (0.5, 2.0), (1.0, 4.0)]):
        rep.solves.append(Solve(Point(10, 5e6, 1e10, 64, 10, i, arrival=arr), None,
                                admitted=arr, finished=fin))
    rep.wall = 4.0
    s = rep.summary()
    assert s["requests"] == 3 and s["solves_per_s"] == pytest.approx(0.75)
    assert s["p50_latency_s"] == pytest.approx(1.5)       # latencies 1.0, 1.5, 3.0
    assert s["p99_latency_s"] == pytest.approx(np.percentile([1.0, 1.5, 3.0], 99))
    assert s["particle_turns"] == 300


def test_serve_plain_timeline(monkeypatch):
    """Requests start when they have arrived and the previous one is done."""
    service = {0: 0.5, 1: 0.2, 2: 1.0, 3: 0.1}

    def fake_run_plain(ctx, points):
        p = points[0]
        return [Solve(p, ("result", p.seed), admitted=0.0, finished=service[p.seed])]

    monkeypatch.setattr(sweep, "run_plain", fake_run_plain)
    reqs = [Point(10, 5e6, 1e10, 64, 10, s, arrival=a)
            for s, a in [(2, 0.6), (0, 0.0), (3, 3.0), (1, 0.1)]]
    rep = sweep.serve_plain(None, reqs)
    got = [(sv.point.seed, sv.admitted, sv.finished) for sv in rep.solves]
    want = [(0, 0.0, 0.5), (1, 0.5, 0.7), (2, 0.7, 1.7), (3, 3.0, 3.1)]
    assert [g[0] for g in got] == [w[0] for w in want]
    for g, w in zip(got, want):
        assert g[1] == pytest.approx(w[1]) and g[2] == pytest.approx(w[2])
    assert rep.wall == pytest.approx(3.1)
    assert all(sv.result == ("result", sv.point.seed) for sv in rep.solves)


def test_request_streams_at_other_rates_hold_the_same_requests():
    """The serving curve reuses one set of plain service times for every
    offered load: only the arrival times scale with the rate."""
    a, b = request_stream(100, rate=5.0), request_stream(100, rate=50.0)
    assert [(p.n, p.turns, p.nbins, p.voltage, p.seed) for p in a] == \
        [(p.n, p.turns, p.nbins, p.voltage, p.seed) for p in b]
    assert np.allclose([p.arrival for p in a], [10.0 * p.arrival for p in b])


def test_plain_timeline_reuses_service_times():
    reqs = [Point(10, 5e6, 1e10, 64, 10, s, arrival=a) for s, a in [(0, 0.0), (1, 0.1)]]
    service = [Solve(reqs[0], "r0", finished=0.5), Solve(reqs[1], "r1", finished=0.2)]
    rep = sweep.plain_timeline(reqs, service)
    assert [(s.admitted, s.finished, s.result) for s in rep.solves] == \
        [(0.0, 0.5, "r0"), (0.5, pytest.approx(0.7), "r1")]


def test_stratified_sample_follows_the_particle_distribution():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import bench
    pts = sweep_points(256)
    idx = bench.stratified_sample(pts, 32)
    assert len(set(idx)) == 32 and idx == sorted(idx)
    n_all = np.sort([p.n for p in pts])
    n_s = np.sort([pts[i].n for i in idx])
    # the j-th sampled count is the middle of the j-th eighth-of-a-percentile stratum
    assert np.array_equal(n_s, n_all[[int((j + 0.5) * 8) for j in range(32)]])
    assert abs(math.log(n_s.mean() / n_all.mean())) < 0.1
