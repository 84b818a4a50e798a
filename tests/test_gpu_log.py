"""Turn log (hj_bunch_set_log / read_log) against the oracle at the same turns."""
import numpy as np
import pytest
import torch

from haissinskijulia_b200 import ResidentBunch, benchmark_ring

from gpu_util import device_pair

pytestmark = pytest.mark.gpu


def test_log_records_match_the_oracle(gpu_ctx, oracle):
    cfg = benchmark_ring(n_turns=20, nbins=1024)
    n, turns, every = 30_001, 20, 5
    rng = np.random.default_rng(8)
    z0 = rng.normal(0.0, cfg.sigma_z, n)
    e0 = rng.normal(0.0, cfg.sigma_E, n)
    draws = rng.standard_normal((turns, n))
    from haissinskijulia_b200 import BinGrid
    grid = BinGrid.make(oracle.global_std(z0), cfg.nbins, cfg.wake.half_width_sigmas)
    dz, de = device_pair(z0, e0)
    dd = torch.from_numpy(draws).cuda()
    b = ResidentBunch(gpu_ctx, dz.data_ptr(), de.data_ptr(), n, cfg.params, cfg.nbins,
                      wake=cfg.wake, grid=grid, seed=1)
    b.set_draws(dd.data_ptr(), 1, turns)
    b.set_log(every, capacity=3, density=True)      # a ring shorter than the run
    b.advance(turns)
    log = b.read_log()
    assert log.shape == (3, 8 + cfg.nbins)
    assert list(log[:, 0]) == [10.0, 15.0, 20.0]
    zo, eo = z0.copy(), e0.copy()
    st = oracle.state(zo, eo, cfg.params.to_c(), cfg.wake.to_c(), cfg.nbins, grid.to_c())
    rows = {}
    for t in range(1, turns + 1):
        assert st.turn(np.ascontiguousarray(draws[t - 1])) == 0
        if t % every == 0:
            r = st.result()
            rows[t] = (st.E0, r.sigma_z, r.sigma_E, r.mean_z, r.mean_dE, st.counts().copy())
    for rec in log:
        E0, sz, sE, mz, mE, counts = rows[int(rec[0])]
        assert rec[1] == pytest.approx(E0, rel=1e-12)
        assert rec[2] == pytest.approx(sz, rel=1e-12)
        assert rec[3] == pytest.approx(sE, rel=1e-12)
        assert abs(rec[4] - mz) <= 1e-12 * cfg.sigma_z
        assert abs(rec[5] - mE) <= 1e-12 * cfg.sigma_E
        assert rec[7] == counts.sum()
        assert np.array_equal(rec[8:].astype(np.int64), counts)
    b.close()
