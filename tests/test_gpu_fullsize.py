"""Parity at the full benchmark size: 1e8 particles, 16384 bins.

Two turns of the whole bunch with host-fed quantum-excitation draws, on the
device (fused pass) and in the oracle: every particle within 1e-12, the bin
counts bit-exact, and the E0 track identical to 1e-12."""
import os

import numpy as np
import pytest
import torch

from haissinskijulia_b200 import BinGrid, ResidentBunch, benchmark_ring

from gpu_util import RTOL, assert_close

pytestmark = pytest.mark.gpu

N = 100_000_000
NBINS = 16_384
TURNS = 2


def test_two_turns_of_the_full_bunch(gpu_ctx):
    from oracle import Oracle
    orc = Oracle(threads=os.cpu_count() or 1)
    cfg = benchmark_ring(n_turns=TURNS, nbins=NBINS)
    rng = np.random.default_rng(314)
    z0 = rng.normal(0.0, cfg.sigma_z, N)
    dE0 = rng.normal(0.0, cfg.sigma_E, N)
    grid = BinGrid.make(cfg.sigma_z, NBINS, cfg.wake.half_width_sigmas)

    dz = torch.from_numpy(z0).cuda()
    de = torch.from_numpy(dE0).cuda()
    b = ResidentBunch(gpu_ctx, dz.data_ptr(), de.data_ptr(), N, cfg.params, NBINS,
                      wake=cfg.wake, grid=grid, seed=1)
    st = orc.state(z0, dE0, cfg.params.to_c(), cfg.wake.to_c(), NBINS, grid.to_c())
    for t in range(1, TURNS + 1):
        draws = rng.standard_normal(N)
        ddraws = torch.from_numpy(draws).cuda()
        b.set_draws(ddraws.data_ptr(), t, 1)
        b.advance(1)
        assert st.turn(draws) == 0
        r = b.observe()
        assert abs(r.E0 - st.E0) / st.E0 <= RTOL, f"E0 turn {t}"
        counts = b.histogram()
        assert counts.sum() > 0.99 * N
        assert np.array_equal(counts, st.counts()), f"counts turn {t}"
        del ddraws
    zg = torch.empty_like(dz)
    eg = torch.empty_like(de)
    b.observe(zg.data_ptr(), eg.data_ptr())
    zh, eh = zg.cpu().numpy(), eg.cpu().numpy()
    assert np.array_equal(b.histogram(), orc.histogram(zh, grid.to_c()))
    b.close()
    assert_close(zh, z0, cfg.sigma_z, what="z")        # z0/dE0 were advanced by the oracle
    assert_close(eh, dE0, cfg.sigma_E, what="dE")
