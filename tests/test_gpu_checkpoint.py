"""Checkpoint and resume of a resident bunch (hj_bunch_checkpoint /
hj_bunch_resume): a run continued from a checkpoint in a new bunch ends where
the uninterrupted run ends (same Philox draws; the grid and the excitation
amplitude from the checkpointed initial spreads)."""
import numpy as np
import pytest
import torch

from haissinskijulia_b200 import HaissinskiError, ResidentBunch, benchmark_ring

from gpu_util import assert_close, device_pair

pytestmark = pytest.mark.gpu


def test_a_resumed_run_continues_the_run(gpu_ctx):
    cfg = benchmark_ring(n_turns=1, nbins=2048)
    n = 200_003
    rng = np.random.default_rng(21)
    z0, e0 = rng.normal(0.0, cfg.sigma_z, n), rng.normal(0.0, cfg.sigma_E, n)
    dz, de = device_pair(z0, e0)
    a = ResidentBunch(gpu_ctx, dz.data_ptr(), de.data_ptr(), n, cfg.params, 2048, wake=cfg.wake,
                      seed=17)
    a.advance(13)
    cz = torch.empty(n, dtype=torch.float64, device="cuda")
    ce = torch.empty_like(cz)
    cp = a.checkpoint(cz.data_ptr(), ce.data_ptr())
    assert cp.turn == 14 and cp.E0 != cfg.params.E0
    a.advance(12)
    ra = a.finish()
    counts_a = a.histogram()
    a.close()

    b = ResidentBunch.resume(gpu_ctx, cz.data_ptr(), ce.data_ptr(), n, cfg.params, 2048, cp,
                             wake=cfg.wake, seed=17)
    b.advance(12)
    rb = b.finish()
    counts_b = b.histogram()
    b.close()
    assert ra.turns == rb.turns == 25
    assert rb.E0 == pytest.approx(ra.E0, rel=1e-12)
    assert rb.sigma_E == pytest.approx(ra.sigma_E, rel=1e-12)
    assert rb.sigma_z == pytest.approx(ra.sigma_z, rel=1e-12)
    assert (rb.sigma_E0_initial, rb.sigma_z0_initial) == (ra.sigma_E0_initial, ra.sigma_z0_initial)
    assert_close(cz.cpu().numpy(), dz.cpu().numpy(), cfg.sigma_z, what="z")
    assert_close(ce.cpu().numpy(), de.cpu().numpy(), cfg.sigma_E, what="dE")
    # same particles within 1e-12: the line density is the same, up to a
    # particle sitting on a bin edge
    assert counts_b.sum() == counts_a.sum()
    assert np.abs(counts_b - counts_a).max() <= 1


def test_resume_needs_a_checkpoint(gpu_ctx):
    from haissinskijulia_b200.api import Checkpoint
    cfg = benchmark_ring(n_turns=1, nbins=256)
    dz, de = device_pair(np.zeros(8), np.zeros(8))
    with pytest.raises(HaissinskiError):
        ResidentBunch.resume(gpu_ctx, dz.data_ptr(), de.data_ptr(), 8, cfg.params, 256,
                             Checkpoint(0, 4e9, 1.0, 1.0), wake=cfg.wake)
