"""The GPU library against the closed forms of tests/anchors.py, through the
C ABI: the small-amplitude synchrotron tune of a one-particle bunch, the
radiation equilibrium of a 4e6-particle bunch over four damping times with
on-device Philox excitation, and the wake potential of a single occupied
bin."""
import math

import numpy as np
import pytest
import torch

import anchors
from haissinskijulia_b200 import (BinGrid, ResidentBunch, WakeModel, benchmark_ring,
                                  create_simulation_buffers, wake_potential)

from gpu_util import device_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("voltage", [3e6, 5e6, 7e6])
def test_synchrotron_tune_of_a_small_orbit(gpu_ctx, voltage):
    cfg = benchmark_ring(voltage=voltage, use_wakefield=False, use_excitation=False)
    p = cfg.params.replace(SR_damping=False, update_E0=False)
    turns = 3000
    dz, de = device_pair(np.array([1e-5]), np.array([0.0]))
    b = ResidentBunch(gpu_ctx, dz.data_ptr(), de.data_ptr(), 1, p, 64, seed=1)
    b.set_log(1, capacity=turns)
    b.advance(turns)
    log = b.read_log()
    b.finish()
    b.close()
    assert log.shape[0] == turns and np.array_equal(log[:, 0], np.arange(1, turns + 1))
    zs = np.concatenate([[1e-5], log[:, 4]])          # mean z of a one-particle bunch
    ab = 2.0 - anchors.synchrotron_trace(p)
    assert abs((2.0 - anchors.trace_from_orbit(zs)) - ab) <= 1e-6 * ab


def test_radiation_equilibrium_spreads(gpu_ctx):
    """σ_z and σ_E of a bunch started in the linear equilibrium, averaged over
    20,000 turns (logged every 10 turns), against the Lyapunov solution
    within 3/sqrt(2N), three standard errors of one snapshot's estimate."""
    cfg = benchmark_ring(use_wakefield=False, use_excitation=True)
    p = cfg.params.replace(update_E0=False)
    n, turns = 4_000_000, 20_000
    S = anchors.equilibrium_covariance(p, cfg.sigma_E)
    x = np.random.default_rng(5).multivariate_normal([0.0, 0.0], S, size=n)
    dz, de = device_pair(np.ascontiguousarray(x[:, 0]), np.ascontiguousarray(x[:, 1]))
    b = ResidentBunch(gpu_ctx, dz.data_ptr(), de.data_ptr(), n, p, 64, seed=21)
    b.set_log(10, capacity=turns // 10)
    b.advance(turns)
    log = b.read_log()
    r = b.finish()
    b.close()
    assert log.shape[0] == turns // 10
    S = anchors.equilibrium_covariance(p, r.sigma_E0_initial)
    tol = 3.0 / math.sqrt(2.0 * n)
    assert abs(math.sqrt(np.mean(log[:, 2] ** 2) / S[0, 0]) - 1.0) <= tol
    assert abs(math.sqrt(np.mean(log[:, 3] ** 2) / S[1, 1]) - 1.0) <= tol


@pytest.mark.parametrize("B", [16384, 4096, 1000, 5])
def test_single_bin_wake_potential(gpu_ctx, B):
    buf = create_simulation_buffers(1, B, ctx=gpu_ctx)
    for wake in (benchmark_ring().wake, WakeModel.reference(benchmark_ring().params)):
        grid = BinGrid.make(4e-3, B, wake.half_width_sigmas)
        for j0 in sorted({0, 1, B // 2 - 1, B // 2, B - 1}):
            counts = np.zeros(B, np.int64)
            counts[j0] = 12345
            cur = 2.9e-15
            want = anchors.single_bin_potential(grid.centers, j0, wake, cur)
            full = cur * np.abs(anchors.wake_function(grid.centers, wake)).max() / (
                math.sqrt(2 * math.pi) * wake.delta_std)
            got = wake_potential(counts, grid, wake, cur, buf)
            assert np.abs(got - want).max() <= 1e-13 * full, (B, j0)
