"""The oracle against closed forms derived by hand from the reference's
formulas (tests/anchors.py): the small-amplitude synchrotron tune, the
radiation equilibrium of the energy spread and bunch length, and the wake
potential of a single occupied bin.  These pin the oracle to the physics of
the reference's equations independently of the restatements in
tests/golden/, which were written from the same reading of the source."""
import math

import numpy as np
import pytest

import anchors
from haissinskijulia_b200 import BinGrid, WakeModel, benchmark_ring
from oracle import Oracle
from oracle.pyoracle import CONV_DIRECT_LD


def _orbit(params, z0, turns, threads=1):
    orc = Oracle(threads=threads)
    z, e = np.array([z0]), np.array([0.0])
    st = orc.state(z, e, params.to_c(), None, 64)
    zs = [z0]
    for _ in range(turns):
        assert st.turn(None) == 0
        zs.append(float(st.z[0]))
    st.close()
    return np.array(zs)


@pytest.mark.parametrize("voltage", [3e6, 5e6, 7e6])
def test_synchrotron_tune_of_a_small_orbit(voltage):
    cfg = benchmark_ring(voltage=voltage, use_wakefield=False, use_excitation=False)
    p = cfg.params.replace(SR_damping=False, update_E0=False)
    zs = _orbit(p, 1e-5, 3000)
    ab = 2.0 - anchors.synchrotron_trace(p)
    ab_orbit = 2.0 - anchors.trace_from_orbit(zs)
    # the RF sine's curvature and η(ΔE) shift it by ~(k z)^2 ~ 1e-8 at 10 µm
    assert abs(ab_orbit - ab) <= 1e-6 * ab
    qs = math.acos(1.0 - ab / 2.0) / (2.0 * math.pi)
    if voltage == 5e6:
        assert qs == pytest.approx(4.62e-3, rel=2e-3)   # ≈ 216 turns per period


def test_radiation_equilibrium_spreads():
    """A bunch started in the linear equilibrium stays there: σ_z, σ_E and
    cov(z, ΔE) averaged over 4000 turns match the Lyapunov solution within
    three standard errors of one snapshot's estimate, 3/sqrt(2N)."""
    cfg = benchmark_ring(use_wakefield=False, use_excitation=True)
    p = cfg.params.replace(update_E0=False)
    n = 100_000
    S = anchors.equilibrium_covariance(p, cfg.sigma_E)
    x = np.random.default_rng(3).multivariate_normal([0.0, 0.0], S, size=n)
    z, e = np.ascontiguousarray(x[:, 0]), np.ascontiguousarray(x[:, 1])
    orc = Oracle(threads=8)
    st = orc.state(z, e, p.to_c(), None, 64, seed=11)
    # the excitation amplitude follows the bunch's own initial spread
    S = anchors.equilibrium_covariance(p, st.result().sigma_E0_initial)
    vz, ve, cv = [], [], []
    for t in range(4000):
        assert st.turn(None) == 0
        if t % 10 == 9:
            vz.append(np.var(st.z, ddof=1))
            ve.append(np.var(st.dE, ddof=1))
            cv.append(np.cov(st.z, st.dE)[0, 1])
    st.close()
    tol = 3.0 / math.sqrt(2.0 * n)
    assert abs(math.sqrt(np.mean(vz) / S[0, 0]) - 1.0) <= tol
    assert abs(math.sqrt(np.mean(ve) / S[1, 1]) - 1.0) <= tol
    rho = S[0, 1] / math.sqrt(S[0, 0] * S[1, 1])
    assert abs(np.mean(cv) / math.sqrt(S[0, 0] * S[1, 1]) - rho) <= 3.0 / math.sqrt(n)


@pytest.mark.parametrize("B", [4096, 1000, 5])
def test_single_bin_wake_potential(B):
    orc = Oracle(threads=1)
    for wake in (benchmark_ring().wake, WakeModel.reference(benchmark_ring().params)):
        grid = BinGrid.make(4e-3, B, wake.half_width_sigmas)
        for j0 in sorted({0, 1, B // 2 - 1, B // 2, B - 1}):
            counts = np.zeros(B, np.int64)
            counts[j0] = 12345
            cur = 2.9e-15
            want = anchors.single_bin_potential(grid.centers, j0, wake, cur)
            full = cur * np.abs(anchors.wake_function(grid.centers, wake)).max() / (
                math.sqrt(2 * math.pi) * wake.delta_std)
            for conv in (0, CONV_DIRECT_LD):
                got = orc.wake_potential(counts, grid.to_c(), wake.to_c(), cur, conv)
                assert np.abs(got - want).max() <= 1e-13 * full, (B, j0, conv)
