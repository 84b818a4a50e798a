"""generate_particles on the device (src/evolution.jl:42-133): covariance
estimate from a 10k sample, correlated draws, two-pass actual spreads."""
import numpy as np
import pytest

from haissinskijulia_b200 import generate_particles

pytestmark = pytest.mark.gpu


def test_generated_bunch_statistics_and_spreads(gpu_ctx):
    n = 2_000_000
    mu_z, mu_E, sz, sE = 1e-3, 5e5, 4e-3, 4e6
    p, aE, az, E0 = generate_particles(mu_z, mu_E, sz, sE, n, 4e9, ctx=gpu_ctx, seed=11)
    z, e = p.coordinates.z, p.coordinates.dE
    assert E0 == 4e9 and z.size == n
    # actual spreads: compute_std, two-pass sample std (src/utils.jl:531-544)
    assert az == pytest.approx(np.std(z, ddof=1), rel=1e-12)
    assert aE == pytest.approx(np.std(e, ddof=1), rel=1e-12)
    # the distribution: means, spreads (within the 10k-sample estimate's
    # statistical error) and a correlation as small as that estimate's
    assert abs(z.mean() - mu_z) < 5 * sz / np.sqrt(n)
    assert abs(e.mean() - mu_E) < 5 * sE / np.sqrt(n)
    assert abs(az / sz - 1) < 0.05 and abs(aE / sE - 1) < 0.05
    assert abs(np.corrcoef(z, e)[0, 1]) < 0.05
    # seeded: the same draws again, other draws under another seed
    p2, aE2, az2, _ = generate_particles(mu_z, mu_E, sz, sE, n, 4e9, ctx=gpu_ctx, seed=11)
    assert np.array_equal(p2.coordinates.z, z) and (aE2, az2) == (aE, az)
    p3, _, _, _ = generate_particles(mu_z, mu_E, sz, sE, n, 4e9, ctx=gpu_ctx, seed=12)
    assert not np.array_equal(p3.coordinates.z, z)


def test_small_bunches_follow_the_reference(gpu_ctx):
    p, aE, az, _ = generate_particles(0.0, 0.0, 4e-3, 4e6, 1, 4e9, ctx=gpu_ctx, seed=1)
    assert len(p) == 1 and (aE, az) == (4e6, 4e-3)          # input spreads for one particle
    p, aE, az, _ = generate_particles(0.0, 0.0, 4e-3, 4e6, 0, 4e9, ctx=gpu_ctx, seed=1)
    assert len(p) == 0 and (aE, az) == (0.0, 0.0)
