"""Single-step parity: each CUDA step through the C ABI against the oracle.

Mirrors the reference's kernel-equivalence tests (tests/loop_benchmark.jl,
rtol = 1e-12 against the serial loop) including its synthetic inputs
(z in [-5, 5), ΔE in [0, 0.1), tests/loop_benchmark.jl:84-122), plus the
benchmark ring's physical inputs and edge cases.  Histograms are bit-exact.
"""
import math

import numpy as np
import pytest

from haissinskijulia_b200 import (BinGrid, HaissinskiError, Particles, WakeModel, apply_wakefield_inplace,
                                  benchmark_ring, calculate_local_histogram, create_simulation_buffers,
                                  gaussian_draws, phase_advance, quantum_excitation, rf_kick,
                                  synchrotron_radiation, wake_potential)
from philox_ref import philox_normals_reference
from gpu_util import assert_close

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ring():
    return benchmark_ring(n_turns=1, nbins=4096)


def physical_bunch(n, seed=5):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 4e-3, n), rng.normal(0, 4e6, n)


def loop_pattern(n=100_000, seed=11):
    rng = np.random.default_rng(seed)
    return rng.random(n) * 10.0 - 5.0, rng.random(n) * 0.1


@pytest.mark.parametrize("case", ["physical", "loop_benchmark"])
@pytest.mark.parametrize("n", [1, 2, 31, 33, 100_000])
def test_rf_kick(gpu_ctx, oracle, case, n):
    if case == "physical":
        z, dE = physical_bunch(n)
        V, phis, k = 5e6, math.pi - math.asin(0.1), 10.479
    else:
        z, dE = loop_pattern(n)
        V, phis, k = 1000.0, 0.1, 0.5            # tests/loop_benchmark.jl:93-96
    buf = create_simulation_buffers(n, 64, ctx=gpu_ctx)
    p = Particles(z, dE.copy())
    rf_kick(V, math.sin(phis), k, phis, p, buf)
    want = dE.copy()
    oracle.rf_kick(V, math.sin(phis), k, phis, z.copy(), want)
    assert_close(p.coordinates.dE, want, np.abs(dE).max() + 1.0, what="rf_kick")


def test_quantum_excitation_host_draws(gpu_ctx, oracle, ring):
    n = 100_003
    z, dE = physical_bunch(n)
    r = np.random.default_rng(2).normal(size=n)
    buf = create_simulation_buffers(n, 64, ctx=gpu_ctx)
    p = Particles(z, dE.copy())
    quantum_excitation(4e9, ring.params.radius, 4e6, buf, p, draws=r)
    want = dE.copy()
    oracle.quantum_excitation(4e9, ring.params.radius, 4e6, r, want)
    assert_close(p.coordinates.dE, want, 4e6, what="quantum_excitation")


def test_synchrotron_radiation(gpu_ctx, oracle, ring):
    n = 4099
    z, dE = physical_bunch(n)
    buf = create_simulation_buffers(n, 64, ctx=gpu_ctx)
    p = Particles(z, dE.copy())
    synchrotron_radiation(4e9, ring.params.radius, p, buf)
    want = dE.copy()
    oracle.synchrotron_radiation(4e9, ring.params.radius, want)
    assert_close(p.coordinates.dE, want, 4e6, what="synchrotron_radiation")


@pytest.mark.parametrize("update_eta", [True, False])
def test_phase_advance(gpu_ctx, oracle, ring, update_eta):
    n = 100_000
    z, dE = physical_bunch(n)
    params = ring.params.replace(update_eta=update_eta)
    buf = create_simulation_buffers(n, 64, ctx=gpu_ctx)
    p = Particles(z.copy(), dE)
    phase_advance(p, params, 4e9 + 1234.5, buf)
    want = z.copy()
    oracle.drift(update_eta, 4e9 + 1234.5, params.mass, params.alpha_c, params.harmonic,
                 params.phi_s, params.freq_rf, dE.copy(), want)
    assert_close(p.coordinates.z, want, 4e-3, what="drift")


def _edge_cases(grid: BinGrid):
    e0, eN = grid.edge_first, grid.edge_last
    c = grid.centers
    return np.array([e0, eN, np.nextafter(e0, -1), np.nextafter(eN, 1), c[0], c[-1],
                     e0 + grid.edge_step, np.nextafter(e0 + grid.edge_step, -1), -1.0, 1.0,
                     0.0, -0.0, np.nan])


@pytest.mark.parametrize("B", [1, 2, 64, 1024, 4096, 16384])
def test_histogram_bit_exact(gpu_ctx, oracle, B):
    grid = BinGrid.make(4e-3, B, 6.0)
    z, _ = physical_bunch(200_000)
    z = np.concatenate([z, _edge_cases(grid)])
    buf = create_simulation_buffers(z.size, B, ctx=gpu_ctx)
    got = calculate_local_histogram(z, grid, buf)
    want = oracle.histogram(z, grid.to_c())
    assert np.array_equal(got, want)


def test_histogram_loop_benchmark_inputs(gpu_ctx, oracle):
    # tests/loop_benchmark.jl:84, :107-115: 1024 bins over [-5, 5]
    z, _ = loop_pattern()
    step = 10.0 / 1024
    centers = np.array([-5.0 + (i - 0.5) * step for i in range(1, 1025)])
    grid = BinGrid(-5.0, 5.0, step, centers)
    buf = create_simulation_buffers(z.size, 1024, ctx=gpu_ctx)
    assert np.array_equal(calculate_local_histogram(z, grid, buf), oracle.histogram(z, grid.to_c()))


def test_histogram_all_in_one_bin(gpu_ctx, oracle):
    grid = BinGrid.make(4e-3, 4096, 6.0)
    z = np.full(100_000, grid.centers[2000])
    buf = create_simulation_buffers(z.size, 4096, ctx=gpu_ctx)
    got = calculate_local_histogram(z, grid, buf)
    assert got[2000] == 100_000 and got.sum() == 100_000


@pytest.mark.parametrize("B", [2, 3, 4, 8, 64, 1000, 4096, 8192, 16384])
def test_wake_potential(gpu_ctx, oracle, ring, B):
    grid = BinGrid.make(4e-3, B, 6.0)
    z, _ = physical_bunch(500_000)
    counts = oracle.histogram(z, grid.to_c())
    buf = create_simulation_buffers(1, B, ctx=gpu_ctx)
    cur = 2.9e-15
    got = wake_potential(counts, grid, ring.wake, cur, buf)
    want = oracle.wake_potential(counts, grid.to_c(), ring.wake.to_c(), cur, 0)
    exact = oracle.wake_potential(counts, grid.to_c(), ring.wake.to_c(), cur, 1)
    scale = np.abs(exact).max()
    assert np.abs(got - exact).max() <= 1e-13 * scale
    assert np.abs(want - exact).max() <= 1e-13 * scale


def test_wake_potential_reference_wake_and_zero_counts(gpu_ctx, oracle):
    from haissinskijulia_b200 import reference_ring
    cfg = reference_ring(100_000)
    grid = BinGrid.make(cfg.sigma_z, cfg.nbins, 7.5)
    buf = create_simulation_buffers(1, cfg.nbins, ctx=gpu_ctx)
    z = np.random.default_rng(1).normal(0, cfg.sigma_z, 100_000)
    counts = oracle.histogram(z, grid.to_c())
    got = wake_potential(counts, grid, cfg.wake, 4e-13, buf)
    exact = oracle.wake_potential(counts, grid.to_c(), cfg.wake.to_c(), 4e-13, 1)
    assert np.abs(got - exact).max() <= 1e-13 * np.abs(exact).max()
    # no particles in range: zero potential (src/wakefield.jl:305-311)
    zero = wake_potential(np.zeros(cfg.nbins, np.int64), grid, cfg.wake, 4e-13, buf)
    assert not zero.any()


def test_apply_wakefield(gpu_ctx, oracle, ring):
    B = 4096
    grid = BinGrid.make(4e-3, B, 6.0)
    z, dE = physical_bunch(300_001)
    z[:13] = _edge_cases(grid)[:13]
    z[12] = 0.5  # far outside instead of NaN here
    buf = create_simulation_buffers(z.size, B, ctx=gpu_ctx)
    p = Particles(z.copy(), dE.copy())
    cur = 2.9e-15
    apply_wakefield_inplace(p, buf, ring.wake.wake_factor, ring.wake.wake_sqrt, ring.wake.ctau,
                            cur, 4e-3, grid, sin_coef=ring.wake.sin_coef)
    counts = oracle.histogram(z, grid.to_c())
    pot = oracle.wake_potential(counts, grid.to_c(), ring.wake.to_c(), cur, 0)
    want = dE.copy()
    oracle.interp_kick(z.copy(), want, grid.to_c(), pot)
    assert_close(p.coordinates.dE, want, 4e6, what="apply_wakefield")


def test_gaussian_matches_philox_restatement(gpu_ctx):
    buf = create_simulation_buffers(1, 1, ctx=gpu_ctx)
    n = 10_001
    got = gaussian_draws(12345, 7, n, buf)
    want = philox_normals_reference(12345, 7, n)
    # same counter -> normal mapping; CUDA's log/sincospi and numpy's log/sin/cos
    # of the same double uniforms agree to a few ulp of the normal
    assert np.max(np.abs(got - want)) < 1e-13
    assert np.median(np.abs(got - want)) < 1e-15
    big = gaussian_draws(99, 1, 2_000_000, buf)
    assert abs(big.mean()) < 5 * 1 / math.sqrt(big.size)
    assert abs(big.std() - 1.0) < 5 * math.sqrt(0.5 / big.size)
    # different turns and seeds give independent streams
    a = gaussian_draws(99, 2, 100_000, buf)
    b = gaussian_draws(100, 1, 100_000, buf)
    assert abs(np.corrcoef(big[:100_000], a)[0, 1]) < 0.02
    assert abs(np.corrcoef(big[:100_000], b)[0, 1]) < 0.02


def test_errors(gpu_ctx):
    buf = create_simulation_buffers(4, 8, ctx=gpu_ctx)
    grid = BinGrid.make(4e-3, 8, 6.0)
    with pytest.raises(HaissinskiError, match="HJ_ERR_WAKE_PARAM"):
        wake_potential(np.ones(8, np.int64), grid, WakeModel(1.0, 1.0, 0.0), 1.0, buf)
    with pytest.raises(HaissinskiError, match="HJ_ERR_TOO_LARGE"):
        big = BinGrid.make(4e-3, 32768, 6.0)
        wake_potential(np.ones(32768, np.int64), big, WakeModel(1.0, 1.0, 1e-3), 1.0,
                       create_simulation_buffers(4, 32768, ctx=gpu_ctx))
