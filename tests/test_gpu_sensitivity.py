"""Parameter scans (src/parameter_sensitivity/) on the batch engine: the
device correlation, each point's figure of merit against the oracle, the
batched scan against the same runs one after another, and the
reduced-complexity retry of a failing point."""
import math

import numpy as np
import pytest
import torch

from haissinskijulia_b200 import (HaissinskiError, Particles, WakeModel, benchmark_ring,
                                  create_simulation_buffers, gaussian_draws, longitudinal_evolve)
from haissinskijulia_b200.api import correlation_device
from haissinskijulia_b200.sensitivity import (
    EmittanceFoM, EnergySpreadFoM, PipeRadiusTransform, VoltageTransform, base_params,
    compute_sensitivity, fallback_params, host_correlation, scan_parameter,
    scan_parameter_sequential)

pytestmark = pytest.mark.gpu

N = 20_000          # nbins = Int(N/10) = 2000


def _initial(seed=5, n=N):
    cfg = benchmark_ring(n_turns=20, nbins=n // 10)
    rng = np.random.default_rng(seed)
    return cfg, Particles(rng.normal(0.0, cfg.sigma_z, n), rng.normal(0.0, cfg.sigma_E, n))


def test_device_correlation_matches_the_host(gpu_ctx):
    rng = np.random.default_rng(1)
    n = 1_000_003
    x = rng.normal(1e-3, 4e-3, n)
    y = 0.37 * x * 1e9 + rng.normal(5e5, 4e6, n)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    r = correlation_device(gpu_ctx, dx.data_ptr(), dy.data_ptr(), n)
    assert abs(r - host_correlation(x, y)) <= 1e-13
    assert abs(r - np.corrcoef(x, y)[0, 1]) <= 1e-13
    neg = -dx
    assert abs(correlation_device(gpu_ctx, dx.data_ptr(), neg.data_ptr(), n) + 1.0) <= 1e-15
    assert math.isnan(correlation_device(gpu_ctx, dx.data_ptr(), dy.data_ptr(), 1))
    with pytest.raises(HaissinskiError):
        correlation_device(gpu_ctx, dx.data_ptr(), dy.data_ptr(), 0)


def test_scan_points_match_the_oracle(gpu_ctx, gpu_buffers, oracle):
    cfg, parts = _initial()
    values = [4e6, 6e6]
    _, fom, grad, gerr = scan_parameter(VoltageTransform(), EmittanceFoM(), values, parts,
                                        cfg.params, ctx=gpu_ctx, seed=3, gradients=False)
    assert np.all(np.isnan(grad)) and np.all(np.isnan(gerr))
    for v, f in zip(values, fom):
        p = base_params(VoltageTransform(), v, cfg.params)
        assert p.n_turns == 100
        z, e = parts.coordinates.z.copy(), parts.coordinates.dE.copy()
        st = oracle.state(z, e, p.to_c(), WakeModel.reference(p).to_c(), N // 10)
        for t in range(p.n_turns):
            assert st.turn(gaussian_draws(3, t + 1, N, gpu_buffers)) == 0
        r = st.result()
        want = r.sigma_z * r.sigma_E * math.sqrt(1.0 - host_correlation(z, e) ** 2)
        assert f == pytest.approx(want, rel=1e-11)


def test_batched_scan_equals_the_sequential_runs(gpu_ctx):
    cfg, parts = _initial(seed=9)
    values = [4.5e6, 5e6, 5.5e6]
    kw = dict(ctx=gpu_ctx, seed=11, n_samples=3, return_runs=True)
    _, fb, gb, eb, runs_b = scan_parameter(VoltageTransform(), EnergySpreadFoM(), values, parts,
                                           cfg.params, **kw)
    _, fs, gs, es, runs_s = scan_parameter_sequential(VoltageTransform(), EnergySpreadFoM(),
                                                      values, parts, cfg.params, **kw)
    assert len(runs_b) == len(runs_s) == 3 * 7
    for a, b in zip(runs_b, runs_s):
        assert (a.point, a.role, a.sample, a.seed) == (b.point, b.role, b.sample, b.seed)
        assert a.error is None and b.error is None
        assert a.fom == pytest.approx(b.fom, rel=1e-12)
    np.testing.assert_allclose(fb, fs, rtol=1e-12)
    # a central difference amplifies the 1e-12 agreement of its two runs
    scale = 4e-12 * max(fb) / (0.02 * min(values))
    assert np.all(np.abs(gb - gs) <= scale)
    assert np.all(np.abs(eb - es) <= scale)
    assert np.all(np.isfinite(gb)) and np.all(eb > 0)
    # each derivative sample uses one seed on both sides
    sens = compute_sensitivity(VoltageTransform(), EnergySpreadFoM(), 5e6, parts,
                               base_params(VoltageTransform(), 5e6, cfg.params), n_samples=3,
                               ctx=gpu_ctx, seed=11)
    assert sens.mean_derivative == pytest.approx(gb[1], rel=1e-9, abs=scale)
    assert len(sens.samples) == 3


def test_a_failing_point_is_retried_with_reduced_complexity(gpu_ctx):
    cfg, parts = _initial(seed=13)
    values = [2.5e-4, -1e-4]                     # pipe_radius <= 0: the wake rejects it
    _, fom, grad, gerr, runs = scan_parameter(PipeRadiusTransform(), EnergySpreadFoM(), values,
                                              parts, cfg.params, ctx=gpu_ctx, seed=2,
                                              n_samples=2, return_runs=True)
    base = [r for r in runs if r.role == "base"]
    assert base[0].error is None and base[1].error is not None
    assert math.isfinite(fom[0]) and math.isfinite(fom[1])
    p = fallback_params(PipeRadiusTransform(), -1e-4, cfg.params)
    q = parts.copy()
    want = longitudinal_evolve(q, p, create_simulation_buffers(N, N // 10, ctx=gpu_ctx))
    assert fom[1] == pytest.approx(want[0], rel=1e-12)
    # without the wakefield the pipe radius does not enter: zero derivative, deterministic
    assert grad[1] == 0.0 and gerr[1] == 0.0
