"""Host logic of the parameter-sensitivity layer (src/parameter_sensitivity/):
apply_transform, compute_fom, the run list of a scan and the assembly of its
results.  No GPU."""
import math

import numpy as np
import pytest

from haissinskijulia_b200 import benchmark_ring
from haissinskijulia_b200.api import EvolveResult, Particles
from haissinskijulia_b200.sensitivity import (
    AlphaCompactionTransform, BunchLengthFoM, EmittanceFoM, EnergySpreadFoM,
    HarmonicNumberTransform, ParameterTransformation, PipeRadiusTransform, Run,
    VoltageTransform, apply_transform, assemble, build_runs, compute_fom, derivative_values,
    fallback_params, fallback_runs, host_correlation, scan_nbins)


def _params():
    return benchmark_ring(n_turns=20, nbins=1000).params


@pytest.mark.parametrize("t,field,value", [
    (VoltageTransform(), "voltage", 4.5e6),
    (AlphaCompactionTransform(), "alpha_c", 2.5e-4),
    (PipeRadiusTransform(), "pipe_radius", 3e-4),
])
def test_apply_transform_replaces_one_field(t, field, value):
    p = _params()
    q = apply_transform(t, value, p)
    assert getattr(q, field) == value
    for k, v in p.__dict__.items():
        if k != field:
            assert getattr(q, k) == v
    assert getattr(p, field) != value                      # a copy, not in place


def test_harmonic_transform_rounds_to_an_int_ties_to_even():
    p = _params()
    for v, h in ((360.4, 360), (360.6, 361), (2.5, 2), (3.5, 4), (-2.5, -2)):
        q = apply_transform(HarmonicNumberTransform(), v, p)
        assert q.harmonic == h and isinstance(q.harmonic, int)
    with pytest.raises(TypeError):
        apply_transform(ParameterTransformation(), 1.0, p)


def test_compute_fom_forms():
    rng = np.random.default_rng(3)
    z = rng.normal(0, 4e-3, 50_001)
    e = 0.3 * z * 1e9 + rng.normal(0, 4e6, z.size)
    parts = Particles(z, e)
    res = (np.std(e, ddof=1), np.std(z, ddof=1), 4e9)
    assert compute_fom(EnergySpreadFoM(), parts, res) == res[0]
    assert compute_fom(BunchLengthFoM(), parts, res) == res[1]
    r = np.corrcoef(z, e)[0, 1]
    em = compute_fom(EmittanceFoM(), parts, res)
    assert em == pytest.approx(res[1] * res[0] * math.sqrt(1 - r * r), rel=1e-12)
    er = EvolveResult(res[0], res[1], 4e9, 0, 0, 0, 0, 20)
    assert compute_fom(EmittanceFoM(), None, er, correlation=r) == pytest.approx(em, rel=1e-12)


def test_host_correlation_edges():
    rng = np.random.default_rng(4)
    x = rng.normal(size=10_001)
    y = -2.0 * x + 1e-3 * rng.normal(size=x.size)
    assert host_correlation(x, y) == pytest.approx(np.corrcoef(x, y)[0, 1], abs=1e-14)
    assert host_correlation(x, -3.0 * x) == -1.0                # clamped
    assert math.isnan(host_correlation(x, np.ones_like(x)))     # zero spread
    assert math.isnan(host_correlation(x[:1], y[:1]))
    with pytest.raises(ValueError):
        host_correlation(x[:0], y[:0])


def test_nbins_rule_is_exact():
    assert scan_nbins(20_000) == 2000
    with pytest.raises(ValueError):
        scan_nbins(20_001)


def test_run_list():
    p = _params()
    runs = build_runs(VoltageTransform(), [4e6, 5e6, 6e6], p, n_samples=3, seed=7,
                      gradients=True, rel_step=0.01)
    assert len(runs) == 3 * (1 + 2 * 3)
    base = [r for r in runs if r.role == "base"]
    assert [r.params.voltage for r in base] == [4e6, 5e6, 6e6]
    assert all(r.params.n_turns == 100 and r.seed == 7 for r in base)   # max(100, 20)
    for r in runs:
        if r.role != "base":
            q = r.params
            assert q.n_turns == 10 and q.use_wakefield and q.update_eta and not q.update_E0
            assert q.SR_damping and q.use_excitation
    plus = sorted((r.point, r.sample, r.seed, r.value) for r in runs if r.role == "+")
    minus = sorted((r.point, r.sample, r.seed, r.value) for r in runs if r.role == "-")
    for a, b in zip(plus, minus):
        assert a[:3] == b[:3] and a[3] > b[3]                 # common random numbers
    assert plus[0][3] == pytest.approx(4e6 * 1.01)
    assert build_runs(VoltageTransform(), [1.0], p.replace(n_turns=500), n_samples=2, seed=0,
                      gradients=False, rel_step=0.01)[0].params.n_turns == 500


def test_harmonic_derivative_sides_are_integers():
    assert derivative_values(HarmonicNumberTransform(), 360.0, 0.01) == (356.0, 364.0)
    assert derivative_values(HarmonicNumberTransform(), 10.0, 0.01) == (9.0, 11.0)
    assert derivative_values(VoltageTransform(), 0.0, 0.01) == (-0.01, 0.01)


def test_fallback_settings():
    p = _params()
    q = fallback_params(PipeRadiusTransform(), -1e-4, p)
    assert q.voltage == -1e-4 and q.pipe_radius == -1e-4      # voltage set to the value first
    assert q.n_turns == 50 and not q.use_wakefield and q.update_eta and not q.update_E0
    assert q.SR_damping and not q.use_excitation
    failed = [Run(0, "base", 0, 2.0, p, 1, error="x")]
    fr = fallback_runs(VoltageTransform(), failed, p, seed=1, gradients=True, rel_step=0.01)
    assert [r.role for r in fr] == ["fallback", "fallback+", "fallback-"]


def test_fallback_derivative_keeps_the_points_voltage():
    p = _params()
    fr = fallback_runs(PipeRadiusTransform(), [Run(0, "base", 0, 2e-4, p, 1, error="x")], p,
                       seed=1, gradients=True, rel_step=0.01)
    assert [r.params.voltage for r in fr] == [2e-4, 2e-4, 2e-4]
    assert [r.params.pipe_radius for r in fr] == pytest.approx([2e-4, 2.02e-4, 1.98e-4])
    fv = fallback_runs(VoltageTransform(), [Run(0, "base", 0, 5e6, p, 1, error="x")], p,
                       seed=1, gradients=True, rel_step=0.01)
    assert [r.params.voltage for r in fv] == pytest.approx([5e6, 5.05e6, 4.95e6])


def test_assemble():
    p = _params()
    runs = [Run(0, "base", 0, 1.0, p, 0, fom=10.0)]
    for k, (a, b) in enumerate(((3.0, 1.0), (4.0, 1.0), (2.5, 1.0))):
        runs += [Run(0, "+", k, 1.5, p, k, fom=a), Run(0, "-", k, 0.5, p, k, fom=b)]
    runs += [Run(1, "base", 0, 2.0, p, 0, error="boom"),
             Run(1, "fallback", 0, 2.0, p, 0, fom=5.0),
             Run(1, "fallback+", 0, 2.5, p, 0, fom=6.0),
             Run(1, "fallback-", 0, 1.5, p, 0, fom=4.0),
             Run(2, "base", 0, 3.0, p, 0, error="boom"),
             Run(2, "fallback", 0, 3.0, p, 0, error="boom too")]
    fom, grad, gerr, samples = assemble(runs, 3)
    s = np.array([2.0, 3.0, 1.5])
    assert fom[0] == 10.0 and grad[0] == pytest.approx(s.mean())
    assert gerr[0] == pytest.approx(s.std(ddof=1) / math.sqrt(3))
    assert (fom[1], grad[1], gerr[1]) == (5.0, 2.0, 0.0)
    assert all(math.isnan(v) for v in (fom[2], grad[2], gerr[2]))
    assert samples[2] == []
