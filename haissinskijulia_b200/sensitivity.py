"""The reference's parameter-sensitivity layer (src/parameter_sensitivity/)
over the batch engine: every run of a scan is a bunch of one Batch.

Kept from the reference:

* the transformation and figure-of-merit types (types.jl:15-71) and
  `ParameterSensitivity` (types.jl:78-84);
* `apply_transform` (transformations.jl:6-107): a copy of the parameters with
  one field replaced; the harmonic number is `Int(round(value))` (ties to
  even, as Python's `round`);
* `compute_fom` (figures_of_merit.jl:16-47): σ_E, σ_z, or the emittance
  σ_z σ_E √(1 − r²) with r = cor(z, ΔE), reduced on the GPU for batched runs
  (`hj_correlation`);
* `scan_parameter`'s per-point run (scan.jl:36-79): nbins = Int(n/10), the
  transformed parameters with n_turns raised to at least 100, a fresh copy of
  the initial particles, longitudinal_evolve!, compute_fom; and its retry with
  reduced complexity when a point fails (scan.jl:101-172: the voltage set to
  the point's value, 50 turns, no wakefield, no E0 update, no excitation), NaN
  when that fails too; the return tuple (param_range, fom_values,
  gradient_values, gradient_errors).

Replaced: the StochasticAD derivative (`derivative_estimate` of a 10-turn run
with update_E0 off, sensitivity.jl:54-69,168) cannot cross a Float64 C ABI.
Each of its `n_samples` samples here is a central difference of the same
10-turn run, (F(p+h) − F(p−h)) / (2h) with h = rel_step·|p|, both sides drawn
from the same Philox seed (common random numbers), so the sample scatter is
the excitation noise of the derivative, not of the two runs.  The mean and
std/√n_samples are reported as the reference reports its samples'
(sensitivity.jl:199-200).  The reference's heuristic fallback gradients
(sensitivity.jl:84-100,136-152,170-190) are not reproduced: a failed sample
is dropped, and a point whose samples all fail takes the reduced-complexity
retry, as a point whose compute_sensitivity raises does in the reference.

All runs of a scan (1 + 2·n_samples per point) are admitted into Batches
(one per combination of the wakefield and excitation switches) and advance
together; `scan_parameter_sequential` runs the same list one after another on
the plain resident path, with the same seeds and the same results.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from .api import (Batch, Context, EvolveResult, HaissinskiError, Particles, ResidentBunch,
                  SimulationParameters, correlation_device)


# ----------------------------------------------------------------------------- types (types.jl)


class ParameterTransformation:
    """ParameterTransformation (types.jl:15); `field` names the parameter."""

    field = ""

    def __eq__(self, other) -> bool:
        return type(self) is type(other)

    def __hash__(self) -> int:
        return hash(type(self))

    def __repr__(self) -> str:
        return f"{type(self).__name__}()"


class VoltageTransform(ParameterTransformation):
    """VoltageTransform (types.jl:22): RF voltage."""

    field = "voltage"


class AlphaCompactionTransform(ParameterTransformation):
    """AlphaCompactionTransform (types.jl:29): momentum compaction α_c."""

    field = "alpha_c"


class HarmonicNumberTransform(ParameterTransformation):
    """HarmonicNumberTransform (types.jl:36): harmonic number (an Int)."""

    field = "harmonic"


class PipeRadiusTransform(ParameterTransformation):
    """PipeRadiusTransform (types.jl:43): beam pipe radius."""

    field = "pipe_radius"


class FigureOfMerit:
    """FigureOfMerit (types.jl:50)."""

    def __eq__(self, other) -> bool:
        return type(self) is type(other)

    def __hash__(self) -> int:
        return hash(type(self))

    def __repr__(self) -> str:
        return f"{type(self).__name__}()"


class EnergySpreadFoM(FigureOfMerit):
    """EnergySpreadFoM (types.jl:57): final σ_E."""


class BunchLengthFoM(FigureOfMerit):
    """BunchLengthFoM (types.jl:64): final σ_z."""


class EmittanceFoM(FigureOfMerit):
    """EmittanceFoM (types.jl:71): σ_z σ_E √(1 − cor(z, ΔE)²)."""


@dataclass
class ParameterSensitivity:
    """ParameterSensitivity (types.jl:78-84)."""

    transform: ParameterTransformation
    fom: FigureOfMerit
    param_value: float
    mean_derivative: float
    uncertainty: float
    samples: List[float]


# ----------------------------------------------------------------------------- transforms, FoMs


def apply_transform(transform: ParameterTransformation, param_value,
                    sim_params: SimulationParameters) -> SimulationParameters:
    """apply_transform (transformations.jl:6-107): sim_params with the
    transformed field set to param_value, every other field kept."""
    if not isinstance(transform, ParameterTransformation) or not transform.field:
        raise TypeError(f"no apply_transform method for {transform!r}")
    if isinstance(transform, HarmonicNumberTransform):
        return sim_params.replace(harmonic=int(round(float(param_value))))   # :95
    return sim_params.replace(**{transform.field: float(param_value)})


def host_correlation(x: np.ndarray, y: np.ndarray) -> float:
    """cor(x, y) of two host arrays: two passes (means, then centred sums),
    r = Sxy/(√Sxx √Syy) clamped to [-1, 1]; the same arithmetic as
    hj_correlation, with numpy's summation order."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    if x.shape != y.shape:
        raise ValueError("x and y have different lengths")
    if x.size == 0:
        raise ValueError("correlation only defined for non-empty vectors")
    dx = x - x.sum() / x.size
    dy = y - y.sum() / y.size
    with np.errstate(invalid="ignore", divide="ignore"):
        r = float(np.float64(np.dot(dx, dy)) / (np.sqrt(np.dot(dx, dx)) * np.sqrt(np.dot(dy, dy))))
    return r if r != r else min(1.0, max(-1.0, r))


def _spreads(results):
    if isinstance(results, EvolveResult):
        return results.sigma_E, results.sigma_z, results.E0
    sigma_E, sigma_z, E0 = results
    return sigma_E, sigma_z, E0


def compute_fom(fom: FigureOfMerit, particles: Optional[Particles], results, *,
                correlation: Optional[float] = None) -> float:
    """compute_fom (figures_of_merit.jl:16-47).  results: the (σ_E, σ_z, E0)
    tuple of longitudinal_evolve or an EvolveResult.  For EmittanceFoM the
    correlation of the final (z, ΔE) is `correlation` when given (e.g. from
    correlation_device), else computed from `particles` on the host."""
    sigma_E, sigma_z, _ = _spreads(results)
    if isinstance(fom, EnergySpreadFoM):
        return float(sigma_E)                                       # :18
    if isinstance(fom, BunchLengthFoM):
        return float(sigma_z)                                       # :28
    if isinstance(fom, EmittanceFoM):
        r = correlation
        if r is None:
            r = host_correlation(particles.coordinates.z, particles.coordinates.dE)   # :42
        return float(sigma_z * sigma_E * math.sqrt(1.0 - r * r))    # :45
    raise TypeError(f"no compute_fom method for {fom!r}")


# ----------------------------------------------------------------------------- the run list


@dataclass
class Run:
    """One longitudinal_evolve of a scan: point `point`, role "base" or a
    derivative side "+"/"-" of sample `sample` (or "fallback", "fallback+",
    "fallback-"), at parameter value `value`."""

    point: int
    role: str
    sample: int
    value: float
    params: SimulationParameters
    seed: int
    fom: float = float("nan")
    result: Optional[EvolveResult] = None
    error: Optional[str] = None
    admitted: float = 0.0
    finished: float = 0.0


def scan_nbins(n_particles: int) -> int:
    """nbins = Int(n_particles/10) (scan.jl:40): exact or an error."""
    if n_particles % 10:
        raise ValueError(f"InexactError: Int64({n_particles / 10})")
    return n_particles // 10


def derivative_values(transform: ParameterTransformation, p: float, rel_step: float):
    """The two sides (p − h, p + h) of the central difference at p."""
    h = rel_step * abs(p) if p != 0 else rel_step
    if isinstance(transform, HarmonicNumberTransform):
        lo, hi = int(round(p - h)), int(round(p + h))
        if lo == hi:
            lo, hi = int(round(p)) - 1, int(round(p)) + 1
        return float(lo), float(hi)
    return p - h, p + h


def base_params(transform, value, sim_params: SimulationParameters) -> SimulationParameters:
    """The point's parameters, n_turns raised to at least 100 (scan.jl:43-68)."""
    p = apply_transform(transform, value, sim_params)
    return p.replace(n_turns=max(100, p.n_turns))


def derivative_params(transform, value, base: SimulationParameters) -> SimulationParameters:
    """sensitivity_fn's run at p (sensitivity.jl:41-69): min(10, n_turns) turns,
    wakefield, η update, damping and excitation on, no E0 update."""
    p = apply_transform(transform, value, base)
    return p.replace(n_turns=min(10, p.n_turns), use_wakefield=True, update_eta=True,
                     update_E0=False, SR_damping=True, use_excitation=True)


def fallback_params(transform, value, sim_params: SimulationParameters,
                    point_value: Optional[float] = None) -> SimulationParameters:
    """The reduced-complexity retry (scan.jl:107-123, 128-130, 162-163): the
    voltage set to the point's value, 50 turns, no wakefield, no E0 update, no
    excitation; then the transform applied at `value` (the point's value, or a
    side of its derivative)."""
    pv = float(value if point_value is None else point_value)
    simpler = sim_params.replace(voltage=pv, n_turns=50, use_wakefield=False, update_eta=True,
                                 update_E0=False, SR_damping=True, use_excitation=False)
    return apply_transform(transform, value, simpler)


def build_runs(transform, param_range: Sequence[float], sim_params: SimulationParameters, *,
               n_samples: int, seed: int, gradients: bool, rel_step: float) -> List[Run]:
    runs: List[Run] = []
    for i, v in enumerate(param_range):
        v = float(v)
        base = base_params(transform, v, sim_params)
        runs.append(Run(i, "base", 0, v, base, seed))
        if gradients:
            lo, hi = derivative_values(transform, v, rel_step)
            pm = derivative_params(transform, lo, base)
            pp = derivative_params(transform, hi, base)
            for k in range(n_samples):
                runs.append(Run(i, "+", k, hi, pp, seed + 1 + k))
                runs.append(Run(i, "-", k, lo, pm, seed + 1 + k))
    return runs


def fallback_runs(transform, failed: Sequence[Run], sim_params: SimulationParameters, *,
                  seed: int, gradients: bool, rel_step: float) -> List[Run]:
    runs: List[Run] = []
    for r in failed:
        runs.append(Run(r.point, "fallback", 0, r.value,
                        fallback_params(transform, r.value, sim_params), seed))
        if gradients:
            lo, hi = derivative_values(transform, r.value, rel_step)
            runs.append(Run(r.point, "fallback+", 0, hi,
                            fallback_params(transform, hi, sim_params, r.value), seed))
            runs.append(Run(r.point, "fallback-", 0, lo,
                            fallback_params(transform, lo, sim_params, r.value), seed))
    return runs


def _gradient(runs: List[Run], point: int, plus: str, minus: str):
    by_k: Dict[int, Dict[str, Run]] = {}
    for r in runs:
        if r.point == point and r.role in (plus, minus):
            by_k.setdefault(r.sample, {})[r.role] = r
    samples = []
    for k in sorted(by_k):
        d = by_k[k]
        if plus in d and minus in d and d[plus].error is None and d[minus].error is None:
            samples.append((d[plus].fom - d[minus].fom) / (d[plus].value - d[minus].value))
    if not samples:
        return float("nan"), float("nan"), samples
    s = np.asarray(samples)
    err = float(s.std(ddof=1) / math.sqrt(s.size)) if s.size > 1 else float("nan")
    return float(s.mean()), err, samples


def assemble(runs: List[Run], n_points: int):
    """(fom_values, gradient_values, gradient_errors, samples per point) of a
    finished run list."""
    fom = np.full(n_points, np.nan)
    grad = np.full(n_points, np.nan)
    gerr = np.full(n_points, np.nan)
    samples: List[list] = [[] for _ in range(n_points)]
    for i in range(n_points):
        base = [r for r in runs if r.point == i and r.role == "base"][0]
        if base.error is None:
            fom[i] = base.fom
            grad[i], gerr[i], samples[i] = _gradient(runs, i, "+", "-")
            continue
        fb = [r for r in runs if r.point == i and r.role == "fallback"]
        if fb and fb[0].error is None:
            fom[i] = fb[0].fom
            g, _, s = _gradient(runs, i, "fallback+", "fallback-")
            # no excitation in the retry: the derivative is deterministic
            grad[i], gerr[i], samples[i] = g, (0.0 if s else float("nan")), s
    return fom, grad, gerr, samples


# ----------------------------------------------------------------------------- execution


class _Initial:
    """The initial particles, once on the device."""

    def __init__(self, particles: Particles):
        import torch
        self.n = len(particles)
        self.z = torch.from_numpy(np.ascontiguousarray(particles.coordinates.z)).cuda()
        self.dE = torch.from_numpy(np.ascontiguousarray(particles.coordinates.dE)).cuda()


def _finish_fom(ctx, fom, r: Run, res: EvolveResult, final) -> None:
    r.result = res
    corr = None
    if isinstance(fom, EmittanceFoM):
        corr = correlation_device(ctx, final[0].data_ptr(), final[1].data_ptr(),
                                  final[0].numel())
    r.fom = compute_fom(fom, None, res, correlation=corr)


def run_batched(ctx: Context, runs: List[Run], fom: FigureOfMerit, init: _Initial, nbins: int,
                *, chunk: int = 65536, layout: int = -1, graph_turns: int = 16,
                block_turns: int = 16, max_resident: Optional[int] = None,
                admit_group: int = 256) -> None:
    """Every run through Batches (one per wakefield/excitation combination):
    admit while there is room (groups of runs with one synchronisation each),
    advance in blocks, take the finished runs together (the emittance's
    correlation reduced on the device as they are taken)."""
    n = init.n
    emittance = isinstance(fom, EmittanceFoM)
    groups: Dict[tuple, List[Run]] = {}
    for r in runs:
        groups.setdefault((bool(r.params.use_wakefield), bool(r.params.use_excitation)),
                          []).append(r)
    zp, ep = init.z.data_ptr(), init.dE.data_ptr()
    t0 = time.perf_counter()
    for todo in groups.values():
        slots = min(len(todo), max_resident or len(todo))
        bt = Batch(ctx, slots * (n + 4), slots, max(nbins, 1), chunk=chunk, layout=layout,
                   graph_turns=graph_turns)
        try:
            pending = list(todo)
            live: Dict[int, Run] = {}
            while pending or live:
                while pending:
                    grp = pending[:admit_group]
                    k = len(grp)
                    ids, err = bt.add_many([zp] * k, [ep] * k, [n] * k, [r.params for r in grp],
                                           [nbins] * k, [r.seed for r in grp],
                                           [r.params.n_turns for r in grp])
                    now = time.perf_counter() - t0
                    for r, bid in zip(grp, ids):
                        r.admitted = now
                        live[bid] = r
                    del pending[:len(ids)]
                    if err is None:
                        continue
                    if err.status == _lib.HJ_ERR_FULL:
                        if live:
                            break
                        raise err
                    pending[0].error = str(err)          # this run cannot be made
                    pending.pop(0)
                if not live:
                    continue
                bt.advance(block_turns)
                done = bt.poll()
                if done:
                    results, corr = bt.take_many(done, correlation=emittance)
                    now = time.perf_counter() - t0
                    for i, bid in enumerate(done):
                        r = live.pop(bid)
                        r.result = results[i]
                        r.fom = compute_fom(fom, None, results[i],
                                            correlation=corr[i] if emittance else None)
                        r.finished = now
        finally:
            bt.close()


def run_sequential(ctx: Context, runs: List[Run], fom: FigureOfMerit, init: _Initial,
                   nbins: int) -> None:
    """The same runs one after another on the plain resident path."""
    n = init.n
    t0 = time.perf_counter()
    for r in runs:
        dz, de = init.z.clone(), init.dE.clone()
        try:
            b = ResidentBunch(ctx, dz.data_ptr(), de.data_ptr(), n, r.params, nbins, seed=r.seed)
        except HaissinskiError as e:
            r.error = str(e)
            continue
        try:
            b.advance(r.params.n_turns)
            res = b.finish()
        finally:
            b.close()
        _finish_fom(ctx, fom, r, res, (dz, de))
        r.finished = time.perf_counter() - t0


def _scan(runner, transform, fom, param_range, initial_particles, sim_params, *, n_samples,
          ctx, seed, nbins, gradients, rel_step, **kw):
    ctx = ctx or Context(0)
    if not isinstance(fom, FigureOfMerit) or type(fom) is FigureOfMerit:
        raise TypeError(f"no compute_fom method for {fom!r}")
    param_range = list(param_range)
    n = len(initial_particles)
    if n == 0:
        raise ValueError("a scan needs at least one particle")
    nb = scan_nbins(n) if nbins is None else int(nbins)
    init = _Initial(initial_particles)
    runs = build_runs(transform, param_range, sim_params, n_samples=n_samples, seed=seed,
                      gradients=gradients, rel_step=rel_step)
    runner(ctx, runs, fom, init, nb, **kw)
    # a point fails when its run fails, or when every derivative sample does
    # (compute_sensitivity raises, scan.jl:77-84 -> :98)
    failed = [r for r in runs if r.role == "base" and (
        r.error is not None or (gradients and not _gradient(runs, r.point, "+", "-")[2]))]
    for r in failed:
        r.error = r.error or "All sensitivity samples failed and no fallback available"
    if failed:
        extra = fallback_runs(transform, failed, sim_params, seed=seed, gradients=gradients,
                              rel_step=rel_step)
        runner(ctx, extra, fom, init, nb, **kw)
        runs += extra
    fom_values, grad, gerr, _ = assemble(runs, len(param_range))
    return param_range, fom_values, grad, gerr, runs


def scan_parameter(transform: ParameterTransformation, fom: FigureOfMerit,
                   param_range: Sequence[float], initial_particles: Particles,
                   sim_params: SimulationParameters, *, n_samples: int = 20,
                   ctx: Optional[Context] = None, seed: int = 0, nbins: Optional[int] = None,
                   gradients: bool = True, rel_step: float = 0.01, return_runs: bool = False,
                   **batch_kw):
    """scan_parameter (scan.jl:14-192) with every run of every point in one
    batch: returns (param_range, fom_values, gradient_values, gradient_errors)
    (and the run records with return_runs).  nbins defaults to the
    reference's Int(n/10); batch_kw: chunk, layout, graph_turns, block_turns,
    max_resident."""
    out = _scan(run_batched, transform, fom, param_range, initial_particles, sim_params,
                n_samples=n_samples, ctx=ctx, seed=seed, nbins=nbins, gradients=gradients,
                rel_step=rel_step, **batch_kw)
    return out if return_runs else out[:4]


def scan_parameter_sequential(transform: ParameterTransformation, fom: FigureOfMerit,
                              param_range: Sequence[float], initial_particles: Particles,
                              sim_params: SimulationParameters, *, n_samples: int = 20,
                              ctx: Optional[Context] = None, seed: int = 0,
                              nbins: Optional[int] = None, gradients: bool = True,
                              rel_step: float = 0.01, return_runs: bool = False):
    """scan_parameter with the runs one after another on the plain resident
    path (the reference's order, scan.jl:182-184); same seeds, same results."""
    out = _scan(run_sequential, transform, fom, param_range, initial_particles, sim_params,
                n_samples=n_samples, ctx=ctx, seed=seed, nbins=nbins, gradients=gradients,
                rel_step=rel_step)
    return out if return_runs else out[:4]


def compute_sensitivity(transform: ParameterTransformation, fom: FigureOfMerit,
                        param_value: float, initial_particles: Particles,
                        sim_params: SimulationParameters, *, n_samples: int = 100,
                        ctx: Optional[Context] = None, seed: int = 0,
                        nbins: Optional[int] = None, rel_step: float = 0.01,
                        **batch_kw) -> ParameterSensitivity:
    """compute_sensitivity (sensitivity.jl:22-212) at one value: the
    derivative samples of the min(10, n_turns)-turn run (central differences
    with common random numbers, all in one batch), their mean and
    std/√n_samples."""
    ctx = ctx or Context(0)
    n = len(initial_particles)
    nb = scan_nbins(n) if nbins is None else int(nbins)
    init = _Initial(initial_particles)
    lo, hi = derivative_values(transform, float(param_value), rel_step)
    pp = derivative_params(transform, hi, sim_params)
    pm = derivative_params(transform, lo, sim_params)
    runs = []
    for k in range(n_samples):
        runs.append(Run(0, "+", k, hi, pp, seed + 1 + k))
        runs.append(Run(0, "-", k, lo, pm, seed + 1 + k))
    run_batched(ctx, runs, fom, init, nb, **batch_kw)
    mean, err, samples = _gradient(runs, 0, "+", "-")
    if not samples:
        raise HaissinskiError(_lib.HJ_ERR_ARG, "All sensitivity samples failed and no fallback "
                              "available")
    return ParameterSensitivity(transform, fom, float(param_value), mean, err, samples)
