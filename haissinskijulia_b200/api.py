"""Python host interface mirroring the reference's Julia API for the tracking path.

Names, argument order and meaning follow module StochasticHaissinski
(src/StochasticHaissinski.jl:46-56); every compute call goes through the C
ABI of libhaissinski_gpu.so (no CPU fallback).  Julia's mutating `!`
functions become functions that mutate the numpy arrays in place:

    reference (Julia)                          here (Python)
    SimulationParameters(...)                  SimulationParameters(...)
    create_simulation_buffers(n, nbins, mpi)   create_simulation_buffers(n, nbins, mpi)
    longitudinal_evolve!(p, params, buf, ...)  longitudinal_evolve(p, params, buf, ...)
    rf_kick!(V, sinϕs, k, ϕs, p, buf)          rf_kick(V, sinϕs, k, ϕs, p, buf)
    quantum_excitation!(E0, R, σE0, buf, p)    quantum_excitation(E0, R, σE0, buf, p)
    synchrotron_radiation!(E0, R, p, buf)      synchrotron_radiation(E0, R, p, buf)
    apply_wakefield_inplace!(p, buf, ...)      apply_wakefield_inplace(p, buf, ...)

Errors the reference raises with `error(...)` raise HaissinskiError here,
carrying the library's message.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from ._lib import HjCheckpoint, HjGrid, HjParams, HjResult, HjWake

# src/constants.jl:5-8
SPEED_LIGHT = 299792458.0
ELECTRON_CHARGE = 1.602176634e-19
MASS_ELECTRON = 0.51099895069e6
INV_SQRT_2π = 1 / math.sqrt(2 * math.pi)


class HaissinskiError(RuntimeError):
    """A library call failed; `.status` holds the HJ_ERR_* code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_lib.status_string(status)}: {message}")
        self.status = status


# ----------------------------------------------------------------------------- data model


@dataclass
class SimulationParameters:
    """Field for field src/data_structures.jl:81-97 (Float64 instantiation)."""

    E0: float
    mass: float
    voltage: float
    harmonic: int
    radius: float
    pipe_radius: float
    alpha_c: float
    phi_s: float
    freq_rf: float
    n_turns: int
    use_wakefield: bool
    update_eta: bool
    update_E0: bool
    SR_damping: bool
    use_excitation: bool

    # Unicode spellings of the reference's field names.
    @property
    def α_c(self) -> float:
        return self.alpha_c

    @property
    def ϕs(self) -> float:
        return self.phi_s

    @property
    def update_η(self) -> bool:
        return self.update_eta

    def to_c(self) -> HjParams:
        p = HjParams()
        p.E0 = float(self.E0)
        p.mass = float(self.mass)
        p.voltage = float(self.voltage)
        p.harmonic = int(self.harmonic)
        p.radius = float(self.radius)
        p.pipe_radius = float(self.pipe_radius)
        p.alpha_c = float(self.alpha_c)
        p.phi_s = float(self.phi_s)
        p.freq_rf = float(self.freq_rf)
        p.n_turns = int(self.n_turns)
        p.use_wakefield = int(bool(self.use_wakefield))
        p.update_eta = int(bool(self.update_eta))
        p.update_E0 = int(bool(self.update_E0))
        p.SR_damping = int(bool(self.SR_damping))
        p.use_excitation = int(bool(self.use_excitation))
        return p

    def replace(self, **kw) -> "SimulationParameters":
        d = dict(self.__dict__)
        d.update(kw)
        return SimulationParameters(**d)


class Coordinates:
    """SoA view `particles.coordinates.z` / `.ΔE` (src/data_structures.jl:26-29)."""

    def __init__(self, z: np.ndarray, dE: np.ndarray):
        self.z = z
        self.dE = dE

    @property
    def ΔE(self) -> np.ndarray:
        return self.dE

    @ΔE.setter
    def ΔE(self, v: np.ndarray) -> None:
        self.dE = v


class Particles:
    """StructArray{Particle{Float64}} as two contiguous float64 arrays."""

    def __init__(self, z, dE):
        z = np.ascontiguousarray(z, dtype=np.float64)
        dE = np.ascontiguousarray(dE, dtype=np.float64)
        if z.shape != dE.shape or z.ndim != 1:
            raise ValueError("z and ΔE must be 1-D arrays of equal length")
        self.coordinates = Coordinates(z, dE)

    def __len__(self) -> int:
        return self.coordinates.z.shape[0]

    def copy(self) -> "Particles":
        return Particles(self.coordinates.z.copy(), self.coordinates.dE.copy())


@dataclass
class WakeModel:
    """Wake form and intensity; WakeModel.reference(params) is the reference's
    hard-coded model (src/evolution.jl:276-280)."""

    wake_factor: float
    wake_sqrt: float
    ctau: float
    sin_coef: float = 0.0
    population: float = 0.0
    half_width_sigmas: float = 7.5
    delta_std: float = 0.15

    @staticmethod
    def reference(params: SimulationParameters) -> "WakeModel":
        w = HjWake()
        p = params.to_c()
        _check(None, _lib.load().hj_wake_reference(ctypes.byref(p), ctypes.byref(w)))
        return WakeModel.from_c(w)

    @staticmethod
    def resonator(Rs: float, Q: float, fr: float, population: float,
                  half_width_sigmas: float = 6.0) -> "WakeModel":
        w = HjWake()
        _check(None, _lib.load().hj_wake_resonator(Rs, Q, fr, population, half_width_sigmas,
                                                   ctypes.byref(w)))
        return WakeModel.from_c(w)

    @staticmethod
    def from_c(w: HjWake) -> "WakeModel":
        return WakeModel(w.wake_factor, w.wake_sqrt, w.ctau, w.sin_coef, w.population,
                         w.half_width_sigmas, w.delta_std)

    def to_c(self) -> HjWake:
        w = HjWake()
        w.wake_factor, w.wake_sqrt, w.ctau = self.wake_factor, self.wake_sqrt, self.ctau
        w.sin_coef, w.population = self.sin_coef, self.population
        w.half_width_sigmas, w.delta_std = self.half_width_sigmas, self.delta_std
        return w


@dataclass
class BinGrid:
    """Uniform bins: edge_first/edge_last/edge_step and the B centers
    (src/evolution.jl:270-274)."""

    edge_first: float
    edge_last: float
    edge_step: float
    centers: np.ndarray

    @property
    def nbins(self) -> int:
        return int(self.centers.shape[0])

    @staticmethod
    def make(sigma_z0: float, nbins: int, half_width_sigmas: float = 7.5) -> "BinGrid":
        c = np.empty(max(int(nbins), 1), dtype=np.float64)
        g = HjGrid()
        _check(None, _lib.load().hj_make_grid(float(sigma_z0), float(half_width_sigmas),
                                              int(nbins), _dp(c), ctypes.byref(g)))
        return BinGrid(g.edge_first, g.edge_last, g.edge_step, c)

    def to_c(self) -> HjGrid:
        self.centers = np.ascontiguousarray(self.centers, dtype=np.float64)
        g = HjGrid()
        g.nbins = self.nbins
        g.edge_first, g.edge_last, g.edge_step = self.edge_first, self.edge_last, self.edge_step
        g.centers = _dp(self.centers)
        return g


class Context:
    """A library context bound to one CUDA device (hj_create)."""

    def __init__(self, device: int = 0):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        rc = self._lib.hj_create(int(device), ctypes.byref(h))
        if rc != _lib.HJ_OK:
            raise HaissinskiError(rc, f"cannot create a context on CUDA device {device}")
        self.handle = h
        self.device = device

    def last_error(self) -> str:
        return self._lib.hj_last_error(self.handle).decode()

    def set_pass_layout(self, layout: int) -> None:
        """Thread layout of the fused pass for bunches created afterwards
        (-1 = automatic; 0-5 = fixed layouts with 16-bit bin counters, 8-13
        the same with 32-bit counters; + 16 for single-precision excitation
        normals, 23 = automatic with them; see hj_set_pass_layout)."""
        _check(self, self._lib.hj_set_pass_layout(self.handle, int(layout)))

    def trim(self) -> None:
        """Free the device and pinned blocks this context keeps for reuse
        (hj_trim)."""
        _check(self, self._lib.hj_trim(self.handle))

    def close(self) -> None:
        """Release the context (hj_destroy).  Bunches and batches created on it
        keep working; the library frees the context when the last of them is
        closed, whatever the order."""
        if getattr(self, "handle", None):
            self._lib.hj_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


@dataclass
class SimulationBuffers:
    """What create_simulation_buffers (src/utils.jl:147-254) sizes: the bin
    count and particle count.  Device memory is owned by the library."""

    n_particles: int
    nbins: int
    use_mpi: bool = False
    comm_size: int = 1
    ctx: Optional[Context] = field(default=None, repr=False)

    def context(self) -> Context:
        if self.ctx is None:
            self.ctx = default_context()
        return self.ctx


def create_simulation_buffers(n_particles: int, nbins: int, use_mpi: bool = False,
                              comm_size: int = 1, ctx: Optional[Context] = None
                              ) -> SimulationBuffers:
    """src/utils.jl:147-160 argument checks included."""
    if nbins <= 0:
        raise ValueError(f"Number of bins (nbins) must be positive. Got {nbins}.")
    if n_particles < 0:
        raise ValueError(f"Number of particles must be non-negative. Got {n_particles}.")
    return SimulationBuffers(int(n_particles), int(nbins), bool(use_mpi), int(comm_size), ctx)


# ----------------------------------------------------------------------------- helpers


def _dp(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


def _check(ctx: Optional[Context], rc: int) -> None:
    if rc != _lib.HJ_OK:
        msg = ctx.last_error() if ctx is not None else ""
        raise HaissinskiError(rc, msg)


def _f64(a) -> np.ndarray:
    a = np.asarray(a)
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("particle arrays must be C-contiguous float64 (they are updated in place)")
    return a


def next_power_of_two(n: int) -> int:
    """src/utils.jl:119-122."""
    if n <= 0:
        return 1
    p = 1
    while p < n:
        p <<= 1
    return p


def calc_rf_factor(freq_rf: float, β: float) -> float:
    """src/utils.jl:484-491."""
    if β <= 0:
        return math.inf
    return freq_rf * (2 * math.pi) / (β * SPEED_LIGHT)


def z_to_ϕ(z_val, rf_factor, ϕs):
    """src/utils.jl:462-464."""
    return -(z_val * rf_factor - ϕs)


def ϕ_to_z(ϕ_val, rf_factor, ϕs):
    """src/utils.jl:471-477."""
    if rf_factor == 0:
        raise HaissinskiError(_lib.HJ_ERR_ARG, "RF factor is zero, cannot convert phase to position.")
    return (-ϕ_val + ϕs) / rf_factor


def synthetic_bunch(n: int, sigma_z: float, sigma_E: float, seed: int) -> Particles:
    """Independent Gaussian (z, ΔE) from a seeded numpy Philox stream (the
    benchmark's initial distribution; the reference samples its bunch with
    generate_particles, src/evolution.jl:42-133, which is not on this path)."""
    rng = np.random.Generator(np.random.Philox(seed))
    return Particles(rng.normal(0.0, sigma_z, n), rng.normal(0.0, sigma_E, n))


@dataclass
class EvolveResult:
    sigma_E: float
    sigma_z: float
    E0: float
    sigma_E0_initial: float
    sigma_z0_initial: float
    mean_z: float
    mean_dE: float
    turns: int

    @staticmethod
    def from_c(r: HjResult) -> "EvolveResult":
        return EvolveResult(r.sigma_E, r.sigma_z, r.E0, r.sigma_E0_initial, r.sigma_z0_initial,
                            r.mean_z, r.mean_dE, r.turns)

    def as_tuple(self):
        return (self.sigma_E, self.sigma_z, self.E0)


# ----------------------------------------------------------------------------- evolution


def longitudinal_evolve(particles: Particles, params: SimulationParameters,
                        buffers: SimulationBuffers, comm=None, use_mpi: bool = False, *,
                        wake: Optional[WakeModel] = None, grid: Optional[BinGrid] = None,
                        qe_draws: Optional[np.ndarray] = None, seed: int = 0,
                        full_result: bool = False):
    """Drop-in for longitudinal_evolve!(particles, params, buffers, comm, use_mpi)
    (src/evolution.jl:206-470): tracks params.n_turns turns on the GPU,
    mutates particles in place and returns (σ_E, σ_z, E0).

    The wake follows the reference's MPI branch, the one that runs with the
    wakefield on.  `comm`/`use_mpi` are accepted for signature parity; a
    multi-rank run shards one bunch's particles over the ranks with
    ShardedBunch (one all-reduce of the bin exchange per turn).
    qe_draws: optional (n_turns, n) standard normals replacing randn!.
    """
    if use_mpi and comm is None:
        raise HaissinskiError(_lib.HJ_ERR_ARG, "MPI mode requires a valid MPI communicator.")
    ctx = buffers.context()
    z = _f64(particles.coordinates.z)
    dE = _f64(particles.coordinates.dE)
    n = z.shape[0]
    p = params.to_c()
    w = (wake or WakeModel.reference(params)).to_c()
    g = grid.to_c() if grid is not None else None
    draws = None
    if qe_draws is not None:
        draws = np.ascontiguousarray(qe_draws, dtype=np.float64)
        if draws.size != int(params.n_turns) * n:
            raise ValueError("qe_draws must hold n_turns * n values")
    res = HjResult()
    rc = ctx._lib.hj_evolve(ctx.handle, _dp(z), _dp(dE), n, ctypes.byref(p), ctypes.byref(w),
                            buffers.nbins, ctypes.byref(g) if g is not None else None,
                            _dp(draws), int(seed) & 0xFFFFFFFFFFFFFFFF, ctypes.byref(res))
    _check(ctx, rc)
    r = EvolveResult.from_c(res)
    return r if full_result else r.as_tuple()


# longitudinal_evolve! spelled the Julia way for callers that look it up by name.
globals()["longitudinal_evolve!"] = longitudinal_evolve


# ----------------------------------------------------------------------------- single steps


def rf_kick(voltage, sin_ϕs, rf_factor, ϕs, particles: Particles,
            buffers: SimulationBuffers) -> None:
    """rf_kick! (src/rf_kick.jl:18-87)."""
    ctx = buffers.context()
    z, dE = _f64(particles.coordinates.z), _f64(particles.coordinates.dE)
    _check(ctx, ctx._lib.hj_rf_kick(ctx.handle, voltage, sin_ϕs, rf_factor, ϕs, _dp(z), _dp(dE),
                                    z.shape[0]))


def quantum_excitation(E0, radius, σ_E0, buffers: SimulationBuffers, particles: Particles, *,
                       draws: Optional[np.ndarray] = None, seed: int = 0, turn: int = 1) -> None:
    """quantum_excitation! (src/quantum_excitation.jl:24-71).  draws replaces randn!;
    without it the on-device Philox normals of (seed, particle, turn) are used."""
    ctx = buffers.context()
    dE = _f64(particles.coordinates.dE)
    d = None if draws is None else np.ascontiguousarray(draws, dtype=np.float64)
    if d is not None and d.shape[0] != dE.shape[0]:
        raise ValueError("draws must have one value per particle")
    _check(ctx, ctx._lib.hj_quantum_excitation(ctx.handle, E0, radius, σ_E0, _dp(d),
                                               int(seed) & 0xFFFFFFFFFFFFFFFF, int(turn),
                                               _dp(dE), dE.shape[0]))


def synchrotron_radiation(E0, radius, particles: Particles, buffers: SimulationBuffers) -> None:
    """synchrotron_radiation! (src/synchrotron_radiation.jl:12-56)."""
    ctx = buffers.context()
    dE = _f64(particles.coordinates.dE)
    _check(ctx, ctx._lib.hj_synchrotron_radiation(ctx.handle, E0, radius, _dp(dE), dE.shape[0]))


def phase_advance(particles: Particles, params: SimulationParameters, E0: float,
                  buffers: SimulationBuffers) -> None:
    """The drift of longitudinal_evolve! (src/evolution.jl:329-348) at energy E0."""
    ctx = buffers.context()
    z, dE = _f64(particles.coordinates.z), _f64(particles.coordinates.dE)
    _check(ctx, ctx._lib.hj_phase_advance(ctx.handle, int(bool(params.update_eta)), E0,
                                          params.mass, params.alpha_c, int(params.harmonic),
                                          params.phi_s, params.freq_rf, _dp(dE), _dp(z),
                                          z.shape[0]))


def _grid_from(bin_edges, bin_centers) -> BinGrid:
    if isinstance(bin_edges, BinGrid):
        return bin_edges
    e = np.asarray(bin_edges, dtype=np.float64)
    c = np.ascontiguousarray(bin_centers, dtype=np.float64)
    if e.shape[0] != c.shape[0] + 1:
        raise HaissinskiError(_lib.HJ_ERR_ARG, "apply_wakefield_inplace: bin_edges length mismatch.")
    step = (e[-1] - e[0]) / (e.shape[0] - 1)
    return BinGrid(float(e[0]), float(e[-1]), float(step), c)


def calculate_local_histogram(z: np.ndarray, grid: BinGrid,
                              buffers: SimulationBuffers) -> np.ndarray:
    """calculate_local_histogram! (src/utils.jl:351-401): integer bin counts."""
    ctx = buffers.context()
    z = np.ascontiguousarray(z, dtype=np.float64)
    counts = np.zeros(grid.nbins, dtype=np.int64)
    g = grid.to_c()
    _check(ctx, ctx._lib.hj_histogram(ctx.handle, _dp(z), z.shape[0], ctypes.byref(g),
                                      _ip(counts)))
    return counts


def wake_potential(counts: np.ndarray, grid: BinGrid, wake: WakeModel, current: float,
                   buffers: SimulationBuffers) -> np.ndarray:
    """The convolution of apply_wakefield_inplace! (src/wakefield.jl:186-327)."""
    ctx = buffers.context()
    c = np.ascontiguousarray(counts, dtype=np.int64)
    pot = np.zeros(grid.nbins, dtype=np.float64)
    g, w = grid.to_c(), wake.to_c()
    _check(ctx, ctx._lib.hj_wake_potential(ctx.handle, _ip(c), ctypes.byref(g), ctypes.byref(w),
                                           float(current), _dp(pot)))
    return pot


def apply_wakefield_inplace(particles: Particles, buffers: SimulationBuffers, wake_factor,
                            wake_sqrt, cτ, current, sigma_z, bin_edges, bin_centers=None,
                            comm=None, use_mpi: bool = True, *, delta_std: float = 0.15,
                            sin_coef: float = 0.0) -> None:
    """apply_wakefield_inplace! (src/wakefield.jl:137-345), MPI-branch semantics.
    bin_edges may be a BinGrid (then bin_centers is ignored)."""
    ctx = buffers.context()
    grid = _grid_from(bin_edges, bin_centers)
    if grid.nbins != buffers.nbins:
        raise HaissinskiError(_lib.HJ_ERR_ARG, "apply_wakefield_inplace: bin_edges length mismatch.")
    z, dE = _f64(particles.coordinates.z), _f64(particles.coordinates.dE)
    w = WakeModel(wake_factor, wake_sqrt, cτ, sin_coef, 0.0, 7.5, delta_std).to_c()
    g = grid.to_c()
    _check(ctx, ctx._lib.hj_apply_wakefield(ctx.handle, _dp(z), _dp(dE), z.shape[0],
                                            ctypes.byref(w), float(current), float(sigma_z),
                                            ctypes.byref(g)))


def gaussian_draws(seed: int, turn: int, n: int, buffers: SimulationBuffers) -> np.ndarray:
    """The on-device Float64 normals of (seed, particle, turn): Philox-4x32-10 and
    a 2048-layer ziggurat (hj_gaussian)."""
    ctx = buffers.context()
    out = np.empty(n, dtype=np.float64)
    _check(ctx, ctx._lib.hj_gaussian(ctx.handle, int(seed) & 0xFFFFFFFFFFFFFFFF, int(turn), n,
                                     _dp(out)))
    return out


# ----------------------------------------------------------------------------- resident bunch


@dataclass
class Checkpoint:
    """hj_checkpoint: the next turn's number, E0 and the initial spreads."""

    turn: int
    E0: float
    sigma_E0_initial: float
    sigma_z0_initial: float


class ResidentBunch:
    """A bunch whose (z, ΔE) stay in device memory between calls.

    d_z, d_dE: device pointers (ints) to n float64 each, 32-byte aligned,
    owned by the caller (e.g. torch tensors' data_ptr()).  stream: a
    cudaStream_t as int (0 = legacy default stream).
    """

    def __init__(self, ctx: Context, d_z: int, d_dE: int, n: int, params: SimulationParameters,
                 nbins: int, *, wake: Optional[WakeModel] = None, grid: Optional[BinGrid] = None,
                 seed: int = 0, stream: int = 0):
        self.ctx = ctx
        self.n = int(n)
        self.nbins = int(nbins)
        self._p = params.to_c()
        self._w = (wake or WakeModel.reference(params)).to_c()
        self._grid = grid
        g = grid.to_c() if grid is not None else None
        h = ctypes.c_void_p()
        rc = ctx._lib.hj_bunch_create(ctx.handle, ctypes.c_void_p(d_z), ctypes.c_void_p(d_dE),
                                      self.n, ctypes.byref(self._p), ctypes.byref(self._w),
                                      self.nbins, ctypes.byref(g) if g is not None else None,
                                      int(seed) & 0xFFFFFFFFFFFFFFFF, ctypes.c_void_p(stream),
                                      ctypes.byref(h))
        _check(ctx, rc)
        self.handle = h

    def checkpoint(self, d_z_out: int, d_dE_out: int) -> "Checkpoint":
        """The particles at the turn boundary into device arrays (ints:
        pointers) and the checkpoint that continues the run
        (hj_bunch_checkpoint); the bunch runs on unchanged."""
        c = HjCheckpoint()
        _check(self.ctx, self.ctx._lib.hj_bunch_checkpoint(
            self.handle, ctypes.c_void_p(d_z_out), ctypes.c_void_p(d_dE_out), ctypes.byref(c)))
        return Checkpoint(int(c.turn), float(c.E0), float(c.sigma_E0_initial),
                          float(c.sigma_z0_initial))

    @classmethod
    def resume(cls, ctx: Context, d_z: int, d_dE: int, n: int, params: SimulationParameters,
               nbins: int, checkpoint: "Checkpoint", *, wake: Optional[WakeModel] = None,
               grid: Optional[BinGrid] = None, seed: int = 0,
               stream: int = 0) -> "ResidentBunch":
        """A bunch continuing from `checkpoint` (hj_bunch_resume): d_z, d_dE
        hold the checkpointed particles; turn counter, E0 and initial spreads
        come from the checkpoint; the same seed continues the same draws."""
        self = cls.__new__(cls)
        self.ctx = ctx
        self.n = int(n)
        self.nbins = int(nbins)
        self._p = params.to_c()
        self._w = (wake or WakeModel.reference(params)).to_c()
        self._grid = grid
        g = grid.to_c() if grid is not None else None
        c = HjCheckpoint(int(checkpoint.turn), float(checkpoint.E0),
                         float(checkpoint.sigma_E0_initial), float(checkpoint.sigma_z0_initial))
        h = ctypes.c_void_p()
        _check(ctx, ctx._lib.hj_bunch_resume(ctx.handle, ctypes.c_void_p(d_z), ctypes.c_void_p(d_dE),
                                             self.n, ctypes.byref(self._p), ctypes.byref(self._w),
                                             self.nbins, ctypes.byref(g) if g is not None else None,
                                             int(seed) & 0xFFFFFFFFFFFFFFFF, ctypes.byref(c),
                                             ctypes.c_void_p(stream), ctypes.byref(h)))
        self.handle = h
        return self

    def set_draws(self, d_draws: int, first_turn: int, turns: int) -> None:
        _check(self.ctx, self.ctx._lib.hj_bunch_set_draws(self.handle, ctypes.c_void_p(d_draws),
                                                          first_turn, turns))

    def advance(self, turns: int) -> None:
        _check(self.ctx, self.ctx._lib.hj_bunch_advance(self.handle, int(turns)))

    def observe(self, d_z_out: int = 0, d_dE_out: int = 0) -> EvolveResult:
        r = HjResult()
        _check(self.ctx, self.ctx._lib.hj_bunch_observe(
            self.handle, ctypes.c_void_p(d_z_out or None), ctypes.c_void_p(d_dE_out or None),
            ctypes.byref(r)))
        return EvolveResult.from_c(r)

    def finish(self) -> EvolveResult:
        r = HjResult()
        _check(self.ctx, self.ctx._lib.hj_bunch_finish(self.handle, ctypes.byref(r)))
        return EvolveResult.from_c(r)

    def set_profiling(self, enable: bool) -> None:
        _check(self.ctx, self.ctx._lib.hj_bunch_set_profiling(self.handle, int(bool(enable))))

    def read_profile(self) -> dict:
        out = np.zeros(4, dtype=np.float64)
        _check(self.ctx, self.ctx._lib.hj_bunch_read_profile(self.handle, _dp(out)))
        return {"pass_ms": float(out[0]), "bins_ms": float(out[1]), "turns": int(out[2]),
                "launches": int(out[3])}

    def set_log(self, every: int, capacity: int = 1024, density: bool = False) -> None:
        """Record [turn, E0, σ_z, σ_E, mean z, mean ΔE, current, n_in] (+ the bin
        counts with density) every `every` turns on the device."""
        self._log_density = bool(density)
        _check(self.ctx, self.ctx._lib.hj_bunch_set_log(self.handle, int(every), int(capacity),
                                                        int(bool(density))))

    def read_log(self, max_records: int = 1 << 20) -> np.ndarray:
        """The logged records, oldest first: rows of 8 (+ nbins) values."""
        width = 8 + (self.nbins if getattr(self, "_log_density", False) else 0)
        out = np.zeros((max_records, width), dtype=np.float64)
        n = np.zeros(1, dtype=np.int64)
        _check(self.ctx, self.ctx._lib.hj_bunch_read_log(self.handle, _dp(out), int(max_records),
                                                         _ip(n)))
        return out[: int(n[0])]

    def histogram(self) -> np.ndarray:
        out = np.zeros(self.nbins, dtype=np.int64)
        _check(self.ctx, self.ctx._lib.hj_bunch_histogram(self.handle, _ip(out)))
        return out

    def potential(self) -> np.ndarray:
        out = np.zeros(self.nbins, dtype=np.float64)
        _check(self.ctx, self.ctx._lib.hj_bunch_potential(self.handle, _dp(out)))
        return out

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.ctx._lib.hj_bunch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent bunches advanced together on one GPU (hj_batch_*).

    Each bunch has its own particles, RF voltage, wake intensity, bins, seed
    and turn count; every turn is one batched particle pass, one histogram
    merge and one batched bins step for all live bunches, and blocks of
    `graph_turns` turns replay a captured CUDA graph.  A bunch's results do
    not depend on which other bunches share the batch.

    pool_particles: particle capacity (16 B each on the device); max_bunches:
    bunch slots; max_nbins: largest bin count; chunk: particles per block of
    the pass (multiple of 4); layout: pass thread layout (-1 = default).
    """

    def __init__(self, ctx: Context, pool_particles: int, max_bunches: int, max_nbins: int,
                 chunk: int = 65536, layout: int = -1, graph_turns: int = 16,
                 resident: bool = False):
        self.ctx = ctx
        h = ctypes.c_void_p()
        _check(ctx, ctx._lib.hj_batch_create(ctx.handle, int(pool_particles), int(max_bunches),
                                             int(max_nbins), int(chunk), int(layout),
                                             ctypes.byref(h)))
        self.handle = h
        self.sizes = {}
        if graph_turns != 16:
            self.set_graph_turns(graph_turns)
        if resident:
            self.set_resident(True)

    def set_resident(self, on: bool) -> None:
        """Resident blocks on a device-side chunk queue (True) or one block per
        chunk (False, the default; hj_batch_set_resident)."""
        _check(self.ctx, self.ctx._lib.hj_batch_set_resident(self.handle, int(bool(on))))

    def set_graph_turns(self, turns: int) -> None:
        _check(self.ctx, self.ctx._lib.hj_batch_set_graph_turns(self.handle, int(turns)))

    def _add(self, zp, ep, n, params, nbins, wake, seed, turns) -> int:
        p = params.to_c()
        w = ctypes.byref(wake.to_c()) if wake is not None else None   # None: the reference's
        out = ctypes.c_int64(0)
        nt = params.n_turns if turns is None else int(turns)
        _check(self.ctx, self.ctx._lib.hj_batch_add(
            self.handle, zp, ep, int(n), ctypes.byref(p), w, int(nbins),
            int(seed) & 0xFFFFFFFFFFFFFFFF, nt, ctypes.byref(out)))
        bid = int(out.value)
        self.sizes[bid] = int(n)
        return bid

    def add(self, z, dE, params: SimulationParameters, nbins: int, *,
            wake: Optional[WakeModel] = None, seed: int = 0, turns: Optional[int] = None) -> int:
        """Admit a bunch from host arrays (copied); returns its id.  Raises
        HaissinskiError with status HJ_ERR_FULL when the batch has no room."""
        z = np.ascontiguousarray(z, dtype=np.float64)
        dE = np.ascontiguousarray(dE, dtype=np.float64)
        if z.shape != dE.shape:
            raise ValueError("z and dE differ in length")
        return self._add(z.ctypes.data_as(ctypes.c_void_p), dE.ctypes.data_as(ctypes.c_void_p),
                         z.size, params, nbins, wake, seed, turns)

    def add_device(self, d_z: int, d_dE: int, n: int, params: SimulationParameters, nbins: int,
                   *, wake: Optional[WakeModel] = None, seed: int = 0,
                   turns: Optional[int] = None) -> int:
        """As add(), from device pointers (ints), copied into the pool."""
        return self._add(ctypes.c_void_p(d_z), ctypes.c_void_p(d_dE), n, params, nbins, wake,
                         seed, turns)

    def add_gaussian(self, n: int, sigma_z: float, sigma_E: float, init_seed: int,
                     params: SimulationParameters, nbins: int, *,
                     wake: Optional[WakeModel] = None, seed: int = 0,
                     turns: Optional[int] = None) -> int:
        """Admit a bunch of n independent Gaussians generated on the device
        (gaussian_bunch with init_seed); returns its id."""
        p = params.to_c()
        w = (wake or WakeModel.reference(params)).to_c()
        out = np.zeros(1, dtype=np.int64)
        nt = params.n_turns if turns is None else int(turns)
        _check(self.ctx, self.ctx._lib.hj_batch_add_gaussian(
            self.handle, int(n), float(sigma_z), float(sigma_E),
            int(init_seed) & 0xFFFFFFFFFFFFFFFF, ctypes.byref(p), ctypes.byref(w), int(nbins),
            int(seed) & 0xFFFFFFFFFFFFFFFF, nt, _ip(out)))
        bid = int(out[0])
        self.sizes[bid] = int(n)
        return bid

    def advance(self, turns: int) -> None:
        _check(self.ctx, self.ctx._lib.hj_batch_advance(self.handle, int(turns)))

    def poll(self, cap: int = 4096) -> list:
        """Waits for the enqueued turns; ids of bunches that ran all their turns."""
        ids = np.zeros(max(cap, 1), dtype=np.int64)
        n = ctypes.c_int32(0)
        _check(self.ctx, self.ctx._lib.hj_batch_poll(self.handle, _ip(ids), int(cap),
                                                     ctypes.byref(n)))
        return [int(x) for x in ids[: n.value]]

    def take(self, bid: int, copy_out: bool = True):
        """Finishes bunch `bid` and frees its slot; returns (z, dE, EvolveResult)
        (z and dE are None without copy_out)."""
        n = self._size(bid)
        z = np.empty(n) if copy_out else None
        dE = np.empty(n) if copy_out else None
        r = HjResult()
        live = self._live()
        rc = self.ctx._lib.hj_batch_take(
            self.handle, int(bid), z.ctypes.data_as(ctypes.c_void_p) if copy_out else None,
            dE.ctypes.data_as(ctypes.c_void_p) if copy_out else None, ctypes.byref(r))
        self._forget([bid], rc, live)
        return z, dE, EvolveResult.from_c(r)

    def _live(self) -> int:
        """Bunches the library holds in this batch (hj_batch_stats, host only)."""
        out = np.zeros(4, dtype=np.int64)
        _check(self.ctx, self.ctx._lib.hj_batch_stats(self.handle, _ip(out)))
        return int(out[0])

    def _forget(self, ids, rc: int, live_before: int) -> None:
        """Drop `ids` from the host bookkeeping once the library has retired
        them, then raise if the call failed.  hj_batch_take(_many) retires its
        bunches as soon as their results are read back and reports a bunch's
        own failure (a non-finite result, short host-fed draws) only after
        that, so a failed take may or may not have retired them: the live
        count says which."""
        if rc == _lib.HJ_OK or self._live() < live_before:
            for b in ids:
                self.sizes.pop(int(b), None)
        _check(self.ctx, rc)

    def _size(self, bid: int) -> int:
        if bid not in self.sizes:
            raise HaissinskiError(_lib.HJ_ERR_ARG, f"no bunch {bid} in this batch")
        return self.sizes[bid]

    def take_device(self, bid: int, d_z: int, d_dE: int) -> EvolveResult:
        """As take(), with (z, dE) copied to device arrays (ints: pointers)."""
        self._size(bid)
        r = HjResult()
        live = self._live()
        rc = self.ctx._lib.hj_batch_take(self.handle, int(bid), ctypes.c_void_p(d_z),
                                         ctypes.c_void_p(d_dE), ctypes.byref(r))
        self._forget([bid], rc, live)
        return EvolveResult.from_c(r)

    def add_many(self, z, dE, n, params, nbins, seeds, turns, wakes=None):
        """Admit bunches in order with one synchronisation (hj_batch_add_many).
        z, dE: per-bunch particle arrays as pointers (ints, host or device) or
        numpy arrays (host, kept alive by the caller until the call returns);
        n, params, nbins, seeds, turns: per-bunch values; wakes: None (each
        params' reference wake) or a list of WakeModel.  Returns (ids of the
        admitted bunches -- the first ones --, the HaissinskiError that stopped
        admission, or None)."""
        k = len(n)
        keep = []                         # host arrays converted for the call

        def ptrs(a):
            arr = (ctypes.c_void_p * max(k, 1))()
            for i, x in enumerate(a):
                if not isinstance(x, int):
                    x = np.ascontiguousarray(x, dtype=np.float64)
                    keep.append(x)
                    x = x.ctypes.data
                arr[i] = x
            return arr
        zp, ep = ptrs(z), ptrs(dE)
        nn = np.ascontiguousarray(n, dtype=np.int64)
        pc = (HjParams * max(k, 1))(*[p.to_c() for p in params])
        wc = None if wakes is None else (HjWake * max(k, 1))(*[w.to_c() for w in wakes])
        nb = np.ascontiguousarray(nbins, dtype=np.int64)
        sd = (ctypes.c_uint64 * max(k, 1))(*[int(x) & 0xFFFFFFFFFFFFFFFF for x in seeds])
        tt = np.ascontiguousarray(turns, dtype=np.int64)
        ids = np.zeros(max(k, 1), dtype=np.int64)
        added = ctypes.c_int32(0)
        rc = self.ctx._lib.hj_batch_add_many(self.handle, k, zp, ep, _ip(nn), pc, wc, _ip(nb), sd,
                                             _ip(tt), _ip(ids), ctypes.byref(added))
        out = [int(x) for x in ids[: added.value]]
        for bid, size in zip(out, nn):
            self.sizes[bid] = int(size)
        err = None
        if rc != 0:
            err = HaissinskiError(rc, self.ctx.last_error())
        return out, err

    def take_many(self, ids, correlation: bool = False):
        """Finish and free bunches `ids` with one synchronisation
        (hj_batch_take_many); returns (results, correlations or None)."""
        k = len(ids)
        idv = np.ascontiguousarray(ids, dtype=np.int64)
        res = (HjResult * max(k, 1))()
        corr = np.zeros(max(k, 1)) if correlation else None
        live = self._live()
        rc = self.ctx._lib.hj_batch_take_many(
            self.handle, k, _ip(idv), None, None, res, _dp(corr) if correlation else None)
        self._forget(ids, rc, live)          # all of them retire, or none
        results = [EvolveResult.from_c(res[i]) for i in range(k)]
        return results, ([float(c) for c in corr[:k]] if correlation else None)

    def histogram(self, bid: int, nbins: int) -> np.ndarray:
        """Bin counts of bunch `bid`'s last completed turn (hj_batch_histogram)."""
        self._size(bid)
        out = np.zeros(int(nbins), dtype=np.int64)
        _check(self.ctx, self.ctx._lib.hj_batch_histogram(self.handle, int(bid), _ip(out)))
        return out

    def stats(self) -> dict:
        out = np.zeros(4, dtype=np.int64)
        _check(self.ctx, self.ctx._lib.hj_batch_stats(self.handle, _ip(out)))
        return {"live": int(out[0]), "largest_free_particles": int(out[1]),
                "free_slots": int(out[2]), "turns_enqueued": int(out[3])}

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.ctx._lib.hj_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gaussian_bunch(ctx: Context, init_seed: int, n: int, sigma_z: float, sigma_E: float,
                   d_z: int, d_dE: int, stream: int = 0) -> None:
    """Fill device arrays (ints: pointers) with n independent Gaussians
    z ~ N(0, sigma_z), dE ~ N(0, sigma_E) from init_seed, on `stream`."""
    _check(ctx, ctx._lib.hj_gaussian_bunch(ctx.handle, int(init_seed) & 0xFFFFFFFFFFFFFFFF,
                                           int(n), float(sigma_z), float(sigma_E),
                                           ctypes.c_void_p(d_z), ctypes.c_void_p(d_dE),
                                           ctypes.c_void_p(stream)))


class _DeviceArray:
    """A device buffer (pointer, length, numpy typestr) seen by torch.as_tensor."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3}


class ShardedBunch:
    """One shard of a bunch split over processes (hj_bunch_create_shard).

    Particles [first_particle, first_particle + n_local) of n_global live on
    this process's GPU (device pointers d_z, d_dE); per turn: `pass_()`, a SUM
    all-reduce of `buffers()` across ranks, `bins()` -- which `advance()` does
    with torch.distributed on the shard's stream (NCCL).  The grid must be the
    same on every rank.  With the Philox draws of the whole bunch, the ranks
    together reproduce the single-GPU run (sums in another order).
    """

    def __init__(self, ctx: Context, d_z: int, d_dE: int, n_local: int, first_particle: int,
                 n_global: int, params: SimulationParameters, grid: "BinGrid", *,
                 wake: Optional[WakeModel] = None, seed: int = 0, stream: int = 0,
                 group=None, exchange_initial: bool = True):
        self.ctx = ctx
        self.n_local, self.n_global, self.nbins = int(n_local), int(n_global), grid.nbins
        self.group = group
        self.stream = stream
        self._p = params.to_c()
        self._w = (wake or WakeModel.reference(params)).to_c()
        self._grid = grid
        g = grid.to_c()
        h = ctypes.c_void_p()
        _check(ctx, ctx._lib.hj_bunch_create_shard(
            ctx.handle, ctypes.c_void_p(d_z), ctypes.c_void_p(d_dE), self.n_local,
            int(first_particle), self.n_global, ctypes.byref(self._p), ctypes.byref(self._w),
            ctypes.byref(g), int(seed) & 0xFFFFFFFFFFFFFFFF, ctypes.c_void_p(stream),
            ctypes.byref(h)))
        self.handle = h
        if exchange_initial:
            self.set_global_moments(self._all_reduce_host(self.local_moments()))

    # -- per-turn steps
    def pass_(self) -> None:
        _check(self.ctx, self.ctx._lib.hj_bunch_pass(self.handle))

    def buffers(self):
        """(counts, sums) as torch tensors viewing the device exchange buffers."""
        import torch
        cp, sp = ctypes.c_void_p(), ctypes.c_void_p()
        nc, ns = np.zeros(1, dtype=np.int64), np.zeros(1, dtype=np.int64)
        _check(self.ctx, self.ctx._lib.hj_bunch_exchange_buffers(
            self.handle, ctypes.byref(cp), _ip(nc), ctypes.byref(sp), _ip(ns)))
        counts = torch.as_tensor(_DeviceArray(cp.value, nc[0], "<i8"), device="cuda")
        sums = torch.as_tensor(_DeviceArray(sp.value, ns[0], "<f8"), device="cuda")
        return counts, sums

    def bins(self) -> None:
        _check(self.ctx, self.ctx._lib.hj_bunch_bins(self.handle))

    def advance(self, turns: int) -> None:
        import torch.distributed as dist
        counts, sums = self.buffers()
        for _ in range(int(turns)):
            self.pass_()
            dist.all_reduce(counts, group=self.group)
            dist.all_reduce(sums, group=self.group)
            self.bins()

    # -- moments
    def local_moments(self) -> np.ndarray:
        out = np.zeros(4, dtype=np.float64)
        _check(self.ctx, self.ctx._lib.hj_bunch_local_moments(self.handle, _dp(out)))
        return out

    def set_global_moments(self, sums4) -> None:
        s = np.ascontiguousarray(sums4, dtype=np.float64)
        _check(self.ctx, self.ctx._lib.hj_bunch_set_global_moments(self.handle, _dp(s)))

    def _all_reduce_host(self, v: np.ndarray) -> np.ndarray:
        import torch
        import torch.distributed as dist
        if not (dist.is_available() and dist.is_initialized()):
            return v
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.from_numpy(v.copy()).to(dev)
        dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def global_result(self, sums4=None) -> EvolveResult:
        """(σ_E, σ_z, E0, ...) of the whole bunch (pending kick applied), from
        the moments summed over the ranks (or the given sums) with the
        reference's single-pass formula (src/utils.jl:593-605)."""
        m = self._all_reduce_host(self.local_moments()) if sums4 is None else np.asarray(sums4)
        r = self.observe_local()
        n = self.n_global

        def gstd(s, s2):
            if n <= 1:
                return 0.0
            mean = s / n
            var = (s2 / n) - mean * mean
            v = var * n / (n - 1)
            return math.sqrt(v) if v > 0 else (v if v != v else 0.0)
        return EvolveResult(gstd(m[2], m[3]), gstd(m[0], m[1]), r.E0, r.sigma_E0_initial,
                            r.sigma_z0_initial, m[0] / n, m[2] / n, r.turns)

    def observe_local(self, d_z_out: int = 0, d_dE_out: int = 0) -> EvolveResult:
        r = HjResult()
        _check(self.ctx, self.ctx._lib.hj_bunch_observe(
            self.handle, ctypes.c_void_p(d_z_out or None), ctypes.c_void_p(d_dE_out or None),
            ctypes.byref(r)))
        return EvolveResult.from_c(r)

    def finish(self) -> None:
        """Apply the pending kick and re-centring to the shard's particles."""
        r = HjResult()
        _check(self.ctx, self.ctx._lib.hj_bunch_finish(self.handle, ctypes.byref(r)))

    def histogram(self) -> np.ndarray:
        out = np.zeros(self.nbins, dtype=np.int64)
        _check(self.ctx, self.ctx._lib.hj_bunch_histogram(self.handle, _ip(out)))
        return out

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.ctx._lib.hj_bunch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def generate_particles_device(ctx: Context, mu_z: float, mu_E: float, sigma_z: float,
                              sigma_E: float, n: int, d_z: int, d_dE: int, *, seed: int = 0,
                              stream: int = 0):
    """generate_particles (src/evolution.jl:42-133) into device arrays (ints:
    pointers); returns (actual σ_E, actual σ_z)."""
    sE = np.zeros(1)
    sz = np.zeros(1)
    _check(ctx, ctx._lib.hj_generate_particles(ctx.handle, float(mu_z), float(mu_E),
                                               float(sigma_z), float(sigma_E), int(n),
                                               int(seed) & 0xFFFFFFFFFFFFFFFF,
                                               ctypes.c_void_p(d_z), ctypes.c_void_p(d_dE),
                                               ctypes.c_void_p(stream), _dp(sE), _dp(sz)))
    return float(sE[0]), float(sz[0])


def generate_particles(mu_z: float, mu_E: float, sigma_z: float, sigma_E: float,
                       num_particles: int, energy: float, mass: float = MASS_ELECTRON,
                       phi_s: float = 0.0, freq_rf: float = 0.0, *,
                       ctx: Optional[Context] = None, seed: int = 0):
    """The reference's generate_particles(μ_z, μ_E, σ_z, σ_E, num_particles,
    energy, mass, ϕs, freq_rf) -> (particles, actual σ_E, actual σ_z, energy),
    drawn on the GPU (mass, ϕs and freq_rf are accepted for signature parity
    and, as in the reference, unused)."""
    import torch
    ctx = ctx or Context(0)
    n = max(int(num_particles), 0)
    dz = torch.empty(max(n, 1), dtype=torch.float64, device="cuda")
    de = torch.empty_like(dz)
    sE, sz = generate_particles_device(ctx, mu_z, mu_E, sigma_z, sigma_E, n, dz.data_ptr(),
                                       de.data_ptr(), seed=seed)
    return Particles(dz[:n].cpu().numpy(), de[:n].cpu().numpy()), sE, sz, energy


def correlation_device(ctx: Context, d_x: int, d_y: int, n: int, stream: int = 0) -> float:
    """Pearson correlation of two device arrays of n doubles (ints: pointers),
    two passes on the GPU (hj_correlation): the cor(z, ΔE) of EmittanceFoM
    (src/parameter_sensitivity/figures_of_merit.jl:42)."""
    out = np.zeros(1)
    _check(ctx, ctx._lib.hj_correlation(ctx.handle, ctypes.c_void_p(d_x), ctypes.c_void_p(d_y),
                                        int(n), ctypes.c_void_p(stream), _dp(out)))
    return float(out[0])
