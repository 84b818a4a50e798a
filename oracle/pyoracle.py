"""ctypes wrapper of the C oracle (oracle.c).  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int32, c_int64, c_uint64, c_void_p
from typing import Optional

import numpy as np

from haissinskijulia_b200._lib import HjGrid, HjParams, HjResult, HjWake

from . import build_oracle

_DP = POINTER(c_double)
_IP = POINTER(c_int64)

SIGS = {
    "or_set_threads": (None, [c_int32]),
    "or_get_threads": (c_int32, []),
    "or_compute_global_std": (c_double, [_DP, c_int64]),
    "or_compute_std": (c_double, [_DP, c_int64]),
    "or_calc_rf_factor": (c_double, [c_double, c_double]),
    "or_next_power_of_two": (c_int64, [c_int64]),
    "or_delta": (c_double, [c_double, c_double]),
    "or_wake_function": (c_double, [c_double, POINTER(HjWake)]),
    "or_rf_kick": (None, [c_double, c_double, c_double, c_double, _DP, _DP, c_int64]),
    "or_quantum_excitation": (None, [c_double, c_double, c_double, _DP, _DP, c_int64]),
    "or_synchrotron_radiation": (None, [c_double, c_double, _DP, c_int64]),
    "or_drift_update_eta": (None, [c_double, c_double, c_double, c_int64, c_double, c_double,
                                   _DP, _DP, c_int64]),
    "or_apply_phase_advance": (c_int32, [c_double, c_double, c_double, c_int64, c_double,
                                         c_double, _DP, _DP, c_int64]),
    "or_histogram": (None, [_DP, c_int64, POINTER(HjGrid), _IP]),
    "or_wake_potential": (None, [_IP, POINTER(HjGrid), POINTER(HjWake), c_double, c_int32, _DP]),
    "or_interp_kick": (None, [_DP, _DP, c_int64, POINTER(HjGrid), _DP]),
    "or_wake_current": (c_double, [c_int64, c_double, c_double, c_double, c_double, c_double,
                                   c_double, c_double]),
    "or_make_grid": (c_int32, [c_double, c_double, c_int64, _DP, POINTER(HjGrid)]),
    "or_gaussian": (None, [c_uint64, c_int64, c_int64, _DP]),
    "or_create": (c_void_p, [_DP, _DP, c_int64, POINTER(HjParams), POINTER(HjWake), c_int64,
                             POINTER(HjGrid), c_uint64, c_int32]),
    "or_turn": (c_int32, [c_void_p, _DP]),
    "or_result": (None, [c_void_p, POINTER(HjResult)]),
    "or_last_sigma_z": (c_double, [c_void_p]),
    "or_last_current": (c_double, [c_void_p]),
    "or_last_mean": (c_double, [c_void_p]),
    "or_E0": (c_double, [c_void_p]),
    "or_nbins": (c_int64, [c_void_p]),
    "or_centers": (_DP, [c_void_p]),
    "or_last_counts": (_IP, [c_void_p]),
    "or_last_potential": (_DP, [c_void_p]),
    "or_grid_edge_first": (c_double, [c_void_p]),
    "or_grid_edge_last": (c_double, [c_void_p]),
    "or_grid_edge_step": (c_double, [c_void_p]),
    "or_destroy": (None, [c_void_p]),
    "or_evolve": (c_int32, [_DP, _DP, c_int64, POINTER(HjParams), POINTER(HjWake), c_int64,
                            POINTER(HjGrid), _DP, c_uint64, c_int32, POINTER(HjResult)]),
    "or_wake_reference": (None, [POINTER(HjParams), POINTER(HjWake)]),
}

CONV_FFT = 0
CONV_DIRECT_LD = 1


def _dp(a):
    return None if a is None else a.ctypes.data_as(_DP)


def _ip(a):
    return a.ctypes.data_as(_IP)


class Oracle:
    """Loaded oracle library with numpy-friendly helpers."""

    _lib = None

    def __init__(self, threads: int = 1):
        if Oracle._lib is None:
            path = build_oracle.build()
            lib = ctypes.CDLL(str(path))
            for name, (res, args) in SIGS.items():
                f = getattr(lib, name)
                f.restype = res
                f.argtypes = args
            Oracle._lib = lib
        self.lib = Oracle._lib
        self.lib.or_set_threads(int(threads))

    def set_threads(self, t: int) -> None:
        self.lib.or_set_threads(int(t))

    # ---- single steps (in place on numpy arrays)
    def rf_kick(self, V, sin_phis, k, phi_s, z, dE):
        self.lib.or_rf_kick(V, sin_phis, k, phi_s, _dp(z), _dp(dE), z.shape[0])

    def quantum_excitation(self, E0, radius, sigma_E0, draws, dE):
        self.lib.or_quantum_excitation(E0, radius, sigma_E0, _dp(draws), _dp(dE), dE.shape[0])

    def synchrotron_radiation(self, E0, radius, dE):
        self.lib.or_synchrotron_radiation(E0, radius, _dp(dE), dE.shape[0])

    def drift(self, update_eta, E0, mass, alpha_c, harmonic, phi_s, freq_rf, dE, z):
        if update_eta:
            self.lib.or_drift_update_eta(E0, mass, alpha_c, harmonic, phi_s, freq_rf, _dp(dE),
                                         _dp(z), z.shape[0])
            return 0
        return self.lib.or_apply_phase_advance(E0, mass, alpha_c, harmonic, phi_s, freq_rf,
                                               _dp(dE), _dp(z), z.shape[0])

    def histogram(self, z, grid_c: HjGrid) -> np.ndarray:
        counts = np.zeros(grid_c.nbins, dtype=np.int64)
        self.lib.or_histogram(_dp(z), z.shape[0], ctypes.byref(grid_c), _ip(counts))
        return counts

    def wake_potential(self, counts, grid_c: HjGrid, wake_c: HjWake, current,
                       conv=CONV_FFT) -> np.ndarray:
        pot = np.zeros(grid_c.nbins, dtype=np.float64)
        c = np.ascontiguousarray(counts, dtype=np.int64)
        self.lib.or_wake_potential(_ip(c), ctypes.byref(grid_c), ctypes.byref(wake_c),
                                   float(current), conv, _dp(pot))
        return pot

    def interp_kick(self, z, dE, grid_c: HjGrid, pot):
        self.lib.or_interp_kick(_dp(z), _dp(dE), z.shape[0], ctypes.byref(grid_c), _dp(pot))

    def gaussian(self, seed, turn, n) -> np.ndarray:
        out = np.empty(n, dtype=np.float64)
        self.lib.or_gaussian(int(seed) & 0xFFFFFFFFFFFFFFFF, int(turn), n, _dp(out))
        return out

    def wake_current(self, n_global, E0, mass, alpha_c, radius, sigma_z, sigma_E0_initial,
                     population) -> float:
        return self.lib.or_wake_current(int(n_global), E0, mass, alpha_c, radius, sigma_z,
                                        sigma_E0_initial, population)

    def rf_factor(self, freq_rf, beta) -> float:
        return self.lib.or_calc_rf_factor(freq_rf, beta)

    def global_std(self, x) -> float:
        x = np.ascontiguousarray(x, dtype=np.float64)
        return self.lib.or_compute_global_std(_dp(x), x.shape[0])

    def make_grid(self, sigma_z0, half_width, nbins):
        c = np.empty(max(nbins, 1), dtype=np.float64)
        g = HjGrid()
        rc = self.lib.or_make_grid(sigma_z0, half_width, nbins, _dp(c), ctypes.byref(g))
        return rc, g, c

    def evolve(self, z, dE, params_c: HjParams, wake_c: Optional[HjWake], nbins: int,
               grid_c: Optional[HjGrid] = None, draws=None, seed: int = 0,
               conv=CONV_FFT) -> tuple[int, HjResult]:
        res = HjResult()
        rc = self.lib.or_evolve(_dp(z), _dp(dE), z.shape[0], ctypes.byref(params_c),
                                ctypes.byref(wake_c) if wake_c is not None else None, nbins,
                                ctypes.byref(grid_c) if grid_c is not None else None,
                                _dp(draws), int(seed) & 0xFFFFFFFFFFFFFFFF, conv,
                                ctypes.byref(res))
        return rc, res

    def state(self, z, dE, params_c, wake_c, nbins, grid_c=None, seed=0, conv=CONV_FFT):
        return OracleState(self, z, dE, params_c, wake_c, nbins, grid_c, seed, conv)


class OracleState:
    """Turn-by-turn oracle over caller-owned numpy arrays (updated in place)."""

    def __init__(self, orc: Oracle, z, dE, params_c, wake_c, nbins, grid_c, seed, conv):
        self.orc = orc
        self.z, self.dE = z, dE
        self._keep = (params_c, wake_c, grid_c)
        h = orc.lib.or_create(_dp(z), _dp(dE), z.shape[0], ctypes.byref(params_c),
                              ctypes.byref(wake_c) if wake_c is not None else None, nbins,
                              ctypes.byref(grid_c) if grid_c is not None else None,
                              int(seed) & 0xFFFFFFFFFFFFFFFF, conv)
        if not h:
            raise RuntimeError("or_create failed")
        self.h = h

    def turn(self, draws=None) -> int:
        return self.orc.lib.or_turn(self.h, _dp(draws))

    def result(self) -> HjResult:
        r = HjResult()
        self.orc.lib.or_result(self.h, ctypes.byref(r))
        return r

    @property
    def E0(self) -> float:
        return self.orc.lib.or_E0(self.h)

    @property
    def last_sigma_z(self) -> float:
        return self.orc.lib.or_last_sigma_z(self.h)

    @property
    def last_current(self) -> float:
        return self.orc.lib.or_last_current(self.h)

    @property
    def last_mean(self) -> float:
        return self.orc.lib.or_last_mean(self.h)

    def counts(self) -> np.ndarray:
        B = self.orc.lib.or_nbins(self.h)
        return np.ctypeslib.as_array(self.orc.lib.or_last_counts(self.h), shape=(B,)).copy()

    def potential(self) -> np.ndarray:
        B = self.orc.lib.or_nbins(self.h)
        return np.ctypeslib.as_array(self.orc.lib.or_last_potential(self.h), shape=(B,)).copy()

    def centers(self) -> np.ndarray:
        B = self.orc.lib.or_nbins(self.h)
        return np.ctypeslib.as_array(self.orc.lib.or_centers(self.h), shape=(B,)).copy()

    def grid_edges(self):
        l = self.orc.lib
        return l.or_grid_edge_first(self.h), l.or_grid_edge_last(self.h), l.or_grid_edge_step(self.h)

    def close(self):
        if self.h:
            self.orc.lib.or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
