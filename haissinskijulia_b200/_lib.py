"""ctypes binding of libhaissinski_gpu.so (the C ABI in include/haissinski_gpu.h).

The library is loaded from this package directory.  There is no fallback:
if the shared object is missing the import of any compute entry point fails
with an error that says how to build it.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_int32, c_int64, c_uint8, c_uint64, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libhaissinski_gpu.so"

HJ_OK = 0
HJ_ERR_ARG = 1
HJ_ERR_NBINS = 2
HJ_ERR_WAKE_PARAM = 3
HJ_ERR_CUDA = 4
HJ_ERR_NOMEM = 5
HJ_ERR_TOO_LARGE = 6
HJ_ERR_EMPTY = 7
HJ_ERR_NONFINITE = 8
HJ_ERR_TIMEOUT = 9
HJ_ERR_NO_DEVICE = 10
HJ_ERR_STATE = 11
HJ_ERR_FULL = 12


class HjParams(ctypes.Structure):
    """Mirror of SimulationParameters (src/data_structures.jl:81-97)."""

    _fields_ = [
        ("E0", c_double),
        ("mass", c_double),
        ("voltage", c_double),
        ("harmonic", c_int64),
        ("radius", c_double),
        ("pipe_radius", c_double),
        ("alpha_c", c_double),
        ("phi_s", c_double),
        ("freq_rf", c_double),
        ("n_turns", c_int64),
        ("use_wakefield", c_uint8),
        ("update_eta", c_uint8),
        ("update_E0", c_uint8),
        ("SR_damping", c_uint8),
        ("use_excitation", c_uint8),
        ("_pad", c_uint8 * 3),
    ]


class HjWake(ctypes.Structure):
    _fields_ = [
        ("wake_factor", c_double),
        ("wake_sqrt", c_double),
        ("ctau", c_double),
        ("sin_coef", c_double),
        ("population", c_double),
        ("half_width_sigmas", c_double),
        ("delta_std", c_double),
    ]


class HjGrid(ctypes.Structure):
    _fields_ = [
        ("nbins", c_int64),
        ("edge_first", c_double),
        ("edge_last", c_double),
        ("edge_step", c_double),
        ("centers", POINTER(c_double)),
    ]


class HjResult(ctypes.Structure):
    _fields_ = [
        ("sigma_E", c_double),
        ("sigma_z", c_double),
        ("E0", c_double),
        ("sigma_E0_initial", c_double),
        ("sigma_z0_initial", c_double),
        ("mean_z", c_double),
        ("mean_dE", c_double),
        ("turns", c_int64),
    ]


class HjCheckpoint(ctypes.Structure):
    _fields_ = [
        ("turn", c_int64),
        ("E0", c_double),
        ("sigma_E0_initial", c_double),
        ("sigma_z0_initial", c_double),
    ]


_DP = POINTER(c_double)
_IP = POINTER(c_int64)
_CTX = c_void_p
_BUNCH = c_void_p

# name -> (restype, argtypes); every entry is declared in include/haissinski_gpu.h
SIGNATURES = {
    "hj_version": (c_char_p, []),
    "hj_status_string": (c_char_p, [c_int32]),
    "hj_create": (c_int32, [c_int32, POINTER(_CTX)]),
    "hj_destroy": (None, [_CTX]),
    "hj_last_error": (c_char_p, [_CTX]),
    "hj_trim": (c_int32, [_CTX]),
    "hj_set_pass_layout": (c_int32, [_CTX, c_int32]),
    "hj_wake_reference": (c_int32, [POINTER(HjParams), POINTER(HjWake)]),
    "hj_wake_resonator": (c_int32, [c_double, c_double, c_double, c_double, c_double,
                                    POINTER(HjWake)]),
    "hj_make_grid": (c_int32, [c_double, c_double, c_int64, _DP, POINTER(HjGrid)]),
    "hj_evolve": (c_int32, [_CTX, _DP, _DP, c_int64, POINTER(HjParams), POINTER(HjWake),
                            c_int64, POINTER(HjGrid), _DP, c_uint64, POINTER(HjResult)]),
    "hj_evolve_device": (c_int32, [_CTX, c_void_p, c_void_p, c_int64, POINTER(HjParams),
                                   POINTER(HjWake), c_int64, POINTER(HjGrid), c_void_p,
                                   c_uint64, c_void_p, POINTER(HjResult)]),
    "hj_bunch_create": (c_int32, [_CTX, c_void_p, c_void_p, c_int64, POINTER(HjParams),
                                  POINTER(HjWake), c_int64, POINTER(HjGrid), c_uint64,
                                  c_void_p, POINTER(_BUNCH)]),
    "hj_bunch_set_draws": (c_int32, [_BUNCH, c_void_p, c_int64, c_int64]),
    "hj_bunch_advance": (c_int32, [_BUNCH, c_int64]),
    "hj_bunch_observe": (c_int32, [_BUNCH, c_void_p, c_void_p, POINTER(HjResult)]),
    "hj_bunch_finish": (c_int32, [_BUNCH, POINTER(HjResult)]),
    "hj_bunch_set_profiling": (c_int32, [_BUNCH, c_int32]),
    "hj_bunch_read_profile": (c_int32, [_BUNCH, _DP]),
    "hj_bunch_histogram": (c_int32, [_BUNCH, _IP]),
    "hj_bunch_checkpoint": (c_int32, [_BUNCH, c_void_p, c_void_p, POINTER(HjCheckpoint)]),
    "hj_bunch_resume": (c_int32, [_CTX, c_void_p, c_void_p, c_int64, POINTER(HjParams),
                                  POINTER(HjWake), c_int64, POINTER(HjGrid), c_uint64,
                                  POINTER(HjCheckpoint), c_void_p, POINTER(_BUNCH)]),
    "hj_bunch_potential": (c_int32, [_BUNCH, _DP]),
    "hj_bunch_set_log": (c_int32, [_BUNCH, c_int64, c_int64, c_int32]),
    "hj_bunch_read_log": (c_int32, [_BUNCH, _DP, c_int64, _IP]),
    "hj_bunch_destroy": (None, [_BUNCH]),
    "hj_bunch_create_shard": (c_int32, [_CTX, c_void_p, c_void_p, c_int64, c_int64, c_int64,
                                        POINTER(HjParams), POINTER(HjWake), POINTER(HjGrid),
                                        c_uint64, c_void_p, POINTER(_BUNCH)]),
    "hj_bunch_local_moments": (c_int32, [_BUNCH, _DP]),
    "hj_bunch_set_global_moments": (c_int32, [_BUNCH, _DP]),
    "hj_bunch_pass": (c_int32, [_BUNCH]),
    "hj_bunch_exchange_buffers": (c_int32, [_BUNCH, POINTER(c_void_p), _IP, POINTER(c_void_p),
                                            _IP]),
    "hj_bunch_bins": (c_int32, [_BUNCH]),
    "hj_batch_create": (c_int32, [_CTX, c_int64, c_int32, c_int32, c_int64, c_int32,
                                  POINTER(c_void_p)]),
    "hj_batch_destroy": (None, [c_void_p]),
    "hj_batch_set_graph_turns": (c_int32, [c_void_p, c_int32]),
    "hj_batch_set_resident": (c_int32, [c_void_p, c_int32]),
    "hj_batch_add": (c_int32, [c_void_p, c_void_p, c_void_p, c_int64, POINTER(HjParams),
                               POINTER(HjWake), c_int64, c_uint64, c_int64, _IP]),
    "hj_batch_add_gaussian": (c_int32, [c_void_p, c_int64, c_double, c_double, c_uint64,
                                        POINTER(HjParams), POINTER(HjWake), c_int64, c_uint64,
                                        c_int64, _IP]),
    "hj_gaussian_bunch": (c_int32, [_CTX, c_uint64, c_int64, c_double, c_double, c_void_p,
                                    c_void_p, c_void_p]),
    "hj_batch_advance": (c_int32, [c_void_p, c_int64]),
    "hj_batch_poll": (c_int32, [c_void_p, _IP, c_int32, POINTER(c_int32)]),
    "hj_batch_take": (c_int32, [c_void_p, c_int64, c_void_p, c_void_p, POINTER(HjResult)]),
    "hj_batch_stats": (c_int32, [c_void_p, _IP]),
    "hj_batch_histogram": (c_int32, [c_void_p, c_int64, _IP]),
    "hj_batch_add_many": (c_int32, [c_void_p, c_int32, POINTER(c_void_p), POINTER(c_void_p), _IP,
                                    POINTER(HjParams), POINTER(HjWake), _IP, POINTER(c_uint64),
                                    _IP, _IP, POINTER(c_int32)]),
    "hj_batch_take_many": (c_int32, [c_void_p, c_int32, _IP, POINTER(c_void_p),
                                     POINTER(c_void_p), POINTER(HjResult), _DP]),
    "hj_rf_kick": (c_int32, [_CTX, c_double, c_double, c_double, c_double, _DP, _DP, c_int64]),
    "hj_quantum_excitation": (c_int32, [_CTX, c_double, c_double, c_double, _DP, c_uint64,
                                        c_int64, _DP, c_int64]),
    "hj_synchrotron_radiation": (c_int32, [_CTX, c_double, c_double, _DP, c_int64]),
    "hj_phase_advance": (c_int32, [_CTX, c_int32, c_double, c_double, c_double, c_int64,
                                   c_double, c_double, _DP, _DP, c_int64]),
    "hj_histogram": (c_int32, [_CTX, _DP, c_int64, POINTER(HjGrid), _IP]),
    "hj_wake_potential": (c_int32, [_CTX, _IP, POINTER(HjGrid), POINTER(HjWake), c_double,
                                    _DP]),
    "hj_wake_potential_noalloc": (c_int32, [_CTX, c_void_p, POINTER(HjGrid), POINTER(HjWake),
                                            c_double, c_void_p, c_void_p]),
    "hj_apply_wakefield": (c_int32, [_CTX, _DP, _DP, c_int64, POINTER(HjWake), c_double,
                                     c_double, POINTER(HjGrid)]),
    "hj_gaussian": (c_int32, [_CTX, c_uint64, c_int64, c_int64, _DP]),
    "hj_normal_tables": (c_int32, [_DP, c_int64]),
    "hj_generate_particles": (c_int32, [_CTX, c_double, c_double, c_double, c_double, c_int64,
                                        c_uint64, c_void_p, c_void_p, c_void_p, _DP, _DP]),
    "hj_correlation": (c_int32, [_CTX, c_void_p, c_void_p, c_int64, c_void_p, _DP]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load the shared library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH.name} is missing: build it with `python -m haissinskijulia_b200.build` "
            "(the tracking path has no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def status_string(code: int) -> str:
    return load().hj_status_string(code).decode()
