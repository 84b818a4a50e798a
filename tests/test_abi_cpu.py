"""The C-ABI library on a machine without a GPU: it loads, exports every
symbol include/*.h declares, and its host-only helpers behave.  No compute
call is made here."""
import ctypes
import math
import re
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

from haissinskijulia_b200 import _lib
from haissinskijulia_b200 import build as hjbuild
from haissinskijulia_b200.api import BinGrid, SimulationParameters, WakeModel

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def lib():
    hjbuild.build()
    return _lib.load()


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(hj_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"
    # and the ctypes table covers exactly the declared entry points
    assert set(_lib.SIGNATURES) == set(names)


def test_version_and_status(lib):
    assert b"sm_100a" in lib.hj_version()
    assert lib.hj_status_string(_lib.HJ_ERR_NBINS) == b"HJ_ERR_NBINS"


def test_create_without_gpu_reports_no_device(lib):
    from conftest import cuda_available
    if cuda_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert lib.hj_create(0, ctypes.byref(h)) == _lib.HJ_ERR_NO_DEVICE


def test_struct_layouts():
    # POD layouts the Julia/C callers rely on (include/haissinski_gpu.h)
    assert ctypes.sizeof(_lib.HjParams) == 88
    assert ctypes.sizeof(_lib.HjWake) == 56
    assert ctypes.sizeof(_lib.HjGrid) == 40
    assert ctypes.sizeof(_lib.HjResult) == 64


@pytest.mark.parametrize("B", [1, 2, 3, 64, 1000, 4096, 16384])
def test_make_grid_correctly_rounded(lib, B):
    sigma = 0.0040123456789
    g = BinGrid.make(sigma, B, 7.5)
    w = 7.5 * sigma
    W = Fraction(w)
    assert g.edge_first == -w and g.edge_last == w
    assert g.edge_step == float(W * 2 / B)
    idx = np.unique(np.linspace(0, B - 1, min(B, 200)).astype(int))
    for k in idx:
        assert g.centers[k] == float(W * (2 * int(k) + 1 - B) / B)


@pytest.mark.parametrize("B", [7, 2000, 4096, 10000])
def test_make_grid_every_center_correctly_rounded(lib, B):
    rng = np.random.default_rng(B)
    for sigma in (0.0040123456789, *rng.uniform(1e-4, 1e-2, 3)):
        g = BinGrid.make(float(sigma), B, 7.5)
        W = Fraction(7.5 * float(sigma))
        want = [float(W * (2 * k + 1 - B) / B) for k in range(B)]
        assert np.array_equal(g.centers, np.array(want))


def test_make_grid_width_floor_and_errors(lib):
    g = BinGrid.make(0.0, 8, 7.5)          # src/evolution.jl:272
    assert g.edge_last == 1e-6
    c = np.empty(1)
    out = _lib.HjGrid()
    assert lib.hj_make_grid(1e-3, 7.5, 0, c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            ctypes.byref(out)) == _lib.HJ_ERR_NBINS


def test_reference_wake_constants(lib):
    p = SimulationParameters(4e9, 0.51099895069e6, 5e6, 360, 250.0, 2.5e-4, 3.68e-4,
                             5 * math.pi / 6, 1.3e8, 10, True, True, True, True, True)
    w = WakeModel.reference(p)
    # src/evolution.jl:276-280
    assert w.wake_factor == (120 * math.pi) * 299792458.0 / (math.pi * 2.5e-4)
    assert w.wake_sqrt == math.sqrt(2 * 30.0 / 2.5e-4)
    assert w.ctau == 4e-3 and w.sin_coef == 0.0 and w.population == 0.0
    assert w.half_width_sigmas == 7.5 and w.delta_std == 0.15


def test_resonator_mapping(lib):
    w = WakeModel.resonator(1e4, 1.0, 20e9, 1e10, 6.0)
    wr = 2 * math.pi * 20e9
    a = wr / 2
    wb = math.sqrt(wr * wr - a * a)
    assert w.ctau == pytest.approx(299792458.0 / a, rel=1e-15)       # 4.771 mm
    assert w.wake_sqrt == pytest.approx(wb / 299792458.0, rel=1e-15)  # 363.0 1/m
    assert w.wake_factor == pytest.approx(2 * a * 1e4, rel=1e-15)
    assert w.sin_coef == pytest.approx(a / wb, rel=1e-15)
    with pytest.raises(Exception):
        WakeModel.resonator(1e4, 0.25, 20e9, 1e10, 6.0)   # overdamped: no ω̄


def test_oracle_grid_matches_library_grid(oracle):
    for B in (64, 4096):
        rc, g, c = oracle.make_grid(3.3e-3, 6.0, B)
        lg = BinGrid.make(3.3e-3, B, 6.0)
        assert rc == 0
        assert np.array_equal(c, lg.centers)
        assert (g.edge_first, g.edge_last, g.edge_step) == (lg.edge_first, lg.edge_last, lg.edge_step)


def test_buffers_argument_checks():
    from haissinskijulia_b200 import create_simulation_buffers
    with pytest.raises(ValueError, match="nbins"):
        create_simulation_buffers(10, 0)
    with pytest.raises(ValueError, match="non-negative"):
        create_simulation_buffers(-1, 8)
