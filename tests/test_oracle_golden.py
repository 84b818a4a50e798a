"""Pin the C oracle against the independent restatements in tests/golden/.

CPU only.  The histogram must agree bit for bit; floating-point steps within
the per-particle tolerance the GPU parity tests use (1e-12 relative, with a
floor of 1e-12 x the coordinate's spread for values near zero).
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from haissinskijulia_b200._lib import HjGrid, HjParams, HjWake

GOLD = Path(__file__).resolve().parent / "golden"
RTOL = 1e-12


def _close(a, b, scale, rtol=RTOL):
    a, b = np.asarray(a), np.asarray(b)
    tol = rtol * np.maximum(np.abs(b), scale)
    bad = np.abs(a - b) > tol
    assert not bad.any(), f"{bad.sum()} mismatches, worst {np.max(np.abs(a - b) / np.maximum(np.abs(b), scale)):.3e}"


def _params(d, n_turns=1):
    p = HjParams()
    p.E0, p.mass, p.voltage = float(d["p_E0"]), float(d["p_mass"]), float(d["p_voltage"])
    p.harmonic, p.radius = int(d["p_harmonic"]), float(d["p_radius"])
    p.pipe_radius, p.alpha_c = float(d["p_pipe_radius"]), float(d["p_alpha_c"])
    p.phi_s, p.freq_rf, p.n_turns = float(d["p_phi_s"]), float(d["p_freq_rf"]), n_turns
    p.use_wakefield = p.update_eta = p.update_E0 = p.SR_damping = p.use_excitation = 1
    return p


def _wake(d):
    w = HjWake()
    for f in ("wake_factor", "wake_sqrt", "ctau", "sin_coef", "population", "half_width_sigmas",
              "delta_std"):
        setattr(w, f, float(d[f"w_{f}"]))
    return w


def _grid(d):
    c = np.ascontiguousarray(d["centers"])
    g = HjGrid()
    g.nbins = c.shape[0]
    g.edge_first, g.edge_last, g.edge_step = float(d["edge_first"]), float(d["edge_last"]), float(d["edge_step"])
    g.centers = c.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return g, c


@pytest.fixture(scope="module")
def steps():
    return dict(np.load(GOLD / "steps.npz"))


def test_rf_kick(oracle, steps):
    s = steps
    dE = s["dE"].copy()
    oracle.rf_kick(float(s["p_voltage"]), float(s["sin_phis"]), float(s["k"]), float(s["p_phi_s"]),
                   s["z"].copy(), dE)
    _close(dE, s["rf"], 4e6)


def test_quantum_excitation(oracle, steps):
    s = steps
    dE = s["dE"].copy()
    oracle.quantum_excitation(float(s["E0"]), float(s["p_radius"]), 4e6, s["draws"].copy(), dE)
    _close(dE, s["qe"], 4e6)


def test_synchrotron_radiation(oracle, steps):
    s = steps
    dE = s["dE"].copy()
    oracle.synchrotron_radiation(float(s["E0"]), float(s["p_radius"]), dE)
    _close(dE, s["sr"], 4e6)


def test_drift(oracle, steps):
    s = steps
    z = s["z"].copy()
    oracle.drift(True, float(s["E0"]), float(s["p_mass"]), float(s["p_alpha_c"]),
                 int(s["p_harmonic"]), float(s["p_phi_s"]), float(s["p_freq_rf"]),
                 s["dE"].copy(), z)
    _close(z, s["drift"], 4e-3)


def test_histogram_bit_exact(oracle, steps):
    g, keep = _grid(steps)
    counts = oracle.histogram(steps["zh"].copy(), g)
    assert np.array_equal(counts, steps["counts"])
    # edge cases planted in zh[:6]: e0 and eN are counted, values 1 ulp outside are not
    assert counts.sum() == np.count_nonzero((steps["zh"] >= steps["edge_first"]) &
                                            (steps["zh"] <= steps["edge_last"]))


def test_wake_tables(oracle, steps):
    w = _wake(steps)
    W = np.array([oracle.lib.or_wake_function(float(c), ctypes.byref(w)) for c in steps["centers"]])
    lam = np.array([oracle.lib.or_delta(float(c), 0.15) for c in steps["centers"]])
    _close(W, steps["W"], np.abs(steps["W"]).max())
    _close(lam, steps["lam"], 1.0)


@pytest.mark.parametrize("conv", [0, 1])
def test_wake_potential(oracle, steps, conv):
    g, keep = _grid(steps)
    pot = oracle.wake_potential(steps["counts"], g, _wake(steps), float(steps["current"]), conv)
    scale = np.abs(steps["pot"]).max()
    assert np.max(np.abs(pot - steps["pot"])) <= 1e-13 * scale


def test_interp_kick(oracle, steps):
    g, keep = _grid(steps)
    dE = steps["dE"].copy()
    oracle.interp_kick(steps["zh"].copy(), dE, g, steps["pot"].copy())
    _close(dE, steps["kick"], 4e6)


def test_whole_turns_vs_numpy_restatement(oracle):
    d = dict(np.load(GOLD / "turns.npz"))
    T = int(d["n_turns"])
    z, dE = d["z0"].copy(), d["dE0"].copy()
    st = oracle.state(z, dE, _params(d, T), _wake(d), int(d["nbins"]))
    e0, eN, step = st.grid_edges()
    assert (e0, eN, step) == (float(d["edge_first"]), float(d["edge_last"]), float(d["edge_step"]))
    assert np.array_equal(st.centers(), d["centers"])
    for t in range(T):
        assert st.turn(np.ascontiguousarray(d["draws"][t])) == 0
        assert np.array_equal(st.counts(), d["counts"][t]), f"turn {t + 1} counts differ"
    _close(z, d["z"], 4e-3)
    _close(dE, d["dE"], 4e6)
    assert abs(st.E0 - float(d["E0"])) <= 1e-12 * float(d["E0"])
    r = st.result()
    assert r.sigma_E0_initial == pytest.approx(float(d["sigma_E0"]), rel=1e-14)
    assert r.sigma_z0_initial == pytest.approx(float(d["sigma_z0"]), rel=1e-14)


def test_std_helpers(oracle):
    x = np.random.default_rng(3).normal(1.0, 2.0, 1001)
    assert oracle.global_std(x) == pytest.approx(np.std(x, ddof=1), rel=1e-12)
    assert oracle.global_std(x[:1]) == 0.0
    assert oracle.lib.or_next_power_of_two(1000) == 1024
    assert oracle.lib.or_next_power_of_two(1024) == 1024
    assert oracle.lib.or_next_power_of_two(0) == 1


def test_wake_current_particle_factor(oracle):
    # src/evolution.jl:377-386: pf = 1e11/10^floor(log10 N) * N
    E0, mass, a, R, sz, sE = 4e9, 0.51099895069e6, 3e-4, 113.28, 4e-3, 4e6
    g0 = E0 / mass
    eta0 = a - 1.0 / (g0 * g0)
    for n, pf in [(1, 1e11), (9, 9e11), (10, 1e11), (100_000, 1e11), (123_456, 1.23456e11),
                  (10**8, 1e11)]:
        want = pf / E0 / (6.283185307179586 * R) * sz / (eta0 * sE * sE)
        got = oracle.lib.or_wake_current(n, E0, mass, a, R, sz, sE, 0.0)
        assert got == pytest.approx(want, rel=1e-15)
