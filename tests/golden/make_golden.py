"""Generate the golden vectors that pin the C oracle (tests/test_oracle_golden.py).

The reference ships no golden vectors for this path and Julia is not
installed here, so the oracle is pinned against two INDEPENDENT restatements
of the reference formulas written in this file:

* steps.npz -- per-step outputs evaluated in 50-digit mpmath from the same
  float64 inputs and float64 per-turn constants (RF kick src/rf_kick.jl:84-87,
  quantum excitation src/quantum_excitation.jl:58-71, SR damping
  src/synchrotron_radiation.jl:44-56, drift src/evolution.jl:331-344, wake
  table src/wakefield.jl:115-118, smoothing weight src/utils.jl:58-66,
  convolution src/wakefield.jl:186-319 as a direct causal sum, interpolation
  src/wakefield.jl:22-105), plus the histogram emulated in numpy float64 with
  the reference's operation order (src/utils.jl:384-398), which must match
  bit for bit.
* turns.npz -- whole turns (src/evolution.jl:295-456, MPI branch) by a
  numpy float64 restatement that uses numpy.fft (pocketfft) for the P-point
  complex FFTs, as the reference uses FFTW.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import mpmath as mp  # noqa: E402

mp.mp.dps = 50
OUT = Path(__file__).resolve().parent

SPEED_LIGHT = 299792458.0
MASS_ELECTRON = 0.51099895069e6
TWO_PI = 6.283185307179586


def ring():
    """Benchmark ring constants (haissinskijulia_b200/rings.py), float64."""
    E0 = 4e9
    radius = 4 * 8.85e-5 * (E0 / 1e9) ** 3 * 5000.0
    p = dict(E0=E0, mass=MASS_ELECTRON, voltage=5e6, harmonic=360, radius=radius,
             pipe_radius=2.5e-4, alpha_c=3e-4, phi_s=math.pi - math.asin(0.5e6 / 5e6),
             freq_rf=500e6)
    wr = TWO_PI * 20e9
    alpha = wr / 2.0
    wbar = math.sqrt(wr * wr - alpha * alpha)
    w = dict(wake_factor=2.0 * alpha * 1e4, wake_sqrt=wbar / SPEED_LIGHT,
             ctau=SPEED_LIGHT / alpha, sin_coef=alpha / wbar, population=1e10,
             half_width_sigmas=6.0, delta_std=0.15)
    return p, w


def turn_scalars(E0, p):
    """src/evolution.jl:300-304 in float64 (the per-turn constants are inputs
    of the per-particle formulas below)."""
    g0 = E0 / p["mass"]
    b2 = 1.0 - 1.0 / (g0 * g0)
    beta0 = math.sqrt(max(b2, 0.0))
    eta0 = p["alpha_c"] - (1.0 / (g0 * g0))
    k = p["freq_rf"] * TWO_PI / (beta0 * SPEED_LIGHT)
    t = E0 / 1e9
    dU = 4 * 8.85e-5 * (t * t * t) / p["radius"]
    return dict(gamma0=g0, beta0=beta0, eta0=eta0, sin_phis=math.sin(p["phi_s"]), k=k, dU=dU)


def exact_grid(sigma_z0, half, B):
    """Correctly rounded edges/centers of range(-w, w, length=B+1)."""
    from fractions import Fraction
    w = half * sigma_z0
    if w < 1e-9:
        w = 1e-6
    W = Fraction(w)
    centers = np.array([float(W * (2 * k + 1 - B) / B) for k in range(B)])
    return dict(edge_first=-w, edge_last=w, edge_step=float(W * 2 / B), centers=centers)


def hist_numpy(z, g):
    """src/utils.jl:384-398 with float64 operations in the reference's order."""
    B = len(g["centers"])
    e0, eN = g["edge_first"], g["edge_last"]
    inv = 1.0 / g["edge_step"]
    counts = np.zeros(B, dtype=np.int64)
    for x in z:
        inr = (x >= e0) and (x <= eN)
        u = math.floor((x - e0) * inv)
        j = min(max(u + 1, 1), B)
        counts[j - 1] += int(inr)
    return counts


def mp_wake(c, w):
    c = mp.mpf(c)
    if c > 0:
        return mp.mpf(0)
    osc = mp.cos(mp.mpf(w["wake_sqrt"]) * c) + mp.mpf(w["sin_coef"]) * mp.sin(mp.mpf(w["wake_sqrt"]) * c)
    return mp.mpf(w["wake_factor"]) * mp.exp(c / mp.mpf(w["ctau"])) * osc


def mp_delta(x, s):
    x, s = mp.mpf(x), mp.mpf(s)
    return 1 / (mp.sqrt(2 * mp.pi) * s) * mp.exp(-x * x / (2 * s * s))


def make_steps():
    rng = np.random.Generator(np.random.Philox(20240601))
    p, w = ring()
    N = 2000
    z = rng.normal(0.0, 4e-3, N)
    dE = rng.normal(0.0, 4e6, N)
    draws = rng.normal(0.0, 1.0, N)
    E0 = p["E0"]
    s = turn_scalars(E0, p)
    V, phis, k = p["voltage"], p["phi_s"], s["k"]
    # RF kick
    rf = np.array([float(mp.mpf(e) + mp.mpf(V) * (mp.sin(-mp.mpf(zz) * mp.mpf(k) + mp.mpf(phis))
                                                  - mp.mpf(s["sin_phis"]))) for zz, e in zip(z, dE)])
    # quantum excitation and SR damping (constants from float64 E0 and radius)
    t = mp.mpf(E0) / mp.mpf(1e9)
    dU = mp.mpf(4) * mp.mpf(8.85e-5) * t ** 3 / mp.mpf(p["radius"])
    A = mp.sqrt(1 - (1 - dU) ** 2) * mp.mpf(4e6)
    qe = np.array([float(mp.mpf(e) + A * mp.mpf(r)) for e, r in zip(dE, draws)])
    sr = np.array([float(mp.mpf(e) * (1 - dU)) for e in dE])
    # drift with energy-dependent slip factor, exact arithmetic from float64 constants
    g0, b0, kk = mp.mpf(s["gamma0"]), mp.mpf(s["beta0"]), mp.mpf(k)
    drift = []
    for zz, e in zip(z, dE):
        e = mp.mpf(e)
        gp = g0 + e / mp.mpf(p["mass"])
        eta = mp.mpf(p["alpha_c"]) - 1 / (gp * gp)
        coeff = mp.mpf(TWO_PI) * p["harmonic"] * eta / (b0 * b0 * mp.mpf(E0))
        ph = -(mp.mpf(zz) * kk - mp.mpf(phis)) + coeff * e
        drift.append(float((-ph + mp.mpf(phis)) / kk))
    drift = np.array(drift)
    # grid, histogram, wake tables, convolution, interpolation
    B = 64
    g = exact_grid(4e-3, w["half_width_sigmas"], B)
    # include edge cases: exact edges, just outside, first/last centers
    zh = z.copy()
    zh[:6] = [g["edge_first"], g["edge_last"], np.nextafter(g["edge_first"], -1.0),
              np.nextafter(g["edge_last"], 1.0), g["centers"][0], g["centers"][-1]]
    counts = hist_numpy(zh, g)
    Wt = [mp_wake(c, w) for c in g["centers"]]
    lam = [mp_delta(c, w["delta_std"]) for c in g["centers"]]
    ntot = int(counts.sum())
    gl = [lam[i] * mp.mpf(int(counts[i])) / ntot for i in range(B)]
    current = 2.9e-15
    pot = np.array([float(mp.mpf(current) * mp.fsum(Wt[j] * gl[i - j] for j in range(i + 1)))
                    for i in range(B)])
    c1, cB = mp.mpf(g["centers"][0]), mp.mpf(g["centers"][-1])
    inv_c = 1 / ((cB - c1) / (B - 1))
    kick = []
    for zz, e in zip(zh, dE):
        x = mp.mpf(zz)
        x = cB if x > cB else (c1 if x < c1 else x)
        u = (x - c1) * inv_c
        fl = mp.floor(u)
        idx = int(min(max(fl, 0), B - 2))
        wgt = u - fl
        kick.append(float(mp.mpf(e) - (mp.mpf(pot[idx]) * (1 - wgt) + mp.mpf(pot[idx + 1]) * wgt)))
    np.savez_compressed(
        OUT / "steps.npz", z=z, dE=dE, draws=draws, zh=zh, E0=E0, k=k, sin_phis=s["sin_phis"],
        rf=rf, qe=qe, sr=sr, drift=drift, counts=counts, pot=pot, kick=kick, current=current,
        W=np.array([float(x) for x in Wt]), lam=np.array([float(x) for x in lam]),
        edge_first=g["edge_first"], edge_last=g["edge_last"], edge_step=g["edge_step"],
        centers=g["centers"], **{f"p_{a}": b for a, b in p.items()},
        **{f"w_{a}": b for a, b in w.items()})


def global_std(x):
    """src/utils.jl:569-606 (single pass)."""
    n = len(x)
    s = 0.0
    s2 = 0.0
    for v in x:
        s += v
        s2 += v * v
    if n <= 1:
        return 0.0
    mean = s / n
    var = (s2 / n) - mean * mean
    return math.sqrt(max(0.0, var * n / (n - 1)))


def numpy_turns(z, dE, draws, p, w, B, n_turns):
    """Whole turns, MPI branch, numpy float64 + pocketfft (numpy.fft)."""
    z = z.copy()
    dE = dE.copy()
    n = len(z)
    E0 = p["E0"]
    sE0 = global_std(dE)
    sz0 = global_std(z)
    g = exact_grid(sz0, w["half_width_sigmas"], B)
    c = g["centers"]
    inv_ctau = 1.0 / w["ctau"]
    Wt = np.array([0.0 if x > 0 else w["wake_factor"] * math.exp(x * inv_ctau) *
                   (math.cos(w["wake_sqrt"] * x) + w["sin_coef"] * math.sin(w["wake_sqrt"] * x))
                   for x in c])
    lam = np.array([1.0 / (math.sqrt(TWO_PI) * w["delta_std"]) *
                    math.exp(x * x * (-0.5 / (w["delta_std"] ** 2))) for x in c])
    P = 1
    while P < 2 * B:
        P <<= 1
    hist = []
    for t in range(n_turns):
        s = turn_scalars(E0, p)
        dE_init = dE.copy()
        phi = -z * s["k"] + p["phi_s"]
        dE = dE + p["voltage"] * (np.sin(phi) - s["sin_phis"])
        A = math.sqrt(1 - (1 - s["dU"]) * (1 - s["dU"])) * sE0
        dE = dE + A * draws[t]
        dE = dE * (1 - s["dU"])
        gp = s["gamma0"] + dE / p["mass"]
        eta = p["alpha_c"] - 1.0 / (gp * gp)
        coeff = TWO_PI * p["harmonic"] * eta / (s["beta0"] * s["beta0"] * E0)
        ph = -(z * s["k"] - p["phi_s"])
        ph = ph + coeff * dE
        z = (-ph + p["phi_s"]) / s["k"]
        sz = global_std(z)
        g0 = E0 / p["mass"]
        eta0 = p["alpha_c"] - 1.0 / (g0 * g0)
        cur = w["population"] / E0 / (TWO_PI * p["radius"]) * sz / (eta0 * sE0 * sE0)
        counts = hist_numpy(z, g)
        ntot = counts.sum()
        fW = np.zeros(P, complex)
        fL = np.zeros(P, complex)
        fW[:B] = Wt
        fL[:B] = lam * (counts * (1.0 / ntot))
        pot = np.fft.ifft(np.fft.fft(fW) * np.fft.fft(fL) * cur).real[:B]
        c1, cBv = c[0], c[-1]
        inv = 1.0 / ((cBv - c1) / (B - 1))
        u = (np.clip(z, c1, cBv) - c1) * inv
        fl = np.floor(u)
        idx = np.clip(fl.astype(np.int64) + 1, 1, B - 1)
        wg = u - fl
        dE = dE - (pot[idx - 1] * (1.0 - wg) + pot[idx] * wg)
        sdiff = 0.0
        for a, b in zip(dE, dE_init):
            sdiff += a - b
        mean = sdiff / n
        E0 = E0 + mean
        dE = dE - mean
        hist.append(counts)
    return z, dE, E0, sE0, sz0, np.array(hist), g


def make_turns():
    rng = np.random.Generator(np.random.Philox(777))
    p, w = ring()
    N, B, T = 512, 64, 8
    z0 = rng.normal(0.0, 4e-3, N)
    dE0 = rng.normal(0.0, 4e6, N)
    draws = rng.normal(0.0, 1.0, (T, N))
    z, dE, E0, sE0, sz0, hist, g = numpy_turns(z0, dE0, draws, p, w, B, T)
    np.savez_compressed(OUT / "turns.npz", z0=z0, dE0=dE0, draws=draws, z=z, dE=dE, E0=E0,
                        sigma_E0=sE0, sigma_z0=sz0, counts=hist, nbins=B, n_turns=T,
                        centers=g["centers"], edge_first=g["edge_first"],
                        edge_last=g["edge_last"], edge_step=g["edge_step"],
                        **{f"p_{a}": b for a, b in p.items()},
                        **{f"w_{a}": b for a, b in w.items()})


if __name__ == "__main__":
    make_steps()
    make_turns()
    print("wrote", OUT / "steps.npz", OUT / "turns.npz")
