"""Closed-form anchors of the tracking path, derived from the reference's
formulas by hand rather than by running either implementation.  Both the
oracle and the GPU library must meet them, so a misreading of the reference
shared by the two restatements would show up here.

* Small-amplitude synchrotron motion.  With the wake, quantum excitation,
  radiation damping and the E0 update off, one turn of src/evolution.jl
  (RF kick src/rf_kick.jl:84-87, then the drift :331-344) linearised about
  z = 0 is the map
      ΔE' = ΔE + a z,   z' = z - b ΔE',
  a = -V k cos ϕs, b = 2π h η0 / (β0² E0 k).  Its trace is 2 - a b, and any
  orbit obeys x_{t+1} + x_{t-1} = (2 - a b) x_t, so cos 2πQs = 1 - a b / 2.
* The radiation equilibrium.  Adding quantum excitation and damping
  (src/quantum_excitation.jl:58-71, src/synchrotron_radiation.jl:44-56) in
  the reference's order RF, QE, SR, drift gives x' = M x + N r with one
  standard normal r per particle and turn; the stationary covariance solves
  the discrete Lyapunov equation Σ = M Σ Mᵀ + N Nᵀ.
* The wake potential of a single occupied bin.  The MPI branch of
  apply_wakefield_inplace! (src/wakefield.jl:186-327) forms
  pot[i] = I Σ_{j<=i} W[j] g[i-j] (0-based) with W[m] the wake function at
  bin centre m (src/wakefield.jl:115-118) and g = delta(c, 0.15) cnt / Σcnt
  (src/utils.jl:58-66, src/wakefield.jl:207-221), so counts in bin j0 alone
  give pot[i] = I W[i - j0] delta(c_j0, 0.15) for i >= j0 and 0 below.
"""
import math

import numpy as np
from scipy.linalg import solve_discrete_lyapunov

SPEED_LIGHT = 299792458.0   # src/constants.jl:5


def turn_scalars(p):
    """k, β0, η0 and the damping decrement u of the reference energy
    (src/evolution.jl:300-304, src/synchrotron_radiation.jl:44)."""
    gamma = p.E0 / p.mass
    beta = math.sqrt(1.0 - 1.0 / gamma ** 2)
    eta = p.alpha_c - 1.0 / gamma ** 2
    k = 2.0 * math.pi * p.freq_rf / (beta * SPEED_LIGHT)
    u = 4 * 8.85e-5 * (p.E0 / 1e9) ** 3 / p.radius
    return k, beta, eta, u


def linear_map_ab(p):
    k, beta, eta, _ = turn_scalars(p)
    a = -p.voltage * k * math.cos(p.phi_s)
    b = 2.0 * math.pi * p.harmonic * eta / (beta ** 2 * p.E0 * k)
    return a, b


def synchrotron_trace(p) -> float:
    """2 cos 2πQs of the linearised turn."""
    a, b = linear_map_ab(p)
    return 2.0 - a * b


def trace_from_orbit(x) -> float:
    """Least-squares (2 - a b) from an orbit x_0..x_T of the linear map."""
    x = np.asarray(x, dtype=np.float64)
    mid = x[1:-1]
    return float(np.dot(mid, x[2:] + x[:-2]) / np.dot(mid, mid))


def equilibrium_covariance(p, sigma_E0: float) -> np.ndarray:
    """Stationary covariance of (z, ΔE) under RF, QE, SR and the drift,
    linearised about z = 0."""
    a, b = linear_map_ab(p)
    _, _, _, u = turn_scalars(p)
    d = 1.0 - u
    A = math.sqrt(1.0 - d * d) * sigma_E0          # src/quantum_excitation.jl:59-60
    M = np.array([[1.0 - b * d * a, -b * d], [d * a, d]])
    N = np.array([[-b * d * A], [d * A]])
    # solved in units of the natural spreads (z in units of sqrt(b/a) σ_E0,
    # ΔE in units of σ_E0), where the system is well conditioned
    D = np.diag([1.0 / (math.sqrt(b / a) * sigma_E0), 1.0 / sigma_E0])
    Di = np.linalg.inv(D)
    S = solve_discrete_lyapunov(D @ M @ Di, (D @ N) @ (D @ N).T)
    return Di @ S @ Di


def wake_function(c, wake) -> np.ndarray:
    c = np.asarray(c, dtype=np.float64)
    osc = np.cos(wake.wake_sqrt * c) + wake.sin_coef * np.sin(wake.wake_sqrt * c)
    return np.where(c > 0.0, 0.0, wake.wake_factor * np.exp(c / wake.ctau) * osc)


def single_bin_potential(centers, j0: int, wake, current: float) -> np.ndarray:
    centers = np.asarray(centers, dtype=np.float64)
    W = wake_function(centers, wake)
    sd = wake.delta_std
    g0 = 1.0 / (math.sqrt(2.0 * math.pi) * sd) * math.exp(centers[j0] ** 2 * (-0.5 / sd ** 2))
    pot = np.zeros(centers.size)
    pot[j0:] = current * W[: centers.size - j0] * g0
    return pot
