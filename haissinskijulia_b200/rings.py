"""Ring configurations used by the benchmark and the tests.

benchmark_ring(): the 4 GeV ring of the tracking benchmark (E0 = 4 GeV,
C = 215.9 m, h = 360 at 500 MHz, V = 5 MV, α_c = 3e-4, U0 = 0.5 MeV/turn,
5000-turn longitudinal damping, σ_E/E = 1e-3, σ_z = 4 mm, broadband
resonator Rs = 10 kΩ, Q = 1, f_r = 20 GHz, 1e10 electrons, bins over ±6σ_z).
The reference API has no circumference or damping-time fields, so they are
expressed through its own parameters:
  * ϕs = π - asin(U0/V) for the ring's voltage V: the reference's
    above-transition convention
    (its benchmark uses ϕs = 5π/6, tests/benchmark_total.jl:152);
  * radius = 4·8.85e-5·(E0/1e9)^3 / 2e-4 = 113.28 m, so that the per-turn
    damping ∂U/∂E of src/synchrotron_radiation.jl:44 is 1/5000;
  * σ_E0_initial = 1e-3·E0, which makes the quantum-excitation equilibrium
    of src/quantum_excitation.jl:59 equal to σ_E/E = 1e-3.

reference_ring(): the reference's own benchmark ring
(tests/benchmark_total.jl:140-166), with its hard-coded wake.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

from .api import MASS_ELECTRON, SPEED_LIGHT, SimulationParameters, WakeModel, next_power_of_two


@dataclass
class RingConfig:
    params: SimulationParameters
    wake: WakeModel
    sigma_z: float      # initial rms bunch length [m]
    sigma_E: float      # initial rms energy spread [eV]
    nbins: int


def benchmark_ring(n_turns: int = 100, nbins: int = 4096, population: float = 1e10,
                   voltage: float = 5e6, half_width_sigmas: float = 6.0,
                   use_wakefield: bool = True, use_excitation: bool = True) -> RingConfig:
    E0 = 4e9
    U0 = 0.5e6
    damping_turns = 5000.0
    radius = 4 * 8.85e-5 * (E0 / 1e9) ** 3 * damping_turns
    params = SimulationParameters(
        E0=E0, mass=MASS_ELECTRON, voltage=voltage, harmonic=360, radius=radius,
        pipe_radius=2.5e-4, alpha_c=3e-4, phi_s=math.pi - math.asin(U0 / voltage),
        freq_rf=500e6, n_turns=n_turns, use_wakefield=use_wakefield, update_eta=True,
        update_E0=True, SR_damping=True, use_excitation=use_excitation)
    wake = WakeModel.resonator(Rs=1e4, Q=1.0, fr=20e9, population=population,
                               half_width_sigmas=half_width_sigmas)
    return RingConfig(params, wake, sigma_z=4e-3, sigma_E=1e-3 * E0, nbins=nbins)


def reference_ring(n_particles: int = 100_000, n_turns: int = 100) -> RingConfig:
    E0 = 4e9
    mass = MASS_ELECTRON
    voltage = 5e6
    harmonic = 360
    radius = 250.0
    alpha_c = 3.68e-4
    gamma = E0 / mass
    beta = math.sqrt(1 - 1 / gamma ** 2)
    phi_s = 5 * math.pi / 6
    freq_rf = (phi_s + 10 * math.pi / 180) * beta * SPEED_LIGHT / (2 * math.pi)
    T_rev = (2 * math.pi * radius) / (beta * SPEED_LIGHT)
    w_rev = 2 * math.pi / T_rev
    sigma_E0 = 1e6
    factor = alpha_c * E0 / (harmonic * voltage * abs(math.cos(phi_s)))
    sigma_z0 = math.sqrt(2 * math.pi) * SPEED_LIGHT / w_rev * math.sqrt(factor) * sigma_E0 / E0
    params = SimulationParameters(
        E0=E0, mass=mass, voltage=voltage, harmonic=harmonic, radius=radius,
        pipe_radius=0.00025, alpha_c=alpha_c, phi_s=phi_s, freq_rf=freq_rf, n_turns=n_turns,
        use_wakefield=True, update_eta=True, update_E0=True, SR_damping=True,
        use_excitation=True)
    nbins = next_power_of_two(max(64, round(n_particles / 100)))   # tests/benchmark_total.jl:255
    return RingConfig(params, WakeModel.reference(params), sigma_z=sigma_z0, sigma_E=sigma_E0,
                      nbins=nbins)
