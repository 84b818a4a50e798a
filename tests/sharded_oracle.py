"""The reference's MPI mode restated over oracle step functions (test
infrastructure): one turn of a bunch whose particles are split over ranks.

Each rank applies the per-particle steps to its shard; the exchange steps are
the reference's: σ_z from globally summed single-pass sums
(compute_global_std, src/utils.jl:569-606), the histogram summed over ranks
(MPI.Allreduce, src/wakefield.jl:175-200), every rank forming the same
potential, and the E0 update from the globally summed energy change
(src/evolution.jl:408-434).  `allreduce(np.ndarray) -> np.ndarray` sums
over ranks."""
import math

import numpy as np


def global_std(s, s2, n):
    """compute_global_std from global sums (src/utils.jl:593-605)."""
    if n <= 1:
        return 0.0
    mean = s / n
    var = (s2 / n) - mean * mean
    v = var * n / (n - 1)
    return math.sqrt(v) if v > 0 else (v if v != v else 0.0)


def sharded_turn(orc, allreduce, z, dE, draws, E0, p, wake_c, grid_c, n_global,
                 sigma_E0_initial):
    """One turn of the shard (z, dE updated in place); returns (E0, counts)."""
    gamma0 = E0 / p.mass
    b2 = 1.0 - 1.0 / (gamma0 * gamma0)
    beta0 = math.sqrt(b2 if b2 > 0.0 else 0.0)
    sin_phis = math.sin(p.phi_s)
    k = orc.rf_factor(p.freq_rf, beta0)
    dE_init = dE.copy()
    orc.rf_kick(p.voltage, sin_phis, k, p.phi_s, z, dE)                  # src/evolution.jl:313
    if p.use_excitation:
        orc.quantum_excitation(E0, p.radius, sigma_E0_initial, draws, dE)  # :318-320
    if p.SR_damping:
        orc.synchrotron_radiation(E0, p.radius, dE)                          # :323-325
    orc.drift(p.update_eta, E0, p.mass, p.alpha_c, p.harmonic, p.phi_s, p.freq_rf, dE, z)
    s = allreduce(np.array([z.sum(), (z * z).sum()]))
    sz = global_std(s[0], s[1], n_global)                                    # :357
    cur = orc.wake_current(n_global, E0, p.mass, p.alpha_c, p.radius, sz, sigma_E0_initial,
                           wake_c.population)
    counts = allreduce(orc.histogram(z, grid_c))                             # Allreduce
    pot = orc.wake_potential(counts, grid_c, wake_c, cur)
    orc.interp_kick(z, dE, grid_c, pot)
    if p.update_E0:
        total = allreduce(np.array([(dE - dE_init).sum()]))[0]               # :408-426
        mean = total / n_global
        E0 = E0 + mean
        dE -= mean
    return E0, counts
