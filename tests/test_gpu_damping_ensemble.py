"""Damping to equilibrium on the benchmark ring (the at-scale configuration's
physics: radius 113.28 m, 5000-turn damping, the resonator wake, every switch
on, 10,000 turns, moments and line density logged every 100 turns) with
on-device Philox excitation, against the oracle's own-RNG ensemble in
tests/golden/ensemble_damping_b4096.npz (tests/golden/make_ensemble.py):
20 seeds of 1e5 particles on 4096 bins, each seed starting from the same
numpy Gaussian bunch on both sides.

For every logged turn and each quantity -- E0, σ_z, σ_E, centroid, mean ΔE
and the line density in 16 coarse bins -- the ensemble means differ by
z = (m_gpu - m_oracle) / sqrt(se_gpu² + se_oracle²) standard errors.  After
damping (the per-seed average over turns 8100-10000) every |z| <= 3; over all
100 logged turns at least 98 % of the |z| are <= 3 (99.7 % is the
expectation) and none exceeds 4.5 (the records of a run are correlated, so
single 3σ excursions are expected among ~2000 comparisons)."""
import math
from pathlib import Path

import numpy as np
import pytest

from haissinskijulia_b200 import ResidentBunch, benchmark_ring

from gpu_util import device_pair

pytestmark = pytest.mark.gpu

FIXTURE = Path(__file__).resolve().parent / "golden" / "ensemble_damping_b4096.npz"
NAMES = ["E0", "sigma_z", "sigma_E", "mean_z", "mean_dE"] + [f"density[{k}]" for k in range(16)]


def _gpu_records(ctx, seeds, n, nbins, turns, every, coarse):
    cfg = benchmark_ring(n_turns=turns, nbins=nbins)
    out = np.zeros((seeds, turns // every, 6 + coarse))
    for s in range(seeds):
        rng = np.random.default_rng(1000 + s)
        z0, e0 = rng.normal(0.0, cfg.sigma_z, n), rng.normal(0.0, cfg.sigma_E, n)
        dz, de = device_pair(z0, e0)
        b = ResidentBunch(ctx, dz.data_ptr(), de.data_ptr(), n, cfg.params, nbins,
                          wake=cfg.wake, seed=s)
        b.set_log(every, capacity=turns // every, density=True)
        b.advance(turns)
        log = b.read_log()
        b.finish()
        b.close()
        assert log.shape[0] == turns // every
        dens = log[:, 8:].reshape(log.shape[0], coarse, -1).sum(axis=2) / n
        out[s] = np.column_stack([log[:, 0], log[:, 1] - 4e9, log[:, 2], log[:, 3], log[:, 4],
                                  log[:, 5], dens])
    return out


def _z(a, b):
    """Standard errors between the ensemble means of a and b (axis 0 = seeds)."""
    k = a.shape[0]
    se = np.sqrt(a.var(axis=0, ddof=1) / k + b.var(axis=0, ddof=1) / k)
    return (a.mean(axis=0) - b.mean(axis=0)) / np.where(se > 0, se, np.inf)


def test_damping_ensemble_matches_the_oracle(gpu_ctx):
    f = np.load(FIXTURE)
    orc = f["records"]
    seeds, n, nbins = int(f["seeds"]), int(f["n"]), int(f["nbins"])
    turns, every, coarse = int(f["turns"]), int(f["every"]), int(f["coarse"])
    gpu = _gpu_records(gpu_ctx, seeds, n, nbins, turns, every, coarse)
    assert np.array_equal(gpu[0, :, 0], orc[0, :, 0])       # the same logged turns
    # the bunch damps: σ_z from 4 mm towards the 2.2 mm equilibrium
    assert gpu[:, 0, 2].mean() > 3.8e-3 and gpu[:, -1, 2].mean() < 3.0e-3
    q = slice(1, None)
    late = gpu[0, :, 0] > 0.8 * turns
    z_late = _z(gpu[:, late, q].mean(axis=1), orc[:, late, q].mean(axis=1))
    worst = int(np.argmax(np.abs(z_late)))
    assert np.all(np.abs(z_late) <= 3.0), (
        f"after damping: {NAMES[worst]} differs by {z_late[worst]:.2f} standard errors")
    z_all = _z(gpu[:, :, q], orc[:, :, q])
    frac = float(np.mean(np.abs(z_all) <= 3.0))
    assert frac >= 0.98, f"only {frac:.3f} of the logged comparisons within 3 SE"
    k, j = np.unravel_index(int(np.argmax(np.abs(z_all))), z_all.shape)
    assert abs(z_all[k, j]) <= 4.5, (
        f"turn {int(gpu[0, k, 0])}: {NAMES[j]} differs by {z_all[k, j]:.2f} standard errors")
    print(f"damping ensemble: worst |z| after damping {abs(z_late[worst]):.2f} ({NAMES[worst]}); "
          f"over all records {abs(z_all[k, j]):.2f} ({NAMES[j]}, turn {int(gpu[0, k, 0])}); "
          f"{100 * frac:.1f} % within 3 SE")
