"""Generate the oracle ensemble of the damping-to-equilibrium comparison
(tests/test_gpu_damping_ensemble.py).

The at-scale configuration tracks the benchmark ring (E0 = 4 GeV, radius
113.28 m so that the longitudinal damping time is 5000 turns, the resonator
wake, every physics switch on) for 10,000 turns and logs the moments and the
line density every 100 turns.  Here the oracle runs that configuration with
its OWN random numbers (or_gaussian: a splitmix64 counter hash and Box-Muller,
independent of the GPU's Philox stream) for 20 seeds of 1e5 particles on 4096
bins (the particle count and bins are reduced so that the oracle finishes;
the ring, wake and turns are the configuration's).  Seed s starts from the
numpy default_rng(1000 + s) Gaussian bunch of σ_z = 4 mm, σ_E = 4 MeV, which
the GPU test regenerates.

Per seed and logged turn the fixture holds: turn, E0 - 4e9, σ_z, σ_E, mean z,
mean ΔE, and the line density in 16 coarse bins (each 256 of the 4096 bins)
as fractions of the particles.

Run from the repository root:  python tests/golden/make_ensemble.py
(about 15 minutes on 8 cores).
"""
from __future__ import annotations

import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

OUT = Path(__file__).resolve().parent / "ensemble_damping_b4096.npz"
SEEDS = 20
N = 100_000
NBINS = 4096
TURNS = 10_000
EVERY = 100
COARSE = 16


def initial_bunch(seed: int, sigma_z: float, sigma_E: float):
    rng = np.random.default_rng(1000 + seed)
    return rng.normal(0.0, sigma_z, N), rng.normal(0.0, sigma_E, N)


def record(turn: int, E0: float, z: np.ndarray, dE: np.ndarray, counts: np.ndarray) -> np.ndarray:
    coarse = counts.reshape(COARSE, -1).sum(axis=1) / z.size
    return np.concatenate([[turn, E0 - 4e9, z.std(ddof=1), dE.std(ddof=1), z.mean(), dE.mean()],
                           coarse])


def main() -> None:
    from haissinskijulia_b200._lib import HjParams, HjWake  # structs only: no GPU library load
    from oracle import Oracle
    sys.path.insert(0, str(ROOT))
    import bench
    params, wake, sigma_z, sigma_E = bench.ring_structs(NBINS)
    assert isinstance(params, HjParams) and isinstance(wake, HjWake)
    orc = Oracle(threads=len(os.sched_getaffinity(0)))
    recs = np.zeros((SEEDS, TURNS // EVERY, 6 + COARSE))
    t0 = time.time()
    for s in range(SEEDS):
        z, dE = initial_bunch(s, sigma_z, sigma_E)
        st = orc.state(z, dE, params, wake, NBINS, None, seed=s)
        for t in range(1, TURNS + 1):
            if st.turn(None) != 0:
                raise RuntimeError(f"oracle turn failed: seed {s}, turn {t}")
            if t % EVERY == 0:
                recs[s, t // EVERY - 1] = record(t, st.E0, st.z, st.dE, st.counts())
        st.close()
        print(f"seed {s}: {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(OUT, records=recs, seeds=SEEDS, n=N, nbins=NBINS, turns=TURNS,
                        every=EVERY, coarse=COARSE)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
