"""Batches at the configurations the sweep, scan and serving measurements run:
8192 and 4096 bins, 262144- and 65536-particle chunks, the 32-bit-counter
layouts 8 and 9 the autotuner picks, and the 4-CTA batched bins step (a
batch whose largest grid has 1024 bins or more).

Each bunch of a batch is checked against the oracle fed the very Philox
normals the GPU draws (gaussian_draws of the bunch's seed, turn by turn):
every particle within 1e-12 relative after the last turn, E0 and the spreads
within 1e-12, and the batch's bin counts of the last turn equal to the
oracle's histogram of the same positions bit for bit (src/utils.jl:384-398).
The bunches are ragged: several chunks with a short last one, an odd count
(a scalar tail), and a bunch smaller than one chunk."""
import numpy as np
import pytest

from haissinskijulia_b200 import Batch, BinGrid, benchmark_ring, gaussian_draws

from gpu_util import assert_close

pytestmark = pytest.mark.gpu

TURNS = 12

# (max bins, particles per chunk, pass layout, bunches: (n, bins, voltage, population))
CASES = {
    "intensity_scan_8192_chunk256k_layout9": (
        8192, 262144, 9,
        [(600_000, 8192, 5e6, 1e9), (300_001, 8192, 5e6, 1e11), (70_000, 8192, 5e6, 1e10)]),
    "sweep_4096_chunk64k_layout8": (
        4096, 65536, 8,
        [(250_000, 4096, 3e6, 1e9), (131_075, 4096, 7e6, 1e11), (10_003, 4096, 4.2e6, 3e10)]),
    "serving_mixed_bins_chunk64k_auto": (
        8192, 65536, -1,
        [(200_000, 2048, 6e6, 2e10), (150_001, 4096, 3.5e6, 5e9), (90_000, 8192, 5.5e6, 7e10)]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_batch_configuration_matches_the_oracle(gpu_ctx, gpu_buffers, oracle, name):
    max_bins, chunk, layout, bunches = CASES[name]
    pool = sum(n for n, *_ in bunches) + 4096
    bt = Batch(gpu_ctx, pool_particles=pool, max_bunches=4, max_nbins=max_bins, chunk=chunk,
               layout=layout, graph_turns=4)
    specs = {}
    for i, (n, nbins, volt, pop) in enumerate(bunches):
        cfg = benchmark_ring(n_turns=TURNS, nbins=nbins, population=pop, voltage=volt)
        rng = np.random.default_rng(500 + i)
        z0, e0 = rng.normal(0.0, cfg.sigma_z, n), rng.normal(0.0, cfg.sigma_E, n)
        seed = 7000 + i
        bid = bt.add(z0, e0, cfg.params, nbins, wake=cfg.wake, seed=seed, turns=TURNS)
        specs[bid] = (cfg, z0, e0, nbins, seed)
    bt.advance(TURNS)
    assert sorted(bt.poll()) == sorted(specs)
    got = {}
    for bid in specs:
        counts = bt.histogram(bid, specs[bid][3])
        z, e, r = bt.take(bid)
        got[bid] = (counts, z, e, r)
    bt.close()

    for bid, (cfg, z0, e0, nbins, seed) in specs.items():
        counts, z, e, r = got[bid]
        n = z0.size
        # the grid the library built from its initial spread of z
        grid = BinGrid.make(r.sigma_z0_initial, nbins, cfg.wake.half_width_sigmas)
        assert r.sigma_z0_initial == pytest.approx(oracle.global_std(z0), rel=1e-14)
        zo, eo = z0.copy(), e0.copy()
        st = oracle.state(zo, eo, cfg.params.to_c(), cfg.wake.to_c(), nbins, grid.to_c())
        for t in range(1, TURNS + 1):
            assert st.turn(gaussian_draws(seed, t, n, gpu_buffers)) == 0
        ro = st.result()
        what = f"{name} bunch of {n}"
        assert_close(z, zo, cfg.sigma_z, what=f"z, {what}")
        assert_close(e, eo, cfg.sigma_E, what=f"dE, {what}")
        assert r.E0 == pytest.approx(ro.E0, rel=1e-12)
        assert r.sigma_E == pytest.approx(ro.sigma_E, rel=1e-12)
        assert r.sigma_z == pytest.approx(ro.sigma_z, rel=1e-12)
        assert r.turns == TURNS
        want = oracle.histogram(z, grid.to_c())
        assert counts.sum() > 0.99 * n
        assert np.array_equal(counts, want), f"bin counts differ, {what}"
        st.close()
