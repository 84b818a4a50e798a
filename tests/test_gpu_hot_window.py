"""The fused pass's hot window at 16384 bins (the largest grid): per-block bin
and cell counters live in shared memory only for the bins around the last
turn's mean z; a deposit outside goes to the bunch's spill histograms in
global memory, which the merge folds in.  Bunches with a wide uniform halo
put several percent of their particles outside the window every turn; the bin
counts must still equal the oracle's histogram of the same positions bit for
bit at every turn, and every particle must stay within 1e-12 relative of the
oracle fed the very normals the GPU draws (gaussian_draws of the bunch's
seed, turn by turn, for the Float64 normals; host draws otherwise).

Cases: the default layout (32-bit counters) and layout 0 (16-bit counter
pairs) with the Float64 normals, whose ziggurat table shrinks the window; host
draws (no table, a wider window); a bunch off the grid's centre, whose window
is clamped at the grid's edge; layout 13 (4 x 256 threads, two blocks per SM:
half the shared memory, a window of about 4000 cells); a batch member at
16384 bins."""
import numpy as np
import pytest
import torch

from haissinskijulia_b200 import (Batch, BinGrid, Context, ResidentBunch, benchmark_ring,
                                  gaussian_draws)

from gpu_util import assert_close, device_pair

pytestmark = pytest.mark.gpu

NBINS = 16384
TURNS = 5


def halo_bunch(n, sigma_z, sigma_E, shift, seed):
    """A Gaussian core (70 %) and a halo uniform over +-7.5 sigma_z (30 %),
    moved by `shift`, with a few particles beyond the grid."""
    rng = np.random.default_rng(seed)
    m = (3 * n) // 10
    z = rng.normal(0.0, sigma_z, n)
    z[:m] = rng.uniform(-7.5 * sigma_z, 7.5 * sigma_z, m)
    z[m:m + 5] = np.array([-9.0, -8.0, 7.6, 8.0, 12.0]) * sigma_z
    rng.shuffle(z)
    return z + shift, rng.normal(0.0, sigma_E, n)


LAYOUTS = {"float64_layout0": 0, "float64_layout13": 13}


@pytest.mark.parametrize("case", ["float64_default", "float64_layout0", "draws_default",
                                  "float64_off_centre", "float64_layout13"])
def test_spilled_deposits_keep_exact_counts(gpu_buffers, oracle, case):
    layout = LAYOUTS.get(case, -1)
    philox = not case.startswith("draws")
    ctx = Context(0)
    ctx.set_pass_layout(layout)
    cfg = benchmark_ring(n_turns=TURNS, nbins=NBINS)
    n = 200_003
    shift = 3.0 * cfg.sigma_z if case == "float64_off_centre" else 0.0
    z0, e0 = halo_bunch(n, cfg.sigma_z, cfg.sigma_E, shift, seed=len(case))
    grid = BinGrid.make(cfg.sigma_z, NBINS, cfg.wake.half_width_sigmas)
    seed = 900 + len(case)
    dz, de = device_pair(z0, e0)
    b = ResidentBunch(ctx, dz.data_ptr(), de.data_ptr(), n, cfg.params, NBINS, wake=cfg.wake,
                      grid=grid, seed=seed)
    draws = None
    if not philox:
        draws = np.random.default_rng(seed).normal(size=(TURNS, n))
        ddraws = torch.from_numpy(draws).cuda()
        b.set_draws(ddraws.data_ptr(), 1, TURNS)
    zo, eo = z0.copy(), e0.copy()
    st = oracle.state(zo, eo, cfg.params.to_c(), cfg.wake.to_c(), NBINS, grid.to_c())
    zout, eout = torch.empty_like(dz), torch.empty_like(de)
    edges = np.abs(np.asarray(grid.centers) - shift)
    for t in range(1, TURNS + 1):
        b.advance(1)
        r = draws[t - 1] if draws is not None else gaussian_draws(seed, t, n, gpu_buffers)
        assert st.turn(np.ascontiguousarray(r)) == 0
        b.observe(zout.data_ptr(), eout.data_ptr())
        zg, eg = zout.cpu().numpy(), eout.cpu().numpy()
        counts = b.histogram()
        want = oracle.histogram(zg, grid.to_c())
        assert np.array_equal(counts, want), f"{case}: counts turn {t}"
        assert np.array_equal(counts, st.counts()), f"{case}: counts vs oracle bunch, turn {t}"
        # at least 3 % of the binned particles sit more than 36 % of the grid's
        # width from the bunch's centre, beyond any window the pass holds at
        # 16384 bins (+-30 % of the width with the Float64 normals' table,
        # +-35 % without)
        far = counts[edges > 0.36 * NBINS * grid.edge_step].sum()
        assert far > 0.03 * counts.sum(), f"{case}: only {far} particles outside the window"
        assert_close(zg, zo, cfg.sigma_z, what=f"{case}: z turn {t}")
        assert_close(eg, eo, cfg.sigma_E, what=f"{case}: dE turn {t}")
    res = b.finish()
    ro = st.result()
    assert res.E0 == pytest.approx(ro.E0, rel=1e-12)
    assert res.sigma_z == pytest.approx(ro.sigma_z, rel=1e-12)
    assert res.sigma_E == pytest.approx(ro.sigma_E, rel=1e-12)
    b.close()
    st.close()
    ctx.close()


def test_batch_member_spills_at_16384_bins(gpu_ctx, gpu_buffers, oracle):
    """A batch member whose halo reaches beyond its window (the batch builds
    the grid from the bunch's own spread: a 10 % halo uniform over +-40
    sigma_z of the core puts about 2 % of the particles outside)."""
    cfg = benchmark_ring(n_turns=TURNS, nbins=NBINS)
    rng = np.random.default_rng(61)
    n = 300_001
    z0 = rng.normal(0.0, cfg.sigma_z, n)
    m = n // 10
    z0[:m] = rng.uniform(-40.0 * cfg.sigma_z, 40.0 * cfg.sigma_z, m)
    e0 = rng.normal(0.0, cfg.sigma_E, n)
    bt = Batch(gpu_ctx, pool_particles=n + 4096, max_bunches=2, max_nbins=NBINS, chunk=65536,
               layout=-1, graph_turns=0)
    seed = 4242
    bid = bt.add(z0, e0, cfg.params, NBINS, wake=cfg.wake, seed=seed, turns=TURNS)
    bt.advance(TURNS)
    assert bt.poll() == [bid]
    counts = bt.histogram(bid, NBINS)
    z, e, r = bt.take(bid)
    bt.close()
    grid = BinGrid.make(r.sigma_z0_initial, NBINS, cfg.wake.half_width_sigmas)
    zo, eo = z0.copy(), e0.copy()
    st = oracle.state(zo, eo, cfg.params.to_c(), cfg.wake.to_c(), NBINS, grid.to_c())
    for t in range(1, TURNS + 1):
        assert st.turn(gaussian_draws(seed, t, n, gpu_buffers)) == 0
    assert_close(z, zo, cfg.sigma_z, what="batch z")
    assert_close(e, eo, cfg.sigma_E, what="batch dE")
    assert np.array_equal(counts, oracle.histogram(z, grid.to_c()))
    edges = np.abs(np.asarray(grid.centers))
    assert counts[edges > 0.31 * NBINS * grid.edge_step].sum() > 0.01 * n
    st.close()
