"""The opt-in single-precision excitation normals of the fused pass (pass
layouts with 16 added, hj_set_pass_layout): the pass draws the normals of the
numpy restatement (tests/philox_ref.py, fast_normals_reference) to the
single-precision transform's accuracy, a batch in this layout equals the
plain path in it, and the default layout's double-precision normals are
what hj_gaussian returns."""
import numpy as np
import pytest

from haissinskijulia_b200 import (Batch, Context, ResidentBunch, benchmark_ring,
                                  create_simulation_buffers, gaussian_draws)

from gpu_util import assert_close, device_pair
from philox_ref import fast_normals_reference

pytestmark = pytest.mark.gpu


def _excitation_kicks(ctx, layout, n=100_001, seed=77):
    """The excitation normals the pass applies in its first turn, read back as
    (ΔE after - ΔE before) / A with RF, SR, wake and the E0 update off."""
    ctx.set_pass_layout(layout)
    cfg = benchmark_ring(use_wakefield=False, use_excitation=True)
    p = cfg.params.replace(voltage=0.0, SR_damping=False, update_E0=False)
    rng = np.random.default_rng(3)
    z0, e0 = rng.normal(0.0, cfg.sigma_z, n), rng.normal(0.0, cfg.sigma_E, n)
    dz, de = device_pair(z0, e0)
    b = ResidentBunch(ctx, dz.data_ptr(), de.data_ptr(), n, p, 64, seed=seed)
    b.advance(1)
    r = b.finish()
    b.close()
    u = 4 * 8.85e-5 * (p.E0 / 1e9) ** 3 / p.radius
    A = np.sqrt(1.0 - (1.0 - u) ** 2) * r.sigma_E0_initial
    return (de.cpu().numpy() - e0) / A


def test_fast_layout_draws_the_restated_normals():
    ctx = Context(0)
    got = _excitation_kicks(ctx, 16 + 8)
    want = fast_normals_reference(77, 1, got.size)
    assert np.max(np.abs(got - want)) < 1e-4
    assert np.median(np.abs(got - want)) < 1e-6
    assert np.max(np.abs(got)) < 6.1           # 24-bit uniforms cut the tails near 6σ
    # the default layout applies the double-precision normals of hj_gaussian
    ctx.set_pass_layout(-1)
    dflt = _excitation_kicks(ctx, -1)
    buf = create_simulation_buffers(1, 1, ctx=ctx)
    assert np.max(np.abs(dflt - gaussian_draws(77, 1, dflt.size, buf))) < 1e-9
    ctx.close()


def test_fast_layout_batch_equals_the_plain_path():
    ctx = Context(0)
    ctx.set_pass_layout(23)                     # the library's layout, fast normals
    cfg = benchmark_ring(n_turns=1, nbins=1024, population=3e10, voltage=4e6)
    rng = np.random.default_rng(8)
    n = 70_003
    z0, e0 = rng.normal(0.0, cfg.sigma_z, n), rng.normal(0.0, cfg.sigma_E, n)
    bt = Batch(ctx, pool_particles=n + 64, max_bunches=2, max_nbins=1024, chunk=16384,
               layout=23)
    bid = bt.add(z0, e0, cfg.params, 1024, wake=cfg.wake, seed=5, turns=25)
    bt.advance(25)
    assert bt.poll() == [bid]
    zb, eb, rb = bt.take(bid)
    bt.close()
    dz, de = device_pair(z0, e0)
    b = ResidentBunch(ctx, dz.data_ptr(), de.data_ptr(), n, cfg.params, 1024, wake=cfg.wake,
                      seed=5)
    b.advance(25)
    rp = b.finish()
    b.close()
    assert_close(zb, dz.cpu().numpy(), cfg.sigma_z, what="z")
    assert_close(eb, de.cpu().numpy(), cfg.sigma_E, what="dE")
    assert rb.E0 == pytest.approx(rp.E0, rel=1e-12)
    ctx.close()
