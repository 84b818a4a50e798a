"""Batches of independent bunches (hj_batch_*) against the plain resident path.

A bunch advanced in a batch sees the same arithmetic as alone: the same
Philox draws (seed, particle, turn), the same per-particle code and the same
bins step; only the blocking of its partial sums differs from the plain
path's grid, so (z, ΔE) agree within 1e-12 relative, and a bunch's results are
bit-identical whichever other bunches share the batch."""
import numpy as np
import pytest
import torch

from haissinskijulia_b200 import Batch, Context, HaissinskiError, ResidentBunch, benchmark_ring
from haissinskijulia_b200 import _lib

from gpu_util import assert_close, device_pair

pytestmark = pytest.mark.gpu


def _bunch(n, seed, cfg):
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, cfg.sigma_z, n), rng.normal(0.0, cfg.sigma_E, n)


def _spec(i):
    """Bunch i of the test sweep: own size, voltage, intensity, bins, seed."""
    n = [5003, 40_000, 123_457, 777, 65_536][i]
    volt = [3e6, 5e6, 7e6, 4e6, 6e6][i]
    pop = [1e9, 1e10, 1e11, 3e10, 5e9][i]
    nbins = [512, 1024, 2048, 256, 1024][i]
    cfg = benchmark_ring(n_turns=1, nbins=nbins, population=pop, voltage=volt)
    z, dE = _bunch(n, 100 + i, cfg)
    return cfg, z, dE, nbins, 1000 + i


def _plain(ctx, cfg, z, dE, nbins, seed, turns):
    dz, de = device_pair(z, dE)
    b = ResidentBunch(ctx, dz.data_ptr(), de.data_ptr(), z.size, cfg.params, nbins,
                      wake=cfg.wake, seed=seed)
    b.advance(turns)
    r = b.finish()
    b.close()
    return dz.cpu().numpy(), de.cpu().numpy(), r


def _check(a, b, cfg, what):
    za, ea, ra = a
    zb, eb, rb = b
    assert_close(za, zb, cfg.sigma_z, what=f"z {what}")
    assert_close(ea, eb, cfg.sigma_E, what=f"dE {what}")
    assert ra.E0 == pytest.approx(rb.E0, rel=1e-12)
    assert ra.sigma_E == pytest.approx(rb.sigma_E, rel=1e-12)
    assert ra.sigma_z == pytest.approx(rb.sigma_z, rel=1e-12)


@pytest.mark.parametrize("layout", [-1, 0, 1, 2, 3, 4, 5, 8, 9, 12, 13])
def test_batch_matches_the_plain_path_with_ragged_turns(gpu_ctx, layout):
    turns = [20, 35, 27, 20, 40]
    bt = Batch(gpu_ctx, pool_particles=300_000, max_bunches=8, max_nbins=2048, chunk=16384,
               layout=layout)
    ids = {}
    for i in range(5):
        cfg, z, dE, nbins, seed = _spec(i)
        ids[bt.add(z, dE, cfg.params, nbins, wake=cfg.wake, seed=seed, turns=turns[i])] = i
    done = {}
    for _ in range(5):                       # 5 x 8 turns, with a poll between blocks
        bt.advance(8)
        for bid in bt.poll():
            done[ids[bid]] = bt.take(bid)
    assert sorted(done) == list(range(5))
    assert bt.stats()["live"] == 0
    for i in range(5):
        cfg, z, dE, nbins, seed = _spec(i)
        _check(done[i], _plain(gpu_ctx, cfg, z, dE, nbins, seed, turns[i]), cfg, f"bunch {i}")
    bt.close()


def test_results_do_not_depend_on_the_mix(gpu_ctx):
    """Bunch 2 alone, and in a batch with others admitted before and after it
    (graph replays and direct launches mixed): bit-identical results."""
    cfg, z, dE, nbins, seed = _spec(2)
    alone = Batch(gpu_ctx, 200_000, 4, 2048, chunk=16384, graph_turns=0)
    a = alone.add(z, dE, cfg.params, nbins, wake=cfg.wake, seed=seed, turns=30)
    alone.advance(30)
    assert alone.poll() == [a]
    za, ea, ra = alone.take(a)
    alone.close()

    mix = Batch(gpu_ctx, 400_000, 6, 2048, chunk=16384, graph_turns=8)
    for i in (0, 1):
        c, zz, ee, nb, s = _spec(i)
        mix.add(zz, ee, c.params, nb, wake=c.wake, seed=s, turns=50)
    mix.advance(5)                                   # the others are already running
    m = mix.add(z, dE, cfg.params, nbins, wake=cfg.wake, seed=seed, turns=30)
    c, zz, ee, nb, s = _spec(4)
    mix.add(zz, ee, c.params, nb, wake=c.wake, seed=s, turns=50)
    mix.advance(17)
    mix.advance(13)
    assert m in mix.poll()
    zm, em, rm = mix.take(m)
    mix.close()
    assert np.array_equal(za, zm) and np.array_equal(ea, em)
    assert (ra.E0, ra.sigma_E, ra.sigma_z) == (rm.E0, rm.sigma_E, rm.sigma_z)


def test_admission_is_refused_when_the_batch_is_full(gpu_ctx):
    cfg, z, dE, nbins, seed = _spec(1)
    bt = Batch(gpu_ctx, 50_000, 2, 1024)
    bt.add(z, dE, cfg.params, nbins, wake=cfg.wake, seed=seed, turns=3)
    with pytest.raises(HaissinskiError) as e:
        bt.add(z, dE, cfg.params, nbins, wake=cfg.wake, seed=seed, turns=3)  # pool
    assert e.value.status == _lib.HJ_ERR_FULL
    c4, z4, e4, nb4, s4 = _spec(3)
    with pytest.raises(HaissinskiError) as e:
        bt.add(z4, e4, c4.params, 4096, wake=c4.wake, seed=s4, turns=3)      # bins
    assert e.value.status == _lib.HJ_ERR_FULL
    bt.advance(3)
    (bid,) = bt.poll()
    bt.take(bid, copy_out=False)
    bt.add(z, dE, cfg.params, nbins, wake=cfg.wake, seed=seed, turns=3)      # room again
    bt.close()


def test_admitting_and_taking_many_at_once(gpu_ctx):
    """hj_batch_add_many / hj_batch_take_many give the bunches that one-by-one
    admission and retirement give, bit for bit, stop at the first bunch that
    does not fit, and take the correlation of each final bunch."""
    from haissinskijulia_b200.api import correlation_device
    specs = [_spec(i) for i in range(5)]
    turns = [12, 9, 15, 12, 10]

    one = Batch(gpu_ctx, 300_000, 8, 2048, chunk=16384)
    ids1 = [one.add(z, dE, c.params, nb, wake=c.wake, seed=s, turns=t)
            for (c, z, dE, nb, s), t in zip(specs, turns)]
    one.advance(16)
    assert sorted(one.poll()) == sorted(ids1)
    outs1 = {}
    for i, bid in enumerate(ids1):
        dz = torch.empty(specs[i][1].size, dtype=torch.float64, device="cuda")
        de = torch.empty_like(dz)
        r = one.take_device(bid, dz.data_ptr(), de.data_ptr())
        outs1[i] = (r, correlation_device(gpu_ctx, dz.data_ptr(), de.data_ptr(), dz.numel()))
    one.close()

    many = Batch(gpu_ctx, 300_000, 8, 2048, chunk=16384)
    keep = [(z, dE) for (_, z, dE, _, _) in specs]          # host arrays alive for the call
    ids, err = many.add_many([k[0] for k in keep], [k[1] for k in keep],
                             [z.size for (_, z, _, _, _) in specs], [c.params for c, *_ in specs],
                             [nb for (_, _, _, nb, _) in specs], [s for *_, s in specs], turns,
                             wakes=[c.wake for c, *_ in specs])
    assert err is None and len(ids) == 5
    many.advance(16)
    assert sorted(many.poll()) == sorted(ids)
    res, corr = many.take_many(ids, correlation=True)
    assert many.stats()["live"] == 0
    for i in range(5):
        r1, c1 = outs1[i]
        assert (res[i].E0, res[i].sigma_E, res[i].sigma_z) == (r1.E0, r1.sigma_E, r1.sigma_z)
        assert abs(corr[i] - c1) <= 1e-13
    # admission stops at the first bunch with no room and says so
    c, z, dE, nb, s = specs[2]                                # 123457 particles
    ids, err = many.add_many([z] * 3, [dE] * 3, [z.size] * 3, [c.params] * 3, [nb] * 3,
                             [s] * 3, [5] * 3)
    assert len(ids) == 2 and err is not None and err.status == _lib.HJ_ERR_FULL
    many.close()


@pytest.mark.parametrize("n", [2, 3, 5, 9])
def test_tiny_bunches_match_the_plain_path(gpu_ctx, n):
    """Bunches of a few particles (the scalar tail of the pass, one partial
    chunk) give in a batch what they give alone on the plain path."""
    cfg = benchmark_ring(n_turns=1, nbins=256)
    z, dE = _bunch(n, 7 + n, cfg)
    bt = Batch(gpu_ctx, 1024, 2, 256, chunk=16384)
    bid = bt.add(z, dE, cfg.params, 256, wake=cfg.wake, seed=3, turns=6)
    bt.advance(6)
    assert bt.poll() == [bid]
    got = bt.take(bid)
    bt.close()
    _check(got, _plain(gpu_ctx, cfg, z, dE, 256, 3, 6), cfg, f"{n} particles")


def test_a_bunch_with_no_turns_is_done_at_once(gpu_ctx):
    cfg, z, dE, nbins, seed = _spec(0)
    bt = Batch(gpu_ctx, 20_000, 2, 1024)
    bid = bt.add(z, dE, cfg.params, nbins, wake=cfg.wake, seed=seed, turns=0)
    bt.advance(1)
    assert bt.poll() == [bid]
    zz, ee, r = bt.take(bid)
    bt.close()
    assert r.turns == 0 and r.E0 == cfg.params.E0
    assert np.array_equal(zz, z) and np.array_equal(ee, dE)


def test_results_count_the_turns_run(gpu_ctx):
    cfg, z, dE, nbins, seed = _spec(1)
    bt = Batch(gpu_ctx, 100_000, 2, 1024)
    bid = bt.add(z, dE, cfg.params, nbins, wake=cfg.wake, seed=seed, turns=11)
    bt.advance(16)
    assert bt.poll() == [bid]
    _, _, r = bt.take(bid, copy_out=False)
    bt.close()
    assert r.turns == 11


def test_closing_the_context_first_leaves_its_bunches_working(gpu_ctx):
    """hj_destroy before the bunch and the batch: both keep working (the batch
    still admits) and the last one destroyed frees the context."""
    cfg = benchmark_ring(n_turns=1, nbins=512)
    z, dE = _bunch(20_000, 7, cfg)
    want = _plain(gpu_ctx, cfg, z, dE, 512, 11, 12)
    ctx = Context(0)
    dz, de = device_pair(z, dE)
    b = ResidentBunch(ctx, dz.data_ptr(), de.data_ptr(), z.size, cfg.params, 512,
                      wake=cfg.wake, seed=11)
    bt = Batch(ctx, pool_particles=50_000, max_bunches=2, max_nbins=512, chunk=16384)
    ctx.close()
    bid = bt.add(z, dE, cfg.params, 512, wake=cfg.wake, seed=11, turns=12)
    b.advance(12)
    r = b.finish()
    b.close()
    _check((dz.cpu().numpy(), de.cpu().numpy(), r), want, cfg, "bunch after close")
    for _ in range(4):
        bt.advance(4)
        if bid in bt.poll():
            break
    got = bt.take(bid)
    bt.close()                          # the last object: frees the context
    _check(got, want, cfg, "batch after close")


def test_resident_queue_and_one_block_per_chunk_agree_bit_for_bit(gpu_ctx):
    """The resident pass (blocks taking chunks from a device-side queue) and
    one block per chunk give the same results: a chunk's slot and arithmetic
    do not depend on the block that takes it."""
    out = []
    for resident in (True, False):
        bt = Batch(gpu_ctx, 400_000, 6, 2048, chunk=16384, graph_turns=4, resident=resident)
        ids = []
        for i in range(5):
            cfg, z, dE, nbins, seed = _spec(i)
            ids.append(bt.add(z, dE, cfg.params, nbins, wake=cfg.wake, seed=seed, turns=21))
        bt.advance(21)
        assert sorted(bt.poll()) == sorted(ids)
        out.append([bt.take(b) for b in ids])
        bt.close()
    for (za, ea, ra), (zb, eb, rb) in zip(*out):
        assert np.array_equal(za, zb) and np.array_equal(ea, eb)
        assert (ra.E0, ra.sigma_E, ra.sigma_z) == (rb.E0, rb.sigma_E, rb.sigma_z)
