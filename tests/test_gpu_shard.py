"""Shards of one bunch (hj_bunch_create_shard / pass / exchange / bins).

Two shards on one GPU, their exchange buffers summed between the pass and
the bins step as an all-reduce across two GPUs would, reproduce the whole
bunch tracked by the plain resident path: the same Philox draws, bin counts
bit-exact every turn, E0 and every particle within 1e-12.  And one shard in a
one-rank NCCL group runs the same turns through ShardedBunch.advance."""
import datetime
import socket

import numpy as np
import pytest
import torch

from haissinskijulia_b200 import BinGrid, ResidentBunch, ShardedBunch, benchmark_ring

from gpu_util import assert_close, device_pair

pytestmark = pytest.mark.gpu

N = 60_002
TURNS = 12
NBINS = 1024


def _setup():
    cfg = benchmark_ring(n_turns=TURNS, nbins=NBINS)
    rng = np.random.default_rng(31)
    z0 = rng.normal(0.0, cfg.sigma_z, N)
    e0 = rng.normal(0.0, cfg.sigma_E, N)
    grid = BinGrid.make(cfg.sigma_z, NBINS, cfg.wake.half_width_sigmas)
    return cfg, z0, e0, grid


def test_two_shards_reproduce_the_whole_bunch(gpu_ctx):
    cfg, z0, e0, grid = _setup()
    dz, de = device_pair(z0, e0)
    whole = ResidentBunch(gpu_ctx, dz.data_ptr(), de.data_ptr(), N, cfg.params, NBINS,
                          wake=cfg.wake, grid=grid, seed=5)
    cut = 24_000
    parts = [device_pair(z0[:cut], e0[:cut]), device_pair(z0[cut:], e0[cut:])]
    shards = [ShardedBunch(gpu_ctx, p[0].data_ptr(), p[1].data_ptr(), p[0].numel(), first, N,
                           cfg.params, grid, wake=cfg.wake, seed=5, exchange_initial=False)
              for p, first in zip(parts, (0, cut))]
    m = sum(s.local_moments() for s in shards)
    for s in shards:
        s.set_global_moments(m)
    bufs = [s.buffers() for s in shards]
    for t in range(TURNS):
        whole.advance(1)
        for s in shards:
            s.pass_()
        tot_c = bufs[0][0] + bufs[1][0]
        tot_s = bufs[0][1] + bufs[1][1]
        for c, sm in bufs:
            c.copy_(tot_c)
            sm.copy_(tot_s)
        for s in shards:
            s.bins()
        counts = whole.histogram()
        for s in shards:
            assert np.array_equal(s.histogram(), counts), f"counts turn {t + 1}"
        r = whole.observe()
        for s in shards:
            assert s.observe_local().E0 == pytest.approx(r.E0, rel=1e-12)
    g = shards[0].global_result(sum(s.local_moments() for s in shards))
    rw = whole.finish()
    assert g.sigma_E == pytest.approx(rw.sigma_E, rel=1e-12)
    assert g.sigma_z == pytest.approx(rw.sigma_z, rel=1e-12)
    for s in shards:
        s.finish()
    zs = torch.cat([parts[0][0], parts[1][0]]).cpu().numpy()
    es = torch.cat([parts[0][1], parts[1][1]]).cpu().numpy()
    assert_close(zs, dz.cpu().numpy(), cfg.sigma_z, what="z")
    assert_close(es, de.cpu().numpy(), cfg.sigma_E, what="dE")
    for s in shards:
        s.close()
    whole.close()


def test_one_rank_nccl_group_advances_a_shard(gpu_ctx):
    import torch.distributed as dist
    cfg, z0, e0, grid = _setup()
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        dz, de = device_pair(z0, e0)
        whole = ResidentBunch(gpu_ctx, dz.data_ptr(), de.data_ptr(), N, cfg.params, NBINS,
                              wake=cfg.wake, grid=grid, seed=9)
        sz, se = device_pair(z0, e0)
        stream = torch.cuda.current_stream().cuda_stream
        shard = ShardedBunch(gpu_ctx, sz.data_ptr(), se.data_ptr(), N, 0, N, cfg.params, grid,
                             wake=cfg.wake, seed=9, stream=stream)
        whole.advance(TURNS)
        shard.advance(TURNS)
        torch.cuda.synchronize()
        assert np.array_equal(shard.histogram(), whole.histogram())
        g = shard.global_result()
        rw = whole.finish()
        assert g.E0 == pytest.approx(rw.E0, rel=1e-12)
        assert g.sigma_E == pytest.approx(rw.sigma_E, rel=1e-12)
        shard.finish()
        assert_close(sz.cpu().numpy(), dz.cpu().numpy(), cfg.sigma_z, what="z")
        assert_close(se.cpu().numpy(), de.cpu().numpy(), cfg.sigma_E, what="dE")
        shard.close()
        whole.close()
    finally:
        dist.destroy_process_group()
