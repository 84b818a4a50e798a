"""The sharded bunch's exchange, checked on the CPU with two gloo ranks.

Each rank tracks half of a bunch with the oracle's per-particle steps and
performs exactly the exchanges the GPU shards perform (the sums behind σ_z,
the bin counts, the energy change); the result must equal the single-process
oracle: bin counts bit-exact, E0 and every particle within 1e-12."""
import os
import socket
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

N = 20_000
TURNS = 6
NBINS = 512


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    sys.path[:0] = [ROOT, HERE]
    import datetime

    import torch
    import torch.distributed as dist

    from haissinskijulia_b200 import BinGrid, benchmark_ring
    from oracle import Oracle
    from sharded_oracle import global_std, sharded_turn

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        def allreduce(a):
            t = torch.from_numpy(np.ascontiguousarray(a))
            dist.all_reduce(t)
            return t.numpy()

        orc = Oracle(threads=1)
        cfg = benchmark_ring(n_turns=TURNS, nbins=NBINS)
        rng = np.random.default_rng(77)
        z0 = rng.normal(0.0, cfg.sigma_z, N)
        e0 = rng.normal(0.0, cfg.sigma_E, N)
        draws = rng.standard_normal((TURNS, N))
        grid = BinGrid.make(orc.global_std(z0), NBINS, cfg.wake.half_width_sigmas)
        gc, wc, p = grid.to_c(), cfg.wake.to_c(), cfg.params

        # single process, whole bunch
        zs, es = z0.copy(), e0.copy()
        st = orc.state(zs, es, p.to_c(), wc, NBINS, gc)
        # this rank's shard (even start, as the GPU shards require)
        lo = (N // world) * rank // 2 * 2
        hi = N if rank == world - 1 else (N // world) * (rank + 1) // 2 * 2
        z, dE = z0[lo:hi].copy(), e0[lo:hi].copy()
        m = allreduce(np.array([dE.sum(), (dE * dE).sum()]))
        sigma_E0 = global_std(m[0], m[1], N)
        E0 = p.E0
        ok = True
        for t in range(TURNS):
            assert st.turn(np.ascontiguousarray(draws[t])) == 0
            E0, counts = sharded_turn(orc, allreduce, z, dE, np.ascontiguousarray(draws[t, lo:hi]),
                                      E0, p, wc, gc, N, sigma_E0)
            ok &= bool(np.array_equal(counts, st.counts()))
            ok &= abs(E0 - st.E0) <= 1e-12 * st.E0
        ok &= bool(np.all(np.abs(z - zs[lo:hi]) <= 1e-12 * cfg.sigma_z))
        ok &= bool(np.all(np.abs(dE - es[lo:hi]) <= 1e-12 * cfg.sigma_E))
        results[rank] = ok
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_single_process_oracle():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    results = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, results)) for r in range(2)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=240)
    for pr in procs:
        if pr.is_alive():
            pr.kill()
    assert [pr.exitcode for pr in procs] == [0, 0]
    assert dict(results) == {0: True, 1: True}
