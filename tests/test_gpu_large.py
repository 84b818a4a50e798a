"""Bunches and particle indices beyond 32 bits (int64 indexing end to end).

* A bunch of 2^32 + 65,538 particles (68.7 GB of z and dE on the device):
  the on-device initial bunch matches the Philox restatement on a window of
  particles around index 2^32 (where the counter's high word comes into
  use); the whole bunch as one shard and that window as a second shard, given
  the whole bunch's exchange buffers every turn, track the window
  bit-identically (the same draws, kicks and E0 updates); the 64-bit bin
  counts, whose total exceeds 2^32, equal the oracle's histogram of the final
  z taken chunk by chunk.
* A shard whose particles sit around index 2^33 draws its quantum excitation
  from Philox pairs beyond 2^32: the kick it adds matches the restatement.
"""
import dataclasses
import os

import numpy as np
import pytest
import torch

from haissinskijulia_b200 import BinGrid, ShardedBunch, benchmark_ring, gaussian_bunch

from gpu_util import device_pair
from philox_ref import philox_normals_reference

pytestmark = pytest.mark.gpu

N_BIG = (1 << 32) + 65_538
FIRST = (1 << 32) - 30_000      # window start: even, and a multiple of 4
M = 60_002                      # window particles (ends in a partial group of 4)
NBINS = 1024
TURNS = 3
INIT_SEED = 77
INIT_TAG = 0x6A09E667F3BCC909   # key tag of the initial-bunch stream (k_gaussian_bunch)
CHUNK = 1 << 27


def test_bunch_beyond_2_32_particles(gpu_ctx):
    torch.cuda.empty_cache()            # memory cached by earlier tests goes back to the device
    gpu_ctx.trim()
    free, _ = torch.cuda.mem_get_info()
    if free < N_BIG * 16 + (4 << 30):
        pytest.skip(f"needs {N_BIG * 16 / 1e9:.0f} GB free on the device ({free / 1e9:.0f} GB)")
    from oracle import Oracle
    cfg = benchmark_ring(n_turns=TURNS, nbins=NBINS)
    grid = BinGrid.make(cfg.sigma_z, NBINS, cfg.wake.half_width_sigmas)
    dz = torch.empty(N_BIG, dtype=torch.float64, device="cuda")
    de = torch.empty_like(dz)
    gaussian_bunch(gpu_ctx, INIT_SEED, N_BIG, cfg.sigma_z, cfg.sigma_E, dz.data_ptr(),
                   de.data_ptr())

    # particle i of the initial bunch is Philox pair i (z, dE)
    want = philox_normals_reference(INIT_SEED ^ INIT_TAG, 0, 2 * M, first_pair=FIRST)
    want = want.reshape(M, 2)
    wz = dz[FIRST:FIRST + M].clone()
    we = de[FIRST:FIRST + M].clone()
    assert np.max(np.abs(wz.cpu().numpy() / cfg.sigma_z - want[:, 0])) < 1e-13
    assert np.max(np.abs(we.cpu().numpy() / cfg.sigma_E - want[:, 1])) < 1e-13

    big = ShardedBunch(gpu_ctx, dz.data_ptr(), de.data_ptr(), N_BIG, 0, N_BIG, cfg.params,
                       grid, wake=cfg.wake, seed=5, exchange_initial=False)
    small = ShardedBunch(gpu_ctx, wz.data_ptr(), we.data_ptr(), M, FIRST, N_BIG, cfg.params,
                         grid, wake=cfg.wake, seed=5, exchange_initial=False)
    m = big.local_moments()
    big.set_global_moments(m)
    small.set_global_moments(m)
    cb, sb = big.buffers()
    cs, ss = small.buffers()
    for _ in range(TURNS):
        big.pass_()
        small.pass_()
        cs.copy_(cb)
        ss.copy_(sb)
        big.bins()
        small.bins()
    counts = big.histogram()
    assert np.array_equal(small.histogram(), counts)
    assert small.observe_local().E0 == big.observe_local().E0
    big.finish()
    small.finish()
    dzw, dew = dz[FIRST:FIRST + M], de[FIRST:FIRST + M]
    assert torch.equal(dzw, wz), f"z: max diff {float((dzw - wz).abs().max()):.3e}"
    assert torch.equal(dew, we), f"dE: max diff {float((dew - we).abs().max()):.3e}"
    small.close()
    big.close()

    assert counts.sum() > (1 << 32)
    orc = Oracle(threads=os.cpu_count() or 1)
    tot = np.zeros(NBINS, dtype=np.int64)
    for s in range(0, N_BIG, CHUNK):
        tot += orc.histogram(dz[s:s + CHUNK].cpu().numpy(), grid.to_c())
    assert np.array_equal(counts, tot)
    del dz, de, cb, sb, cs, ss
    torch.cuda.empty_cache()


def test_quantum_excitation_beyond_2_32_pairs(gpu_ctx):
    cfg = benchmark_ring(n_turns=1, nbins=NBINS)
    n_global = (1 << 33) + (1 << 17)
    first = (1 << 33) - 30_000           # pairs 2^32 - 15000 ... 2^32 + 15000
    rng = np.random.default_rng(8)
    z0 = rng.normal(0.0, cfg.sigma_z, M)
    e0 = rng.normal(0.0, cfg.sigma_E, M)
    grid = BinGrid.make(cfg.sigma_z, NBINS, cfg.wake.half_width_sigmas)
    # shards keep the wakefield on: a one-electron population makes its kick
    # ~1e-11 of the excitation's
    wake = dataclasses.replace(cfg.wake, population=1.0)
    out = []
    for qe in (True, False):
        p = dataclasses.replace(cfg.params, update_E0=False, use_excitation=qe)
        dz, de = device_pair(z0, e0)
        s = ShardedBunch(gpu_ctx, dz.data_ptr(), de.data_ptr(), M, first, n_global, p, grid,
                         wake=wake, seed=21, exchange_initial=False)
        s.set_global_moments(s.local_moments() * (n_global / M))
        s.pass_()
        s.bins()
        s.finish()
        out.append(de.cpu().numpy())
        s.close()
    # with and without excitation the turns differ by A·(1 - u)·r, r the draws of turn 1
    kick = out[0] - out[1]
    r = philox_normals_reference(21, 1, M, first_pair=first // 2)
    amp = float(np.dot(kick, r) / np.dot(r, r))
    assert amp > 0
    assert np.max(np.abs(kick / amp - r)) < 1e-6
    assert np.median(np.abs(kick / amp - r)) < 1e-8
