"""hj_wake_potential_noalloc: the wake potential for callers that cannot
call cudaMalloc (device memory owned by another allocator, latency-critical
loops).  Through the C ABI, on consecutive calls that reuse the shared static
scratch, its output must match the allocating entry point hj_wake_potential
and the oracle's long-double direct convolution within 1e-13 of the largest
|potential|, the tolerance of the other wake-potential tests.  The grids reach
every branch of the convolution: the 8-CTA (16384 bins), 4-CTA (4096) and
2-CTA (512) cluster FFTs and the direct sum of tiny grids (3 bins).  This file
is collected last so that a run stopping at the first failure has already run
every other test."""
import ctypes

import numpy as np
import pytest
import torch

from haissinskijulia_b200 import (BinGrid, Context, benchmark_ring, create_simulation_buffers,
                                  wake_potential)
from haissinskijulia_b200 import _lib

pytestmark = pytest.mark.gpu


def _noalloc(ctx, counts, grid, wake, current):
    d_counts = torch.from_numpy(np.ascontiguousarray(counts, dtype=np.int64)).cuda()
    d_pot = torch.full((grid.nbins,), float("nan"), dtype=torch.float64, device="cuda")
    g, w = grid.to_c(), wake.to_c()
    stream = torch.cuda.current_stream().cuda_stream
    rc = ctx._lib.hj_wake_potential_noalloc(ctx.handle, ctypes.c_void_p(d_counts.data_ptr()),
                                            ctypes.byref(g), ctypes.byref(w), float(current),
                                            ctypes.c_void_p(d_pot.data_ptr()),
                                            ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, d_pot.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_and_oracle():
    from haissinskijulia_b200 import build as hjbuild
    from oracle import Oracle
    from oracle.pyoracle import CONV_DIRECT_LD
    hjbuild.build()
    ctx = Context(0)
    orc = Oracle(threads=1)
    wake = benchmark_ring().wake
    rng = np.random.default_rng(17)
    # consecutive calls over the scratch the previous one left behind: a
    # smaller grid after a larger one, tiny grids, then the first grid again
    cases = [(16384, 4e-3, 2.9e-15), (4096, 3.1e-3, 1.7e-15), (512, 4e-3, 2.9e-15),
             (3, 4e-3, 2.9e-15), (3, 2e-3, 1.1e-15), (16384, 4e-3, 2.9e-15)]
    for B, sigma, current in cases:
        grid = BinGrid.make(sigma, B, 6.0)
        z = rng.normal(0.0, sigma, 400_000)
        counts = orc.histogram(z, grid.to_c())
        rc, got = _noalloc(ctx, counts, grid, wake, current)
        assert rc == _lib.HJ_OK, ctx.last_error()
        assert ctx.last_error() == ""
        want = wake_potential(counts, grid, wake, current,
                              create_simulation_buffers(1, B, ctx=ctx))
        exact = orc.wake_potential(counts, grid.to_c(), wake.to_c(), current, CONV_DIRECT_LD)
        scale = np.abs(exact).max()
        assert scale > 0
        assert np.all(np.isfinite(got))
        assert np.abs(got - want).max() <= 1e-13 * scale, B
        assert np.abs(got - exact).max() <= 1e-13 * scale, B


def test_noalloc_restores_the_callers_device_and_clears_the_last_error():
    ctx = Context(0)
    grid = BinGrid.make(4e-3, 32768, 6.0)
    rc, _ = _noalloc(ctx, np.ones(32768, np.int64), grid, benchmark_ring().wake, 1e-15)
    assert rc == _lib.HJ_ERR_TOO_LARGE
    assert "16384" in ctx.last_error()
    # a successful call clears the error the failed one left
    small = BinGrid.make(4e-3, 64, 6.0)
    rc, pot = _noalloc(ctx, np.arange(64, dtype=np.int64), small, benchmark_ring().wake, 1e-15)
    assert rc == _lib.HJ_OK and ctx.last_error() == "" and np.all(np.isfinite(pot))
    assert torch.cuda.current_device() == 0


def test_noalloc_rejects_bad_grids():
    ctx = Context(0)
    wake = benchmark_ring().wake
    grid = BinGrid.make(4e-3, 64, 6.0)
    g = grid.to_c()
    g.edge_step = 0.0                 # the check_grid rule of the allocating entry point
    d_counts = torch.zeros(64, dtype=torch.int64, device="cuda")
    d_pot = torch.zeros(64, dtype=torch.float64, device="cuda")
    rc = ctx._lib.hj_wake_potential_noalloc(ctx.handle, ctypes.c_void_p(d_counts.data_ptr()),
                                            ctypes.byref(g), ctypes.byref(wake.to_c()), 1e-15,
                                            ctypes.c_void_p(d_pot.data_ptr()), None)
    assert rc == _lib.HJ_ERR_ARG and "zero step" in ctx.last_error()
