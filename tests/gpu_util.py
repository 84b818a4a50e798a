"""Helpers shared by the GPU parity tests."""
import numpy as np
import torch

RTOL = 1e-12   # per-particle relative tolerance of the parity checks


def rel_err(a, b, scale):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), scale)


def assert_close(a, b, scale, rtol=RTOL, what=""):
    e = rel_err(a, b, scale)
    worst = float(e.max()) if e.size else 0.0
    assert worst <= rtol, f"{what}: worst relative error {worst:.3e} > {rtol:.0e} ({int((e > rtol).sum())} values)"
    return worst


def device_pair(z, dE):
    """Copies of host arrays in 32-byte aligned device memory (torch allocations)."""
    dz = torch.from_numpy(np.ascontiguousarray(z)).cuda()
    de = torch.from_numpy(np.ascontiguousarray(dE)).cuda()
    assert dz.data_ptr() % 32 == 0 and de.data_ptr() % 32 == 0
    return dz, de
