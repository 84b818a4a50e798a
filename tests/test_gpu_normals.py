"""The device's quantum-excitation normals (Philox-4x32-10 and a 2048-layer
Float64 ziggurat, hj_device.cuh) as a distribution:
the two-sided tail frequencies beyond 4, 5 and 6 standard deviations over
1e10 draws against the exact normal tail, and a Kolmogorov-Smirnov test of
1e7 draws.  The reference draws Float64 normals with randn!
(src/quantum_excitation.jl:36)."""
import math

import numpy as np
import pytest
import torch

from haissinskijulia_b200 import create_simulation_buffers, gaussian_bunch, gaussian_draws

pytestmark = pytest.mark.gpu


def test_tail_frequencies_over_1e10_draws(gpu_ctx):
    m = 500_000_000                         # pairs per call: 1e9 normals in two arrays
    calls = 10
    z = torch.empty(m, dtype=torch.float64, device="cuda")
    e = torch.empty_like(z)
    counts = {4.0: 0, 5.0: 0, 6.0: 0}
    total = 0
    largest = 0.0
    for c in range(calls):
        gaussian_bunch(gpu_ctx, 1000 + c, m, 1.0, 1.0, z.data_ptr(), e.data_ptr())
        torch.cuda.synchronize()
        for x in (z, e):
            a = x.abs()
            for k in counts:
                counts[k] += int((a > k).sum().item())
            largest = max(largest, float(a.max().item()))
        total += 2 * m
    assert total == 10 ** 10
    for k, got in counts.items():
        p = math.erfc(k / math.sqrt(2.0))
        want = total * p
        assert abs(got - want) <= 4.0 * math.sqrt(want), (k, got, want)
    # 1e10 draws reach beyond 6σ with probability 1 - 3e-9; the tail method
    # gives at most r - ln(2^-53)/r = 12.93σ
    assert 6.0 < largest < 12.93
    del z, e
    torch.cuda.empty_cache()


def test_kolmogorov_smirnov_of_1e7_draws(gpu_ctx):
    from scipy.special import ndtr
    buf = create_simulation_buffers(1, 1, ctx=gpu_ctx)
    x = np.sort(gaussian_draws(31337, 9, 10_000_000, buf))
    n = x.size
    cdf = ndtr(x)
    d = max(np.max(np.arange(1, n + 1) / n - cdf), np.max(cdf - np.arange(n) / n))
    assert d < 1.63 / math.sqrt(n)          # 1 % critical value
