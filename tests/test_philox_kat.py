"""Philox-2x32-10 known-answer vectors (Random123 kat_vectors) for the
restatement the GPU normals are checked against."""
import numpy as np

from philox_ref import philox2x32_10, philox_normals_reference


def _kat(ctr, key):
    out = philox2x32_10(np.array([ctr[0]], np.uint64), np.array([ctr[1]], np.uint64), key)
    return [int(o[0]) for o in out]


def test_philox_zero():
    assert _kat([0, 0], 0) == [0xFF1DAE59, 0x6CD10DF2]


def test_philox_ones():
    assert _kat([0xFFFFFFFF, 0xFFFFFFFF], 0xFFFFFFFF) == [0x2C3F628B, 0xAB4FD7AD]


def test_philox_pi_digits():
    assert _kat([0x243F6A88, 0x85A308D3], 0x13198A2E) == [0xDD7CE038, 0xF62A4C12]


def test_normals_moments():
    x = philox_normals_reference(7, 3, 400_000)
    assert abs(x.mean()) < 0.01 and abs(x.std() - 1) < 0.01


def test_normals_from_a_pair_offset():
    whole = philox_normals_reference(11, 5, 1000)
    assert np.array_equal(philox_normals_reference(11, 5, 600, first_pair=200), whole[400:])
    # beyond 2^32 pairs the counter's high word carries p >> 32
    hi = philox_normals_reference(11, 5, 4, first_pair=(1 << 32) - 1)
    lo = philox_normals_reference(11, 5, 2, first_pair=0)
    assert not np.array_equal(hi[2:], lo)
