"""Philox-4x32-10 known-answer vectors (Random123 kat_vectors) for the
restatement the GPU normals are checked against."""
import numpy as np

from philox_ref import philox4x32_10, philox_normals_reference


def _kat(ctr, key):
    out = philox4x32_10(*[np.array([c], np.uint64) for c in ctr], *key)
    return [int(o[0]) for o in out]


def test_philox_zero():
    assert _kat([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]


def test_philox_ones():
    f = 0xFFFFFFFF
    assert _kat([f, f, f, f], [f, f]) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]


def test_philox_pi_digits():
    ctr = [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344]
    assert _kat(ctr, [0xA4093822, 0x299F31D0]) == [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_normals_moments():
    x = philox_normals_reference(7, 3, 400_000)
    assert abs(x.mean()) < 0.01 and abs(x.std() - 1) < 0.01
