"""Philox-4x32-10 known-answer vectors (Random123 kat_vectors) for the
restatement the GPU normals are checked against, the Box-Muller transform's
tables against 40-digit values, its table-driven logarithm, sine and cosine
restated against math, and the restated normals as a distribution."""
import math

import numpy as np

from philox_ref import normal_tables, philox4x32_10, philox_normals_reference, uniforms


def _kat(ctr, key):
    out = philox4x32_10([np.array([c], np.uint64) for c in ctr], key)
    return [int(o[0]) for o in out]


def test_philox_zero():
    assert _kat([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]


def test_philox_ones():
    assert _kat([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                        0x6D5451FD]


def test_philox_pi_digits():
    assert _kat([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_uniforms_stay_inside_the_open_interval():
    lo = np.zeros(1, np.uint64)
    hi = np.full(1, 0xFFFFFFFF, np.uint64)
    u1, w = uniforms(lo, lo, lo, lo)
    assert u1[0] == 2.0 ** -53 and w[0] == 0.0
    u1, w = uniforms(hi, hi, hi, hi)
    assert u1[0] == 1.0 - 2.0 ** -53 and w[0] == 1.0 - 2.0 ** -52
    # the largest normal radius the transform can produce
    assert math.sqrt(-2.0 * math.log(2.0 ** -53)) < 8.58


def test_normals_moments():
    x = philox_normals_reference(7, 3, 400_000)
    assert abs(x.mean()) < 0.01 and abs(x.std() - 1) < 0.01


def test_normals_from_a_pair_offset():
    whole = philox_normals_reference(11, 5, 1000)
    assert np.array_equal(philox_normals_reference(11, 5, 600, first_pair=200), whole[400:])
    # beyond 2^32 pairs the counter's second word carries p >> 32
    hi = philox_normals_reference(11, 5, 4, first_pair=(1 << 32) - 1)
    lo = philox_normals_reference(11, 5, 2, first_pair=0)
    assert not np.array_equal(hi[2:], lo)


def test_seeds_differing_only_in_the_high_word_give_different_streams():
    a = philox_normals_reference(5, 1, 64)
    b = philox_normals_reference(5 + (1 << 32), 1, 64)
    c = philox_normals_reference(5, 1 + (1 << 32), 64)
    assert not np.array_equal(a, b) and not np.array_equal(a, c)


def test_transform_tables_against_40_digit_values():
    """The library's tables against 40-digit mpmath: r_j, -ln r_j, sin θ_j,
    cos θ_j, and the two-part ln 2 and 2π."""
    import mpmath as mp
    mp.mp.dps = 40
    t = normal_tables()
    for j in range(128):
        r = t["lr"][j][0]
        assert abs(r - float(1 / (1 + (mp.mpf(j) + 0.5) / 128))) <= 2.0 ** -53 * r
        # extended precision rounded once: within one ulp of the exact value
        lnr = -mp.log(mp.mpf(r))
        assert abs(mp.mpf(t["lr"][j][1]) - lnr) <= 2.0 ** -52 * abs(lnr)
        th = 2 * mp.pi * (mp.mpf(j) + 0.5) / 128
        for got, want in ((t["sc"][j][0], mp.sin(th)), (t["sc"][j][1], mp.cos(th))):
            assert abs(mp.mpf(got) - want) <= 2.0 ** -52 * abs(want)
    # the two parts carry the long double constants (64-bit mantissas): 1e-18 is
    # far below what e ln 2 (|e| <= 53) and 2π w need
    assert abs(mp.mpf(t["ln2_hi"]) + mp.mpf(t["ln2_lo"]) - mp.log(2)) < 1e-18
    assert t["ln2_hi"] * 2.0 ** 42 == int(t["ln2_hi"] * 2.0 ** 42)   # e * hi exact, |e| < 2^11
    assert abs(mp.mpf(t["twopi_hi"]) + mp.mpf(t["twopi_lo"]) - 2 * mp.pi) < 1e-18


def test_table_driven_transform_restated():
    """The device's table-driven logarithm, sine and cosine (hj_device.cuh,
    box_muller_f64) restated in float64 with the library's tables, against
    40-digit logarithms, sines and cosines on uniforms that span their
    ranges."""
    import mpmath as mp
    mp.mp.dps = 40
    t = normal_tables()
    rng = np.random.default_rng(4)
    us = np.concatenate([rng.random(3000), 2.0 ** -rng.uniform(1, 53, 3000),
                         [2.0 ** -53, 0.5, 1 - 2.0 ** -53]])
    for u in us:
        m, e = math.frexp(u)                       # u = m 2^e, m in [0.5, 1)
        m, e = 2 * m, e - 1
        j = int((m - 1) * 128)
        r, nlr = t["lr"][j]
        tt = m * r - 1.0
        q = sum((-1) ** (k + 1) * tt ** (k - 1) / k for k in range(1, 7))
        got = e * t["ln2_hi"] + nlr + e * t["ln2_lo"] + tt * q
        want = float(mp.log(mp.mpf(u)))
        assert abs(got - want) <= 6e-16 * max(1.0, abs(want))
    for w in np.concatenate([rng.random(3000), [0.0, 0.5, 1 - 2.0 ** -52]]):
        k = int(w * 128)
        xs = w - (k + 0.5) / 128
        a = xs * t["twopi_hi"] + xs * t["twopi_lo"]
        sn = sum((-1) ** i * a ** (2 * i + 1) / math.factorial(2 * i + 1) for i in range(4))
        cm1 = sum((-1) ** i * a ** (2 * i) / math.factorial(2 * i) for i in range(1, 5))
        sk, ck = t["sc"][k]
        th = 2 * mp.pi * mp.mpf(w)
        assert abs(sk * (1 + cm1) + ck * sn - float(mp.sin(th))) <= 4e-16
        assert abs(ck * (1 + cm1) - sk * sn - float(mp.cos(th))) <= 4e-16


def test_normal_tail_and_ks_of_the_restatement():
    """KS distance of 4e6 restated normals to the standard normal CDF, and the
    two-sided 3σ tail frequency against its exact value."""
    x = np.sort(philox_normals_reference(2024, 1, 4_000_000))
    from scipy.special import ndtr
    cdf = ndtr(x)
    n = x.size
    d = max(np.max(np.arange(1, n + 1) / n - cdf), np.max(cdf - np.arange(n) / n))
    assert d < 1.63 / math.sqrt(n)             # KS critical value at the 1 % level
    p3 = math.erfc(3.0 / math.sqrt(2.0))
    k = np.count_nonzero(np.abs(x) > 3.0)
    assert abs(k - n * p3) < 4.0 * math.sqrt(n * p3)
