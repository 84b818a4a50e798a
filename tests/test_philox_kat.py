"""Philox-4x32-10 known-answer vectors (Random123 kat_vectors) for the
restatement the GPU normals are checked against, the ziggurat's tables
against their defining equations in 40-digit arithmetic, its
fast-acceptance rate, its tail sampler against the conditional normal tail,
and the restated normals as a distribution."""
import math

import numpy as np

from philox_ref import (fraction, normal_tables, philox4x32_10, philox_normals_reference, zig_fast,
                        zig_slow)


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


def test_draw_decoding_and_extremes():
    """A draw's layer is hi >> 21, its sign bit 20 of hi and its fraction the
    52 bits (hi mod 2^20):lo; the all-zero draw is 0 (accepted) and every draw
    of the top layer goes to the slow path."""
    t = normal_tables()
    zero = np.zeros(1, np.uint64)
    x, ok = zig_fast(zero, zero, t)
    assert x[0] == 0.0 and ok[0]
    hi = np.array([(7 << 21) | (1 << 20) | 0xABCDE], np.uint64)
    lo = np.array([0x12345678], np.uint64)
    assert fraction(hi, lo)[0] == float((0xABCDE << 32) | 0x12345678)
    x, _ = zig_fast(hi, lo, t)
    assert x[0] == -(fraction(hi, lo)[0] * 2.0 ** -52) * t["xd"][7, 0]
    top = np.array([0xFFEFFFFF], np.uint64)
    _, ok = zig_fast(top, np.zeros(1, np.uint64), t)
    assert not ok[0] and t["xd"][2047, 1] == 1.0


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


def test_ziggurat_tables_against_40_digit_values():
    """The library's tables against their defining equations in 40-digit
    mpmath: every layer's area equal to v, the base layer (rectangle and
    tail) too, the recursion ending at the top, f(X_i) to its rounding, and
    each fast bound D_i = 1 + ceil(2^52 X_{i+1}/X_i) 2^-52 (to one unit of
    K_i).  (For 256 layers the same construction gives Marsaglia and Tsang's
    published r = 3.6541528853610088.)"""
    import mpmath as mp
    mp.mp.dps = 40
    t = normal_tables()
    n = len(t["xd"])
    X = [mp.mpf(float(x)) for x in t["xd"][:, 0]] + [mp.mpf(0)]
    r, v = X[1], mp.mpf(float(t["v"]))
    assert n == 2048 and 4.2 < float(t["r"]) < 4.23 and X[1] == mp.mpf(float(t["r"]))
    f = lambda x: mp.exp(-x * x / 2)
    base = r * f(r) + mp.sqrt(mp.pi / 2) * mp.erfc(r / mp.sqrt(2))
    assert abs(base - v) <= 1e-15 * v
    assert abs(X[0] * f(r) - v) <= 1e-15 * v
    for i in range(1, n):
        area = X[i] * (f(X[i + 1]) - f(X[i]))
        assert abs(area - v) <= 2e-12 * v, (i, float(area / v - 1))
    assert abs(f(X[n - 1]) + v / X[n - 1] - 1) <= 1e-14
    # f was rounded once from the extended-precision X_i, X_i once to double:
    # both within an ulp, and |d ln f / d ln X| = X² < 16
    for i in range(n + 1):
        assert abs(mp.mpf(float(t["f"][i])) - f(X[i])) <= 2.0 ** -52 * (1 + X[i] ** 2) * f(X[i])
    # K_i comes from the extended-precision X: within one unit of the value
    # from the double X_i
    for i in range(n):
        k = mp.ceil(mp.ldexp(X[i + 1] / X[i], 52))
        assert abs(mp.ldexp(mp.mpf(float(t["xd"][i, 1])) - 1, 52) - k) <= 1


def test_fast_acceptance_rate():
    """The fraction of draws the fast path accepts is the mean of
    X_{i+1}/X_i over the layers (99.77 % for 2048 layers); 1e6 restated first
    draws agree within 4 standard errors."""
    from philox_ref import philox_words
    t = normal_tables()
    X = np.append(t["xd"][:, 0], 0.0)
    p = float(np.mean(X[1:] / X[:-1]))
    assert 0.9975 < p < 0.998
    w0, w1, w2, w3 = philox_words(99, 4, np.arange(500_000, dtype=np.uint64))
    ok = np.concatenate([zig_fast(w1, w0, t)[1], zig_fast(w3, w2, t)[1]])
    n = ok.size
    assert abs(ok.sum() - n * p) <= 4 * math.sqrt(n * p * (1 - p))


def test_tail_sampler_is_the_conditional_normal_tail():
    """Draws of the base layer beyond r go to Marsaglia's tail method: 2e5 of
    them (distinct pairs) follow P(|x| > s | |x| > r) = erfc(s/√2)/erfc(r/√2)
    (KS at the 1 % level), with the draw's sign."""
    from scipy.special import erfc
    t = normal_tables()
    n = 200_000
    hi = np.full(n, 0x000FFFFF, np.uint64)          # layer 0, positive, fraction near 1
    lo = np.full(n, 0xFFFFFFFF, np.uint64)
    assert not np.any(zig_fast(hi, lo, t)[1])
    x = zig_slow(17, 3, np.arange(n, dtype=np.uint64), 0, hi, lo, t)
    assert np.all(x > t["r"])
    xs = np.sort(x)
    r = t["r"]
    cdf = 1.0 - erfc(xs / math.sqrt(2.0)) / erfc(r / math.sqrt(2.0))
    d = max(np.max(np.arange(1, n + 1) / n - cdf), np.max(cdf - np.arange(n) / n))
    assert d < 1.63 / math.sqrt(n)
    neg = zig_slow(17, 3, np.arange(8, dtype=np.uint64), 1, hi[:8] | np.uint64(1 << 20),
                   lo[:8], t)
    assert np.all(neg < -t["r"])


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
