"""numpy restatement of the device random numbers (test infrastructure):
Philox-4x32-10 (Salmon et al., SC'11) with the 64-bit seed as its key and the
counter (p mod 2^32, p >> 32, turn mod 2^32, turn >> 32) for the particle
pair p = i // 2, whose words 1:0 and 3:2 make the two normals of the pair by
the 2048-layer ziggurat of haissinskijulia_b200/csrc/hj_device.cuh (Marsaglia
and Tsang, J. Stat. Softw. 5(8), 2000): layer = hi >> 21, sign = bit 20 of
hi, fraction m = (hi mod 2^20):lo; fast acceptance when 1 + m 2^-52 < D_i,
else the slow path with the retry words of attempt a (counter word 3 =
(turn >> 32) | (2a - 1 + h) << 24), numpy's exp and log standing in for the
device's."""
import numpy as np

_M = np.uint64(0xFFFFFFFF)


def philox4x32_10(c, key):
    """Philox-4x32-10 of counters c = (c0, c1, c2, c3) (arrays) under a
    64-bit key given as (k0, k1)."""
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint64) & _M for x in c)
    k0, k1 = (np.uint64(int(x) & 0xFFFFFFFF) for x in key)
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c0
        p1 = np.uint64(0xCD9E8D57) * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _M
        hi1, lo1 = p1 >> np.uint64(32), p1 & _M
        c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
        k0 = (k0 + np.uint64(0x9E3779B9)) & _M
        k1 = (k1 + np.uint64(0xBB67AE85)) & _M
    return c0, c1, c2, c3


def philox_words(seed: int, turn: int, pairs: np.ndarray, word3_tag=None):
    """The four Philox words of pairs `pairs` at `turn`; word3_tag (an array
    or int) is OR-ed into counter word 3 (the slow path's retry draws)."""
    p = np.asarray(pairs, dtype=np.uint64)
    t = np.uint64(turn & 0xFFFFFFFFFFFFFFFF)
    c3 = np.full_like(p, t >> np.uint64(32))
    if word3_tag is not None:
        c3 = c3 | np.asarray(word3_tag, dtype=np.uint64)
    ctr = (p & _M, p >> np.uint64(32), np.full_like(p, t & _M), c3)
    return philox4x32_10(ctr, (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF))


LAYERS = 2048


def normal_tables() -> dict:
    """The ziggurat's tables as the library builds them (hj_normal_tables,
    host only): rows (X_i, D_i), f(X_i) for i = 0..2048, r = X_1 and the
    layers' area v."""
    from haissinskijulia_b200 import _lib
    size = 3 * LAYERS + 3
    out = np.zeros(size)
    rc = _lib.load().hj_normal_tables(out.ctypes.data_as(_lib.POINTER(_lib.c_double)), size)
    assert rc == 0
    return {"xd": out[0:2 * LAYERS].reshape(LAYERS, 2), "f": out[2 * LAYERS:3 * LAYERS + 1],
            "r": out[3 * LAYERS + 1], "v": out[3 * LAYERS + 2]}


_TABLES = None


def _tables() -> dict:
    global _TABLES
    if _TABLES is None:
        _TABLES = normal_tables()
    return _TABLES


def fraction(hi, lo):
    """The 52-bit fraction (hi mod 2^20):lo of a draw as exact float64."""
    hi = np.asarray(hi, dtype=np.uint64)
    lo = np.asarray(lo, dtype=np.uint64)
    return (((hi & np.uint64(0xFFFFF)) << np.uint64(32)) | lo).astype(np.float64)


def zig_fast(hi, lo, t=None):
    """(x, accepted) of the fast path for draws (hi:lo): x = ±U X_i with one
    rounding, accepted where 1 + U < D_i (U = m 2^-52)."""
    t = t or _tables()
    hi = np.asarray(hi, dtype=np.uint64)
    i = (hi >> np.uint64(21)).astype(np.int64)
    d = 1.0 + fraction(hi, lo) * 2.0 ** -52
    x = (d - 1.0) * t["xd"][i, 0]
    neg = ((hi >> np.uint64(20)) & np.uint64(1)) == 1
    return np.where(neg, -x, x), d < t["xd"][i, 1]


def zig_slow(seed: int, turn: int, pairs, h, hi, lo, t=None) -> np.ndarray:
    """The slow path for the normals of particles 2p + h whose first draws
    (hi:lo) failed the fast test (arrays), attempt by attempt as the device
    runs it."""
    t = t or _tables()
    p = np.asarray(pairs, dtype=np.uint64)
    h = np.broadcast_to(np.asarray(h, dtype=np.uint64), p.shape).copy()
    hi = np.asarray(hi, dtype=np.uint64).copy()
    i = (hi >> np.uint64(21)).astype(np.int64)
    neg = ((hi >> np.uint64(20)) & np.uint64(1)) == 1
    d = 1.0 + fraction(hi, lo) * 2.0 ** -52
    x = np.zeros(p.shape)
    done = np.zeros(p.shape, dtype=bool)
    r = t["r"]
    for a in range(1, 128):
        idx = np.nonzero(~done)[0]
        if idx.size == 0:
            break
        tag = (np.uint64(2 * a - 1) + h[idx]) << np.uint64(24)
        w0, w1, w2, w3 = philox_words(seed, turn, p[idx], tag)
        tail = i[idx] == 0
        ti = idx[tail]
        if ti.size:
            u1 = (fraction(w1[tail], w0[tail]) + 0.5) * 2.0 ** -52
            u2 = (fraction(w3[tail], w2[tail]) + 0.5) * 2.0 ** -52
            ta = -np.log(u1) / r
            tb = -np.log(u2)
            x[ti] = r + ta
            done[ti] = (tb + tb) > ta * ta
        wi = idx[~tail]
        if wi.size:
            iw = i[wi]
            xw = (d[wi] - 1.0) * t["xd"][iw, 0]
            fi, fi1 = t["f"][iw], t["f"][iw + 1]
            u = fraction(w1[~tail], w0[~tail]) * 2.0 ** -52
            y = fi + u * (fi1 - fi)
            acc = y < np.exp((xw * xw) * -0.5)
            x[wi] = xw
            done[wi[acc]] = True
            rej = wi[~acc]
            if rej.size:
                hi2, lo2 = w3[~tail][~acc], w2[~tail][~acc]
                i[rej] = (hi2 >> np.uint64(21)).astype(np.int64)
                neg[rej] = ((hi2 >> np.uint64(20)) & np.uint64(1)) == 1
                d[rej] = 1.0 + fraction(hi2, lo2) * 2.0 ** -52
                x[rej] = (d[rej] - 1.0) * t["xd"][i[rej], 0]
                done[rej] = d[rej] < t["xd"][i[rej], 1]
    return np.where(neg, -x, x)


def philox_normals_reference(seed: int, turn: int, n: int, first_pair: int = 0) -> np.ndarray:
    """n normals of the pairs first_pair, first_pair + 1, ... (two per pair),
    as the device draws them."""
    t = _tables()
    npairs = (n + 1) // 2
    p = np.arange(first_pair, first_pair + npairs, dtype=np.uint64)
    x0, x1, x2, x3 = philox_words(seed, turn, p)
    out = np.empty((npairs, 2))
    for h, (hi, lo) in enumerate(((x1, x0), (x3, x2))):
        x, ok = zig_fast(hi, lo, t)
        bad = np.nonzero(~ok)[0]
        if bad.size:
            x[bad] = zig_slow(seed, turn, p[bad], h, hi[bad], lo[bad], t)
        out[:, h] = x
    return out.reshape(-1)[:n]


def fast_normals_reference(seed: int, turn: int, n: int, first_pair: int = 0) -> np.ndarray:
    """The opt-in single-precision normals of the fused pass (the layouts with
    16 added): Philox words 0 and 1 of the pair, u1 = (x0 + 1/2) 2^-32,
    θ = 2π ((x1 + 1/2) 2^-32 - 1/2), evaluated here in double precision (the
    device evaluates the transform in single precision)."""
    npairs = (n + 1) // 2
    p = np.arange(first_pair, first_pair + npairs, dtype=np.uint64)
    x0, x1, _, _ = philox_words(seed, turn, p)
    u1 = (x0.astype(np.float32) * np.float32(2.0 ** -32) + np.float32(2.0 ** -33)).astype(np.float64)
    th = 2.0 * np.pi * (x1.astype(np.float64) * 2.0 ** -32 - 0.5)
    rad = np.sqrt(-2.0 * np.log(u1))
    out = np.empty((npairs, 2))
    out[:, 0] = rad * np.cos(th)
    out[:, 1] = rad * np.sin(th)
    return out.reshape(-1)[:n]
