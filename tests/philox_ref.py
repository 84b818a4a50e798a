"""numpy restatement of the device random numbers (test infrastructure):
Philox-4x32-10 (Salmon et al., SC'11) with the 64-bit seed as its key and the
counter (p mod 2^32, p >> 32, turn mod 2^32, turn >> 32) for the particle
pair p = i // 2, followed by the Box-Muller transform of
haissinskijulia_b200/csrc/hj_device.cuh (u1 = (2a + 1) 2^-53 and w = b 2^-52
from the top 52 bits of the word pairs, normals sqrt(-2 ln u1)(cos 2πw,
sin 2πw)) with numpy's log, cos and sin."""
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


def philox_words(seed: int, turn: int, pairs: np.ndarray):
    p = np.asarray(pairs, dtype=np.uint64)
    t = np.uint64(turn & 0xFFFFFFFFFFFFFFFF)
    ctr = (p & _M, p >> np.uint64(32), np.full_like(p, t & _M), np.full_like(p, t >> np.uint64(32)))
    return philox4x32_10(ctr, (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF))


def normal_tables() -> dict:
    """The transform's tables as the library builds them (hj_normal_tables,
    host only)."""
    from haissinskijulia_b200 import _lib
    out = np.zeros(516)
    rc = _lib.load().hj_normal_tables(out.ctypes.data_as(_lib.POINTER(_lib.c_double)), 516)
    assert rc == 0
    return {"lr": out[0:256].reshape(128, 2), "sc": out[256:512].reshape(128, 2),
            "ln2_hi": out[512], "ln2_lo": out[513], "twopi_hi": out[514], "twopi_lo": out[515]}


def uniforms(x0, x1, x2, x3):
    """(u1, w) of the transform exactly as the device forms them:
    u1 = (2a + 1) 2^-53, w = b 2^-52, a and b the top 52 bits of (x1:x0) and
    (x3:x2)."""
    a = ((x1 << np.uint64(32)) | x0) >> np.uint64(12)
    b = ((x3 << np.uint64(32)) | x2) >> np.uint64(12)
    u1 = a.astype(np.float64) * 2.0 ** -52 + 2.0 ** -53
    w = b.astype(np.float64) * 2.0 ** -52
    return u1, w


def philox_normals_reference(seed: int, turn: int, n: int, first_pair: int = 0) -> np.ndarray:
    """n normals of the pairs first_pair, first_pair + 1, ... (two per pair):
    sqrt(-2 ln u1) (cos 2πw, sin 2πw) with numpy's log, cos and sin."""
    npairs = (n + 1) // 2
    p = np.arange(first_pair, first_pair + npairs, dtype=np.uint64)
    u1, w = uniforms(*philox_words(seed, turn, p))
    rad = np.sqrt(-2.0 * np.log(u1))
    out = np.empty((npairs, 2))
    out[:, 0] = rad * np.cos(2.0 * np.pi * w)
    out[:, 1] = rad * np.sin(2.0 * np.pi * w)
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
