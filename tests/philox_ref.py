"""numpy restatement of the device random numbers (test infrastructure):
Philox-4x32-10 (Salmon et al., SC'11) keyed by (seed_lo, seed_hi) over the
counter (q_lo, q_hi, turn_lo, turn_hi), q = particle // 4, followed by the
Box-Muller transform of haissinskijulia_b200/csrc/hj_device.cuh (evaluated
here in double precision; the device evaluates it in single precision)."""
import numpy as np

_M = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint64) & _M for x in (c0, c1, c2, c3))
    k0 = np.uint64(k0) & _M
    k1 = np.uint64(k1) & _M
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c0
        p1 = np.uint64(0xCD9E8D57) * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _M
        hi1, lo1 = p1 >> np.uint64(32), p1 & _M
        c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
        k0 = (k0 + np.uint64(0x9E3779B9)) & _M
        k1 = (k1 + np.uint64(0xBB67AE85)) & _M
    return c0, c1, c2, c3


def philox_normals_reference(seed: int, turn: int, n: int) -> np.ndarray:
    nq = (n + 3) // 4
    q = np.arange(nq, dtype=np.uint64)
    x0, x1, x2, x3 = philox4x32_10(q & _M, q >> np.uint64(32),
                                   np.full(nq, turn & 0xFFFFFFFF, np.uint64),
                                   np.full(nq, (turn >> 32) & 0xFFFFFFFF, np.uint64),
                                   seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    s = np.float32(2.0 ** -32)
    h = np.float32(2.0 ** -33)
    u1 = x0.astype(np.float32) * s + h
    u3 = x2.astype(np.float32) * s + h
    ta = 2.0 * np.pi * (x1.astype(np.float64) * 2.0 ** -32 - 0.5)
    tb = 2.0 * np.pi * (x3.astype(np.float64) * 2.0 ** -32 - 0.5)
    ra = np.sqrt(-2.0 * np.log(u1.astype(np.float64)))
    rb = np.sqrt(-2.0 * np.log(u3.astype(np.float64)))
    out = np.empty((nq, 4))
    out[:, 0] = ra * np.cos(ta)
    out[:, 1] = ra * np.sin(ta)
    out[:, 2] = rb * np.cos(tb)
    out[:, 3] = rb * np.sin(tb)
    return out.reshape(-1)[:n]
