"""numpy restatement of the device random numbers (test infrastructure):
Philox-2x32-10 (Salmon et al., SC'11) with key = seed folded to 32 bits
(seed ^ seed >> 32) and counter (p mod 2^32, (turn mod 2^24) | (p >> 32) << 24)
for the particle pair p = i // 2, followed by the Box-Muller transform of
haissinskijulia_b200/csrc/hj_device.cuh (evaluated here in double precision;
the device evaluates it in single precision)."""
import numpy as np

_M = np.uint64(0xFFFFFFFF)


def philox2x32_10(c0, c1, k):
    c0, c1 = (np.asarray(x, dtype=np.uint64) & _M for x in (c0, c1))
    k = np.uint64(k) & _M
    for _ in range(10):
        pr = np.uint64(0xD256D193) * c0
        hi, lo = pr >> np.uint64(32), pr & _M
        c0, c1 = hi ^ k ^ c1, lo
        k = (k + np.uint64(0x9E3779B9)) & _M
    return c0, c1


def philox_normals_reference(seed: int, turn: int, n: int, first_pair: int = 0) -> np.ndarray:
    """n normals of the pairs first_pair, first_pair + 1, ... (two per pair)."""
    npairs = (n + 1) // 2
    p = np.arange(first_pair, first_pair + npairs, dtype=np.uint64)
    key = (seed ^ (seed >> 32)) & 0xFFFFFFFF
    c1 = (np.uint64(turn & 0xFFFFFF) | ((p >> np.uint64(32)) << np.uint64(24))) & _M
    x0, x1 = philox2x32_10(p & _M, c1, key)
    u1 = x0.astype(np.float32) * np.float32(2.0 ** -32) + np.float32(2.0 ** -33)
    th = 2.0 * np.pi * (x1.astype(np.float64) * 2.0 ** -32 - 0.5)
    rad = np.sqrt(-2.0 * np.log(u1.astype(np.float64)))
    out = np.empty((npairs, 2))
    out[:, 0] = rad * np.cos(th)
    out[:, 1] = rad * np.sin(th)
    return out.reshape(-1)[:n]
