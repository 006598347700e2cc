"""TEST INFRASTRUCTURE ONLY -- restatement of the ensemble's noise generator.

Philox4x32-10 as published by Salmon, Moraes, Dror and Shaw ("Parallel random
numbers: as easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64-bit
multiplications (0xD2511F53, 0xCD9E8D57) with Weyl key bumps (0x9E3779B9,
0xBB67AE85); and the Box-Muller map used for the ensemble's Langevin noise:
counter = (p, p>>32, s, s>>32) for pair p = i/2 of step s, key = (seed,
seed>>32); 53-bit uniforms u1, u2 from output words (0,1) and (2,3);
z0, z1 = sqrt(-2 ln(1-u1)) (cos, sin)(2 pi u2); point 2p gets z0, 2p+1 gets z1.
The reference has no such generator (it uses std::mt19937_64 on the host);
this restates the published algorithm so the GPU's stream can be checked.
"""
from __future__ import annotations

import numpy as np

_M32 = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised over numpy uint64 arrays holding 32-bit values."""
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint64) for x in (c0, c1, c2, c3))
    k0 = np.uint64(k0)
    k1 = np.uint64(k1)
    for r in range(10):
        if r:
            k0 = (k0 + np.uint64(0x9E3779B9)) & _M32
            k1 = (k1 + np.uint64(0xBB67AE85)) & _M32
        p0 = np.uint64(0xD2511F53) * c0
        p1 = np.uint64(0xCD9E8D57) * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _M32
        hi1, lo1 = p1 >> np.uint64(32), p1 & _M32
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0), lo1, (hi0 ^ c3 ^ k1), lo0
    return c0, c1, c2, c3


def uniforms(seed: int, step: int, n_pairs: int):
    p = np.arange(n_pairs, dtype=np.uint64)
    s = np.uint64(step)
    o0, o1, o2, o3 = philox4x32_10(p & _M32, p >> np.uint64(32), np.full(n_pairs, s & _M32),
                                   np.full(n_pairs, s >> np.uint64(32)), seed & 0xFFFFFFFF, seed >> 32)
    u1 = ((o0 >> np.uint64(5)).astype(np.float64) * 67108864.0 + (o1 >> np.uint64(6)).astype(np.float64)) / 2.0**53
    u2 = ((o2 >> np.uint64(5)).astype(np.float64) * 67108864.0 + (o3 >> np.uint64(6)).astype(np.float64)) / 2.0**53
    return u1, u2


def noise(seed: int, step: int, n: int, sigma: float) -> np.ndarray:
    """sigma * z for points 0..n-1 of step `step`."""
    u1, u2 = uniforms(seed, step, (n + 1) // 2)
    r = np.sqrt(-2.0 * np.log(1.0 - u1))
    z = np.empty(2 * len(u1))
    z[0::2] = r * np.cos(np.pi * (2.0 * u2))
    z[1::2] = r * np.sin(np.pi * (2.0 * u2))
    return sigma * z[:n]
