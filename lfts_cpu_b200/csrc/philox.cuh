// Counter-based Gaussian noise for the ensemble's Langevin steps.
//
// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): a 4 x 32-bit counter and a 2 x 32-bit key through
// ten rounds of two 32x32->64 multiplications (multipliers 0xD2511F53 and
// 0xCD9E8D57) with Weyl-sequence key bumps (0x9E3779B9, 0xBB67AE85).  The
// deviate for mesh point i of Langevin step s of a replica with stream seed
// `seed` is a function of (seed, s, i) alone, so no noise is stored: a step
// regenerates the previous step's deviates instead of keeping them.
//
//   counter = (p, p >> 32, s, s >> 32) with p = i / 2, key = (seed, seed >> 32)
//   u1, u2  = 53-bit uniforms in [0, 1) from output words (0, 1) and (2, 3)
//   z0, z1  = sqrt(-2 ln(1 - u1)) (cos, sin)(2 pi u2)        (Box-Muller)
//   point 2p gets z0, point 2p + 1 gets z1; the noise is sigma * z.
#pragma once
#include <cstdint>

namespace lfts {

struct Philox4 {
    uint32_t x[4];
};

__host__ __device__ inline void mulhilo32(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo)
{
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

__host__ __device__ inline Philox4 philox4x32_10(Philox4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c.x[0], hi0, lo0);
        mulhilo32(0xCD9E8D57u, c.x[2], hi1, lo1);
        Philox4 n;
        n.x[0] = hi1 ^ c.x[1] ^ k0;
        n.x[1] = lo1;
        n.x[2] = hi0 ^ c.x[3] ^ k1;
        n.x[3] = lo0;
        c = n;
    }
    return c;
}

// the two N(0,1) deviates of pair p (mesh points 2p, 2p + 1) of step s
__device__ inline void philox_normal2(unsigned long long seed, long long s, long long p, double &z0, double &z1)
{
    Philox4 c;
    c.x[0] = (uint32_t)(unsigned long long)p;
    c.x[1] = (uint32_t)((unsigned long long)p >> 32);
    c.x[2] = (uint32_t)(unsigned long long)s;
    c.x[3] = (uint32_t)((unsigned long long)s >> 32);
    const Philox4 o = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    // exact: integers below 2^53 and power-of-two scalings
    const double u1 = ((double)(o.x[0] >> 5) * 67108864.0 + (double)(o.x[1] >> 6)) * (1.0 / 9007199254740992.0);
    const double u2 = ((double)(o.x[2] >> 5) * 67108864.0 + (double)(o.x[3] >> 6)) * (1.0 / 9007199254740992.0);
    const double r = sqrt(-2.0 * log(1.0 - u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    z0 = __dmul_rn(r, cs);
    z1 = __dmul_rn(r, sn);
}

// sigma * z of mesh point i
__device__ inline double philox_noise(unsigned long long seed, long long s, long long i, double sigma)
{
    double z0, z1;
    philox_normal2(seed, s, i >> 1, z0, z1);
    return __dmul_rn(sigma, (i & 1) ? z1 : z0);
}

}  // namespace lfts
