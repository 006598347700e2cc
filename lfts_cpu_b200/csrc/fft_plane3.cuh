// Three-stage yz-plane kernels (FP32-mixed path): 64 x 64, 96 x 96, 128 x 128.
//
// Same job and spectrum layout as plane_c_kernel (fft_packed.cuh): one CTA per
// x-plane carries the packed field Z = q + i q^ through the inverse 2-D
// transform, the h multiply and propagator stores, and the forward transform.
// The 2-D transform is split so that a whole plane crosses shared memory four
// times per contour step instead of six (shared-memory bandwidth bounds the
// two-stage-per-axis kernel at these sizes):
//
//   y: NY = Y1 x Y2   ky = j2 + Y2 a,  y = k1 + Y1 k2
//   z: NZ = Z1 x Z2   kz = jz + Z2 b,  z = c1 + Z1 c2
//
//   inverse:  S1  DFT-Y1 over a       (task: column kz, j2)          global -> smem
//             S2  twiddle w^(j2 k1), DFT-Y2 over j2 (-> y rows), then
//                 DFT-Z1 over b, twiddle w^(jz c1)  (task: k1, jz; a Y2 x Z1 block)
//             S3  DFT-Z2 over jz (-> z = c1 + Z1 c2), x h, store q   (task: y, c1)
//   forward:  S3  DFT-Z2 over c2 on the same registers
//             S2  twiddle w^-(jz c1), DFT-Z1 over c1, DFT-Y2 over k2, twiddle w^-(j2 k1)
//             S1  DFT-Y1 over k1                                        smem -> global
//
// Shared-memory rows hold (after S1) T[j2][k1] at row k1 + Y1 j2, and (after
// S2) natural y; columns are at pos(p) = p + 2 (p / Z2) with p = kz (S1) or
// jz + Z2 c1 (S2, S3), so every stage is in place.  Z2 = 16: an S1 / S2
// half-warp reads 16 consecutive slots of one row, and each S3 task's 16
// values are one 16-byte-aligned run (moved with 16-byte accesses); the row
// pitch KP is the one for which every access pattern is conflict-free
// (checked by a bank model of the three stages' lane mappings).
#pragma once
#include "fft_packed.cuh"

namespace lfts {

template <int NY_, int NZ_, int Y1_, int Z1_, int NT_, int KP_>
struct Plane3Cfg {
    static constexpr int NY = NY_, NZ = NZ_, Y1 = Y1_, Y2 = NY_ / Y1_, Z1 = Z1_, Z2 = NZ_ / Z1_;
    static constexpr int NT = NT_, KP = KP_;
    static constexpr int NS1 = NZ * Y2, NS2 = Y1 * Z2, NS3 = NY * Z1;  // tasks per stage
    // TY[j2 * Y1 + k1] = w^(j2 k1) (NY entries), TZ[c1 * Z2 + jz] = w^(jz c1) (NZ entries)
    static constexpr size_t TOFF = sizeof(cpx<float>) * (size_t)(NY * KP);
    // ... followed by gz[NZ] (PLANE_G)
    static constexpr size_t SMEM = TOFF + sizeof(cpx<float>) * (NY + NZ) + sizeof(float) * NZ;
    static __host__ __device__ constexpr int pos(int p) { return p + 2 * (p / Z2); }
    static_assert(Z2 == 16, "S3 runs of 16 values");
    static_assert(NS1 <= NT && NS2 <= NT && NY + 2 * NZ <= NT, "at most one S1 / S2 task (table entry) per thread");
    static_assert(pos(NZ - 1) < KP && KP % 2 == 0, "row pitch");
};

// the instances: 128 = (32 x 4, 8 x 16), 96 = (32 x 3, 6 x 16), 64 = (16 x 4, 4 x 16)
using Plane3_128 = Plane3Cfg<128, 128, 32, 8, 512, 142>;
using Plane3_96 = Plane3Cfg<96, 96, 32, 6, 512, 108>;
using Plane3_64 = Plane3Cfg<64, 64, 16, 4, 256, 72>;

// the 16 values of an S3 task: a run of 16 slots, 16-byte aligned
__device__ __forceinline__ void p3_ld16(const cpx<float> *run, cpx<float> (&g)[16])
{
#pragma unroll
    for (int m = 0; m < 8; m++) {
        const float4 v = reinterpret_cast<const float4 *>(run)[m];
        g[2 * m] = {v.x, v.y};
        g[2 * m + 1] = {v.z, v.w};
    }
}
__device__ __forceinline__ void p3_st16(cpx<float> *run, const cpx<float> (&g)[16])
{
#pragma unroll
    for (int m = 0; m < 8; m++)
        reinterpret_cast<float4 *>(run)[m] = make_float4(g[2 * m].x, g[2 * m].y, g[2 * m + 1].x, g[2 * m + 1].y);
}

// S1 inverse: one (kz, j2) task per thread, Y1 strided rows from the global spectrum
template <typename C>
__device__ __forceinline__ void p3_s1_inv(cpx<float> *P, const cpx<float> *__restrict__ Sg)
{
    const int t = threadIdx.x;
    if (t >= C::NS1) return;
    const int kz = t % C::NZ, j2 = t / C::NZ;
    cpx<float> v[C::Y1];
#pragma unroll
    for (int a = 0; a < C::Y1; a++) v[a] = Sg[(j2 + C::Y2 * a) * C::NZ + kz];
    Dft<C::Y1, 1, float>::run(v);
    const int pc = C::pos(kz);
#pragma unroll
    for (int k1 = 0; k1 < C::Y1; k1++) P[(k1 + C::Y1 * j2) * C::KP + pc] = v[k1];
}

// S1 forward: DFT-Y1 over k1 of rows k1 + Y1 j2, to global rows ky = j2 + Y2 a
template <typename C>
__device__ __forceinline__ void p3_s1_fwd(const cpx<float> *P, cpx<float> *__restrict__ Sg)
{
    const int t = threadIdx.x;
    if (t >= C::NS1) return;
    const int kz = t % C::NZ, j2 = t / C::NZ;
    const int pc = C::pos(kz);
    cpx<float> v[C::Y1];
#pragma unroll
    for (int k1 = 0; k1 < C::Y1; k1++) v[k1] = P[(k1 + C::Y1 * j2) * C::KP + pc];
    Dft<C::Y1, -1, float>::run(v);
#pragma unroll
    for (int a = 0; a < C::Y1; a++) Sg[(j2 + C::Y2 * a) * C::NZ + kz] = v[a];
}

template <typename C>
__device__ __forceinline__ void p3_s2_inv(cpx<float> *P, const cpx<float> *TY, const cpx<float> *TZ)
{
    const int t = threadIdx.x;
    if (t >= C::NS2) return;
    const int jz = t % C::Z2, k1 = t / C::Z2;  // half-warps share k1, lanes run over jz
    cpx<float> d[C::Y2][C::Z1];
#pragma unroll
    for (int j2 = 0; j2 < C::Y2; j2++)
#pragma unroll
        for (int b = 0; b < C::Z1; b++) d[j2][b] = P[(k1 + C::Y1 * j2) * C::KP + C::pos(jz + C::Z2 * b)];
#pragma unroll
    for (int j2 = 1; j2 < C::Y2; j2++) {
        const cpx<float> tw = TY[j2 * C::Y1 + k1];
#pragma unroll
        for (int b = 0; b < C::Z1; b++) d[j2][b] = ctw<1>(d[j2][b], tw);
    }
#pragma unroll
    for (int b = 0; b < C::Z1; b++) {
        cpx<float> u[C::Y2];
#pragma unroll
        for (int j2 = 0; j2 < C::Y2; j2++) u[j2] = d[j2][b];
        Dft<C::Y2, 1, float>::run(u);
#pragma unroll
        for (int k2 = 0; k2 < C::Y2; k2++) d[k2][b] = u[k2];
    }
#pragma unroll
    for (int k2 = 0; k2 < C::Y2; k2++) Dft<C::Z1, 1, float>::run(d[k2]);
#pragma unroll
    for (int c1 = 1; c1 < C::Z1; c1++) {
        const cpx<float> tw = TZ[c1 * C::Z2 + jz];
#pragma unroll
        for (int k2 = 0; k2 < C::Y2; k2++) d[k2][c1] = ctw<1>(d[k2][c1], tw);
    }
#pragma unroll
    for (int k2 = 0; k2 < C::Y2; k2++)
#pragma unroll
        for (int c1 = 0; c1 < C::Z1; c1++) P[(k1 + C::Y1 * k2) * C::KP + C::pos(jz + C::Z2 * c1)] = d[k2][c1];
}

template <typename C>
__device__ __forceinline__ void p3_s2_fwd(cpx<float> *P, const cpx<float> *TY, const cpx<float> *TZ)
{
    const int t = threadIdx.x;
    if (t >= C::NS2) return;
    const int jz = t % C::Z2, k1 = t / C::Z2;
    cpx<float> d[C::Y2][C::Z1];
#pragma unroll
    for (int k2 = 0; k2 < C::Y2; k2++)
#pragma unroll
        for (int c1 = 0; c1 < C::Z1; c1++) d[k2][c1] = P[(k1 + C::Y1 * k2) * C::KP + C::pos(jz + C::Z2 * c1)];
#pragma unroll
    for (int c1 = 1; c1 < C::Z1; c1++) {
        const cpx<float> tw = TZ[c1 * C::Z2 + jz];
#pragma unroll
        for (int k2 = 0; k2 < C::Y2; k2++) d[k2][c1] = ctw<-1>(d[k2][c1], tw);
    }
#pragma unroll
    for (int k2 = 0; k2 < C::Y2; k2++) Dft<C::Z1, -1, float>::run(d[k2]);
#pragma unroll
    for (int b = 0; b < C::Z1; b++) {
        cpx<float> u[C::Y2];
#pragma unroll
        for (int k2 = 0; k2 < C::Y2; k2++) u[k2] = d[k2][b];
        Dft<C::Y2, -1, float>::run(u);
#pragma unroll
        for (int j2 = 0; j2 < C::Y2; j2++) d[j2][b] = u[j2];
    }
#pragma unroll
    for (int j2 = 1; j2 < C::Y2; j2++) {
        const cpx<float> tw = TY[j2 * C::Y1 + k1];
#pragma unroll
        for (int b = 0; b < C::Z1; b++) d[j2][b] = ctw<-1>(d[j2][b], tw);
    }
#pragma unroll
    for (int j2 = 0; j2 < C::Y2; j2++)
#pragma unroll
        for (int b = 0; b < C::Z1; b++) P[(k1 + C::Y1 * j2) * C::KP + C::pos(jz + C::Z2 * b)] = d[j2][b];
}

// S3 tasks: (y, c1) = (u / Z1, u % Z1) for u = threadIdx.x + NT s, s < ROUNDS
// MODE PLANE_G multiplies by the Boltzmann weight g = gx[x] (gy[y] gz[z]) of
// plane x instead of h and stores nothing (the h-in-pencil chain)
template <typename C, int MODE>
__device__ __forceinline__ void p3_s3(cpx<float> *P, const PlaneArgs<float> &a, long long plane_off, double &qsum,
                                      int x, const float *GZ)
{
    constexpr int NZ = C::NZ, Z1 = C::Z1, Z2 = C::Z2;
    // stored propagators and h as (chain 1, chain 2) pairs (fft_packed.cuh)
    const cpx<float> *__restrict__ hp = reinterpret_cast<const cpx<float> *>(a.h) + plane_off;
    cpx<float> *__restrict__ qp = reinterpret_cast<cpx<float> *>(a.qout) + plane_off;
    const int hs0 = a.hsel0, hs1 = a.hsel1;
    constexpr int ROUNDS = (C::NS3 + C::NT - 1) / C::NT;
#pragma unroll 1
    for (int s = 0; s < ROUNDS; s++) {
        const int u = threadIdx.x + C::NT * s;
        if (C::NS3 % C::NT != 0 && u >= C::NS3) break;
        const int y = u / Z1, c1 = u % Z1;
        cpx<float> *row = P + y * C::KP;
        float ha[Z2], hb[Z2];
        if (MODE == PLANE_G) {
            const float gx = __ldg(a.gx + x), gy = __ldg(a.gy + y);
#pragma unroll
            for (int c2 = 0; c2 < Z2; c2++) ha[c2] = hb[c2] = gx * (gy * GZ[c1 + Z1 * c2]);
        } else {
#pragma unroll
            for (int c2 = 0; c2 < Z2; c2++) {
                const cpx<float> h = ld_pair(hp + y * NZ + c1 + Z1 * c2);
                ha[c2] = hs0 ? h.y : h.x;
                hb[c2] = hs1 ? h.y : h.x;
            }
        }
        cpx<float> g[Z2];
        p3_ld16(row + C::pos(Z2 * c1), g);
        Dft<Z2, 1, float>::run(g);
#pragma unroll
        for (int c2 = 0; c2 < Z2; c2++) {
            const int z = c1 + Z1 * c2;
            const float va = g[c2].x * ha[c2];
            const float vb = g[c2].y * hb[c2];
            if (MODE != PLANE_G) st_pair(qp + y * NZ + z, va, vb);
            if (MODE == PLANE_LAST) qsum += (double)va;
            g[c2] = {va, vb};
        }
        if (MODE == PLANE_STEP || MODE == PLANE_G) {
            Dft<Z2, -1, float>::run(g);
            p3_st16(row + C::pos(Z2 * c1), g);
        }
    }
}

// INIT: real rows from global (h from the fields, or given rows), forward S3
template <typename C, int MODE>
__device__ __forceinline__ void p3_s3_init(cpx<float> *P, const PlaneArgs<float> &a, long long plane_off, long long M)
{
    constexpr int NZ = C::NZ, Z1 = C::Z1, Z2 = C::Z2;
    constexpr int ROUNDS = (C::NS3 + C::NT - 1) / C::NT;
#pragma unroll 1
    for (int s = 0; s < ROUNDS; s++) {
        const int u = threadIdx.x + C::NT * s;
        if (C::NS3 % C::NT != 0 && u >= C::NS3) break;
        const int y = u / Z1, c1 = u % Z1;
        cpx<float> g[Z2];
#pragma unroll
        for (int c2 = 0; c2 < Z2; c2++) {
            const long long i = plane_off + y * NZ + c1 + Z1 * c2;
            float v1, v2;
            if (MODE == PLANE_INIT_W) {
                // hA = exp(-(W- + w+)/N), hB = exp(-(-W- + w+)/N)  (src/diblock.cc:64-72)
                // (single-precision exponential: h is stored in FP32)
                const double wm = a.w[i], wp = a.w[M + i];
                v1 = expf((float)(-(wm + wp) / a.Nd));
                v2 = expf((float)(-(-wm + wp) / a.Nd));
                reinterpret_cast<cpx<float> *>(a.qout)[i] = {v1, v2};
            } else if (a.src) {
                v1 = a.src[i];
                v2 = a.src[a.src_stride + i];
            } else {
                v1 = (float)a.src64[i];
                v2 = (float)a.src64[a.src_stride + i];
            }
            g[c2] = {v1, v2};
        }
        Dft<Z2, -1, float>::run(g);
        p3_st16(P + y * C::KP + C::pos(Z2 * c1), g);
    }
}

// body of one CTA: x-plane x of an mx-plane field (the ensemble's batched
// launches call it with their own plane numbering)
template <typename C, int MODE>
__device__ __forceinline__ void plane3_body(const PlaneArgs<float> &a, const int x, const int mx)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<float> *P = reinterpret_cast<cpx<float> *>(smem_raw);
    cpx<float> *TY = reinterpret_cast<cpx<float> *>(smem_raw + C::TOFF);
    cpx<float> *TZ = TY + C::NY;
    float *GZ = reinterpret_cast<float *>(TZ + C::NZ);

    const long long M = (long long)mx * C::NY * C::NZ;
    const long long plane_off = (long long)x * C::NY * C::NZ;
    cpx<float> *Sg = a.spec + plane_off;

    // constant tables (never written by the chain): before the grid dependency
    if (threadIdx.x < C::NY) {
        const int j2 = threadIdx.x / C::Y1, k1 = threadIdx.x % C::Y1;
        TY[threadIdx.x] = a.twy[(j2 * k1) % C::NY];
    } else if (threadIdx.x < C::NY + C::NZ) {
        const int t = threadIdx.x - C::NY, c1 = t / C::Z2, jz = t % C::Z2;
        TZ[t] = a.twz[(jz * c1) % C::NZ];
    } else if (MODE == PLANE_G && threadIdx.x < C::NY + 2 * C::NZ) {
        GZ[threadIdx.x - C::NY - C::NZ] = a.gz[threadIdx.x - C::NY - C::NZ];
    }
    // The summing x-pencil after this launch reads a stored slot written many
    // steps earlier, long gone from L2; this plane's share of it (plane x, one
    // float pair per point) is fetched into L2 while the transforms run.
    if (MODE == PLANE_G && a.pf && a.pf_ctas == 0) {
        const char *base = reinterpret_cast<const char *>(a.pf + 2 * plane_off);
        constexpr int BYTES = 2 * C::NY * C::NZ * (int)sizeof(float);
        for (int o = 128 * threadIdx.x; o < BYTES; o += 128 * C::NT) prefetch_l2(base + o);
    }
    pdl_launch_dependents();
    pdl_wait();

    if (MODE == PLANE_INIT_W || MODE == PLANE_INIT_Q) {
        p3_s3_init<C, MODE>(P, a, plane_off, M);
        __syncthreads();
        p3_s2_fwd<C>(P, TY, TZ);
        __syncthreads();
        p3_s1_fwd<C>(P, Sg);
        return;
    }

    p3_s1_inv<C>(P, Sg);
    __syncthreads();
    p3_s2_inv<C>(P, TY, TZ);
    __syncthreads();
    double qsum = 0.0;
    p3_s3<C, MODE>(P, a, plane_off, qsum, x, GZ);
    if (MODE == PLANE_LAST) {
        __shared__ double red[C::NT / 32];
        for (int o = 16; o > 0; o >>= 1) qsum += __shfl_xor_sync(0xffffffffu, qsum, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = qsum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int i = 0; i < C::NT / 32; i++) s += red[i];
            a.qpart[x] = s;
        }
        return;
    }
    __syncthreads();
    p3_s2_fwd<C>(P, TY, TZ);
    __syncthreads();
    p3_s1_fwd<C>(P, Sg);
}

// A PLANE_G launch ahead of a summing x-pencil can carry pf_ctas CTAs past
// the mx planes: they run on SMs the planes leave idle (128 planes, 148 SMs)
// and pull the whole partner slot into L2 there, instead of each plane CTA
// issuing its own plane's share between its transforms.
template <typename C>
__device__ __forceinline__ void p3_prefetch_tail(const PlaneArgs<float> &a, const int j, const int nj, const int mx)
{
    const char *base = reinterpret_cast<const char *>(a.pf);
    const long long bytes = 2LL * mx * C::NY * C::NZ * (long long)sizeof(float);
    const long long per = (bytes / nj + 127) / 128 * 128;
    const long long lo = (long long)j * per;
    const long long hi = lo + per < bytes ? lo + per : bytes;
    for (long long o = lo + 128LL * threadIdx.x; o < hi; o += 128LL * C::NT) prefetch_l2(base + o);
}

template <typename C, int MODE>
__global__ void __launch_bounds__(C::NT, 1) plane3_kernel(PlaneArgs<float> a)
{
    if (MODE == PLANE_G && a.pf_ctas > 0) {
        const int mx = (int)gridDim.x - a.pf_ctas;
        if ((int)blockIdx.x >= mx) {
            if (a.pf) p3_prefetch_tail<C>(a, (int)blockIdx.x - mx, a.pf_ctas, mx);
            return;
        }
        plane3_body<C, MODE>(a, blockIdx.x, mx);
        return;
    }
    plane3_body<C, MODE>(a, blockIdx.x, gridDim.x);
}

}  // namespace lfts
