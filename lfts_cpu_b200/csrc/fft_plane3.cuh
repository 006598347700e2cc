// Three-stage yz-plane kernel for 128 x 128 planes (FP32-mixed path).
//
// Same job and spectrum layout as plane_c_kernel (fft_packed.cuh): one CTA per
// x-plane carries the packed field Z = q + i q^ through the inverse 2-D
// transform, the h multiply and propagator stores, and the forward transform.
// The 2-D transform is split so that a whole plane crosses shared memory four
// times per contour step instead of six (shared-memory bandwidth bounds the
// two-stage-per-axis kernel at this size):
//
//   y: 128 = 32 x 4   ky = j2 + 4a,  y = k1 + 32 k2
//   z: 128 = 8 x 16   kz = jz + 16b, z = c1 + 8 c2
//
//   inverse:  S1  DFT-32 over a       (task: column kz, j2)        global -> smem
//             S2  twiddle w^(j2 k1), DFT-4 over j2 (-> y rows), then
//                 DFT-8 over b, twiddle w^(jz c1)  (task: k1, jz; a 4 x 8 block)
//             S3  DFT-16 over jz (-> z = c1 + 8 c2), x h, store q   (task: y, c1)
//   forward:  S3  DFT-16 over c2 on the same registers
//             S2  twiddle w^-(jz c1), DFT-8 over c1, DFT-4 over k2, twiddle w^-(j2 k1)
//             S1  DFT-32 over k1                                       smem -> global
//
// Shared-memory rows hold (after S1) T[j2][k1] at row k1 + 32 j2, and (after
// S2) natural y; columns are at pos(p) = p + 2 (p/16) with p = kz (S1) or
// jz + 16 c1 (S2, S3), so every stage is in place.  The two pad slots per 16
// make each S3 task's 16 values one 16-byte-aligned run (read and written with
// 16-byte accesses, conflict-free per quarter-warp); the S1/S2 half-warps read
// 16 consecutive slots of one row.  Row pitch 142 slots.
#pragma once
#include "fft_packed.cuh"

namespace lfts {

struct Plane3Cfg {
    static constexpr int N = 128;
    static constexpr int NT = 512;
    static constexpr int KP = 142;
    // TY[j2 * 32 + k1] = w^(j2 k1), TZ[c1 * 16 + jz] = w^(jz c1), w = exp(-2 pi i/128)
    static constexpr size_t TOFF = sizeof(cpx<float>) * (size_t)(N * KP);
    static constexpr size_t SMEM = TOFF + sizeof(cpx<float>) * 256;
    static __device__ __forceinline__ int pos(int p) { return p + 2 * (p >> 4); }
};

// the 16 values of an S3 task: row[pos(16 c1) .. +15], 16-byte aligned
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

// S1 inverse: one (kz, j2) task per thread, 32 strided rows from the global spectrum
__device__ __forceinline__ void p3_s1_inv(cpx<float> *P, const cpx<float> *__restrict__ Sg)
{
    using C = Plane3Cfg;
    const int kz = threadIdx.x & 127, j2 = threadIdx.x >> 7;
    cpx<float> v[32];
#pragma unroll
    for (int a = 0; a < 32; a++) v[a] = Sg[(j2 + 4 * a) * 128 + kz];
    Dft<32, 1, float>::run(v);
    const int pc = C::pos(kz);
#pragma unroll
    for (int k1 = 0; k1 < 32; k1++) P[(k1 + 32 * j2) * C::KP + pc] = v[k1];
}

// S1 forward: DFT-32 over k1 of rows k1 + 32 j2, to global rows ky = j2 + 4a
__device__ __forceinline__ void p3_s1_fwd(const cpx<float> *P, cpx<float> *__restrict__ Sg)
{
    using C = Plane3Cfg;
    const int kz = threadIdx.x & 127, j2 = threadIdx.x >> 7;
    const int pc = C::pos(kz);
    cpx<float> v[32];
#pragma unroll
    for (int k1 = 0; k1 < 32; k1++) v[k1] = P[(k1 + 32 * j2) * C::KP + pc];
    Dft<32, -1, float>::run(v);
#pragma unroll
    for (int a = 0; a < 32; a++) Sg[(j2 + 4 * a) * 128 + kz] = v[a];
}

// S2 task of this thread: half-warps share k1, lanes of a half run over jz
__device__ __forceinline__ void p3_s2_task(int &k1, int &jz)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    jz = lane & 15;
    k1 = 2 * w + (lane >> 4);
}

__device__ __forceinline__ void p3_s2_inv(cpx<float> *P, const cpx<float> *TY, const cpx<float> *TZ)
{
    using C = Plane3Cfg;
    int k1, jz;
    p3_s2_task(k1, jz);
    cpx<float> d[4][8];
#pragma unroll
    for (int j2 = 0; j2 < 4; j2++)
#pragma unroll
        for (int b = 0; b < 8; b++) d[j2][b] = P[(k1 + 32 * j2) * C::KP + C::pos(jz + 16 * b)];
#pragma unroll
    for (int j2 = 1; j2 < 4; j2++) {
        const cpx<float> tw = TY[j2 * 32 + k1];
#pragma unroll
        for (int b = 0; b < 8; b++) d[j2][b] = ctw<1>(d[j2][b], tw);
    }
#pragma unroll
    for (int b = 0; b < 8; b++) {
        cpx<float> t[4] = {d[0][b], d[1][b], d[2][b], d[3][b]};
        Dft<4, 1, float>::run(t);
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) d[k2][b] = t[k2];
    }
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) Dft<8, 1, float>::run(d[k2]);
#pragma unroll
    for (int c1 = 1; c1 < 8; c1++) {
        const cpx<float> tw = TZ[c1 * 16 + jz];
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) d[k2][c1] = ctw<1>(d[k2][c1], tw);
    }
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++)
#pragma unroll
        for (int c1 = 0; c1 < 8; c1++) P[(k1 + 32 * k2) * C::KP + C::pos(jz + 16 * c1)] = d[k2][c1];
}

__device__ __forceinline__ void p3_s2_fwd(cpx<float> *P, const cpx<float> *TY, const cpx<float> *TZ)
{
    using C = Plane3Cfg;
    int k1, jz;
    p3_s2_task(k1, jz);
    cpx<float> d[4][8];
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++)
#pragma unroll
        for (int c1 = 0; c1 < 8; c1++) d[k2][c1] = P[(k1 + 32 * k2) * C::KP + C::pos(jz + 16 * c1)];
#pragma unroll
    for (int c1 = 1; c1 < 8; c1++) {
        const cpx<float> tw = TZ[c1 * 16 + jz];
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) d[k2][c1] = ctw<-1>(d[k2][c1], tw);
    }
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) Dft<8, -1, float>::run(d[k2]);
#pragma unroll
    for (int b = 0; b < 8; b++) {
        cpx<float> t[4] = {d[0][b], d[1][b], d[2][b], d[3][b]};
        Dft<4, -1, float>::run(t);
#pragma unroll
        for (int j2 = 0; j2 < 4; j2++) d[j2][b] = t[j2];
    }
#pragma unroll
    for (int j2 = 1; j2 < 4; j2++) {
        const cpx<float> tw = TY[j2 * 32 + k1];
#pragma unroll
        for (int b = 0; b < 8; b++) d[j2][b] = ctw<-1>(d[j2][b], tw);
    }
#pragma unroll
    for (int j2 = 0; j2 < 4; j2++)
#pragma unroll
        for (int b = 0; b < 8; b++) P[(k1 + 32 * j2) * C::KP + C::pos(jz + 16 * b)] = d[j2][b];
}

// S3 tasks: (y, c1) = (u >> 3, u & 7) for u = threadIdx.x + 512 s, s = 0, 1
// (a half-warp covers two adjacent rows, whose pitch differs by 8 bank pairs)
template <int MODE>
__device__ __forceinline__ void p3_s3(cpx<float> *P, const PlaneArgs<float> &a, long long plane_off, long long M,
                                      double &qsum)
{
    using C = Plane3Cfg;
    // stored propagators and h as (chain 1, chain 2) pairs (fft_packed.cuh)
    const cpx<float> *__restrict__ hp = reinterpret_cast<const cpx<float> *>(a.h) + plane_off;
    cpx<float> *__restrict__ qp = reinterpret_cast<cpx<float> *>(a.qout) + plane_off;
    const int hs0 = a.hsel0, hs1 = a.hsel1;
#pragma unroll 1
    for (int s = 0; s < 2; s++) {
        const int u = threadIdx.x + 512 * s;
        const int y = u >> 3, c1 = u & 7;
        cpx<float> *row = P + y * C::KP;
        float ha[16], hb[16];
#pragma unroll
        for (int c2 = 0; c2 < 16; c2++) {
            const cpx<float> h = ld_pair(hp + y * 128 + c1 + 8 * c2);
            ha[c2] = hs0 ? h.y : h.x;
            hb[c2] = hs1 ? h.y : h.x;
        }
        cpx<float> g[16];
        p3_ld16(row + C::pos(16 * c1), g);
        Dft<16, 1, float>::run(g);
#pragma unroll
        for (int c2 = 0; c2 < 16; c2++) {
            const int z = c1 + 8 * c2;
            const float va = g[c2].x * ha[c2];
            const float vb = g[c2].y * hb[c2];
            st_pair(qp + y * 128 + z, va, vb);
            if (MODE == PLANE_LAST) qsum += (double)va;
            g[c2] = {va, vb};
        }
        if (MODE == PLANE_STEP) {
            Dft<16, -1, float>::run(g);
            p3_st16(row + C::pos(16 * c1), g);
        }
    }
}

// INIT: real rows from global (h from the fields, or given rows), forward S3
template <int MODE>
__device__ __forceinline__ void p3_s3_init(cpx<float> *P, const PlaneArgs<float> &a, long long plane_off, long long M)
{
    using C = Plane3Cfg;
#pragma unroll 1
    for (int s = 0; s < 2; s++) {
        const int u = threadIdx.x + 512 * s;
        const int y = u >> 3, c1 = u & 7;
        cpx<float> g[16];
#pragma unroll
        for (int c2 = 0; c2 < 16; c2++) {
            const long long i = plane_off + y * 128 + c1 + 8 * c2;
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
        Dft<16, -1, float>::run(g);
        p3_st16(P + y * C::KP + C::pos(16 * c1), g);
    }
}

template <int MODE>
__global__ void __launch_bounds__(Plane3Cfg::NT, 1) plane3_kernel(PlaneArgs<float> a)
{
    using C = Plane3Cfg;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<float> *P = reinterpret_cast<cpx<float> *>(smem_raw);
    cpx<float> *TY = reinterpret_cast<cpx<float> *>(smem_raw + C::TOFF);
    cpx<float> *TZ = TY + 128;

    const int x = blockIdx.x;
    const long long M = (long long)gridDim.x * 128 * 128;
    const long long plane_off = (long long)x * 128 * 128;
    cpx<float> *Sg = a.spec + plane_off;

    // constant tables (never written by the chain): before the grid dependency
    if (threadIdx.x < 128) {
        const int j2 = threadIdx.x >> 5, k1 = threadIdx.x & 31;
        TY[threadIdx.x] = a.twy[(j2 * k1) & 127];
    } else if (threadIdx.x < 256) {
        const int t = threadIdx.x - 128, c1 = t >> 4, jz = t & 15;
        TZ[t] = a.twz[(jz * c1) & 127];
    }
    pdl_launch_dependents();
    pdl_wait();

    if (MODE == PLANE_INIT_W || MODE == PLANE_INIT_Q) {
        p3_s3_init<MODE>(P, a, plane_off, M);
        __syncthreads();
        p3_s2_fwd(P, TY, TZ);
        __syncthreads();
        p3_s1_fwd(P, Sg);
        return;
    }

    p3_s1_inv(P, Sg);
    __syncthreads();
    p3_s2_inv(P, TY, TZ);
    __syncthreads();
    double qsum = 0.0;
    p3_s3<MODE>(P, a, plane_off, M, qsum);
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
    p3_s2_fwd(P, TY, TZ);
    __syncthreads();
    p3_s1_fwd(P, Sg);
}

}  // namespace lfts
