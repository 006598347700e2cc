// yz-plane kernel of the h-in-pencil chain (PLANE_G) with each x-plane split
// over a cluster of CL CTAs (FP32-mixed path, 128 x 128 planes).
//
// The whole-plane kernel (plane3_kernel, fft_plane3.cuh) runs one 512-thread
// CTA per x-plane: 128 planes leave 20 of the 148 SMs idle, and the one CTA
// per SM runs its load, arithmetic and store phases in lockstep.  Here the
// same three-stage transform (the same DFTs, twiddles and g products, value
// for value: the results are bitwise those of plane3_kernel) is spread over
// CL = 8 CTAs of 64 threads, each holding 1/8 of the plane (18 KB), so about
// seven CTAs of different planes share an SM and every SM carries work.
//
// Work split, with ky = j2 + Y2 a, y = k1 + Y1 k2, kz / z as in fft_plane3.cuh
// (Y1 = 32, Y2 = 4, Z1 = 8, Z2 = 16) and r the CTA's rank in its cluster:
//   S1 (DFT-Y1 over a):  kz in [16 r, 16 r + 16), all j2      (64 tasks)
//   S2 (DFT-Y2, DFT-Z1): k1 in [4 r, 4 r + 4), all jz         (64 tasks)
//   S3 (DFT-Z2, x g):    rows y = k1 + 32 k2 of those k1      (128 tasks)
// S2 and S3 work on the same 16 rows, so only the S1 <-> S2 transposes cross
// CTAs: S1 inverse pushes each value into the shared memory of the CTA whose
// S2 rows hold it, S2 forward pushes into the CTA whose S1 columns hold it
// (distributed shared memory stores, st.shared::cluster), each push followed
// by a cluster barrier.  One 2272-slot buffer per CTA serves both layouts:
//   layout B (S2, S3):   slot lr * KP + pos(p), local row lr = (k1 - 4 r) + 4 k2,
//                        column p = kz (after S1) or jz + 16 c1 (after S2)
//   layout A (S1 fwd):   slot (k1 + 32 j2) * 16 + (kz - 16 r)
// A barrier after every CTA's last S2 forward load separates the two uses.
// No CTA touches another's memory after the last barrier, so none waits at
// its exit.  Only this GPU's shared memory is addressed; there are no TMA
// copies.
#pragma once
#include <cstdint>

#include "fft_plane3.cuh"

namespace lfts {

template <typename C, int CL_>
struct Plane3Split {
    using Cfg = C;
    static constexpr int CL = CL_;
    static constexpr int NT = C::NT / CL;        // threads per CTA
    static constexpr int KZB = C::NZ / CL;       // S1 columns per CTA
    static constexpr int K1B = C::Y1 / CL;       // S2 k1 values per CTA
    static constexpr int ROWS = K1B * C::Y2;     // layout-B rows per CTA
    static constexpr int SLOTS_B = ROWS * C::KP;
    static constexpr int SLOTS_A = C::NY * KZB;
    static constexpr int SLOTS = SLOTS_B > SLOTS_A ? SLOTS_B : SLOTS_A;
    static constexpr size_t TOFF = sizeof(cpx<float>) * (size_t)SLOTS;
    // ... followed by TY[NY], TZ[NZ] (complex) and gz[NZ]
    static constexpr size_t SMEM = TOFF + sizeof(cpx<float>) * (C::NY + C::NZ) + sizeof(float) * C::NZ;
    static constexpr int NS3 = ROWS * C::Z1;     // S3 tasks per CTA
    static_assert(KZB == C::Z2, "an S1 column block is one run of Z2 slots of layout B");
    static_assert(KZB * C::Y2 == NT && K1B * C::Z2 == NT, "one S1 and one S2 task per thread");
    static_assert(NS3 % NT == 0, "whole S3 rounds");
};

using Plane3Split128 = Plane3Split<Plane3_128, 8>;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
// the same shared-memory offset in the CTA of rank `rank` of this cluster
__device__ __forceinline__ uint32_t cluster_addr(uint32_t a, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_cluster(uint32_t a, cpx<float> v)
{
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void cluster_arrive_relaxed() { asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

template <typename S>
__global__ void __launch_bounds__(S::NT, 8) __cluster_dims__(S::CL, 1, 1) plane3_split_g_kernel(PlaneArgs<float> a)
{
    using C = typename S::Cfg;
    constexpr int NY = C::NY, NZ = C::NZ, Y1 = C::Y1, Y2 = C::Y2, Z1 = C::Z1, Z2 = C::Z2, KP = C::KP;
    constexpr int KZB = S::KZB, K1B = S::K1B;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<float> *P = reinterpret_cast<cpx<float> *>(smem_raw);
    cpx<float> *TY = reinterpret_cast<cpx<float> *>(smem_raw + S::TOFF);
    cpx<float> *TZ = TY + NY;
    float *GZ = reinterpret_cast<float *>(TZ + NZ);

    const int t = threadIdx.x;
    const int r = (int)cluster_rank();
    const int x = blockIdx.x / S::CL;
    const long long plane_off = (long long)x * NY * NZ;
    cpx<float> *Sg = a.spec + plane_off;

    // every CTA of the cluster has started before any pushes into it
    cluster_arrive_relaxed();
    for (int i = t; i < NY + 2 * NZ; i += S::NT) {
        if (i < NY) {
            const int j2 = i / Y1, k1 = i % Y1;
            TY[i] = a.twy[(j2 * k1) % NY];
        } else if (i < NY + NZ) {
            const int u = i - NY, c1 = u / Z2, jz = u % Z2;
            TZ[u] = a.twz[(jz * c1) % NZ];
        } else {
            GZ[i - NY - NZ] = a.gz[i - NY - NZ];
        }
    }
    if (a.pf) {
        // this CTA's 1/CL of plane x of the slot the next (summing) x-pencil reads
        constexpr int BYTES = 2 * NY * NZ * (int)sizeof(float) / S::CL;
        const char *base = reinterpret_cast<const char *>(a.pf + 2 * plane_off) + (size_t)r * BYTES;
        for (int o = 128 * t; o < BYTES; o += 128 * S::NT) prefetch_l2(base + o);
    }
    pdl_launch_dependents();
    pdl_wait();

    const uint32_t Pa = smem_addr(P);
    // ---- S1 inverse: DFT-Y1 over a of column kz, pushed to the S2 owners
    {
        const int kzl = t % KZB, j2 = t / KZB, kz = KZB * r + kzl;
        cpx<float> v[Y1];
#pragma unroll
        for (int aa = 0; aa < Y1; aa++) v[aa] = Sg[(j2 + Y2 * aa) * NZ + kz];
        Dft<Y1, 1, float>::run(v);
        const int pc = C::pos(kz);
        cluster_wait();
#pragma unroll
        for (int k1 = 0; k1 < Y1; k1++) {
            const int lr = (k1 % K1B) + K1B * j2;
            st_cluster(cluster_addr(Pa + 8u * (uint32_t)(lr * KP + pc), (uint32_t)(k1 / K1B)), v[k1]);
        }
    }
    cluster_arrive();  // (the cluster barrier also publishes the tables)
    cluster_wait();

    // ---- S2 inverse (local): twiddles, DFT-Y2 over j2, DFT-Z1 over b, twiddles
    const int jz = t % Z2, k1l = t / Z2, k1 = K1B * r + k1l;
    {
        cpx<float> d[Y2][Z1];
#pragma unroll
        for (int j2 = 0; j2 < Y2; j2++)
#pragma unroll
            for (int b = 0; b < Z1; b++) d[j2][b] = P[(k1l + K1B * j2) * KP + C::pos(jz + Z2 * b)];
#pragma unroll
        for (int j2 = 1; j2 < Y2; j2++) {
            const cpx<float> tw = TY[j2 * Y1 + k1];
#pragma unroll
            for (int b = 0; b < Z1; b++) d[j2][b] = ctw<1>(d[j2][b], tw);
        }
#pragma unroll
        for (int b = 0; b < Z1; b++) {
            cpx<float> u[Y2];
#pragma unroll
            for (int j2 = 0; j2 < Y2; j2++) u[j2] = d[j2][b];
            Dft<Y2, 1, float>::run(u);
#pragma unroll
            for (int k2 = 0; k2 < Y2; k2++) d[k2][b] = u[k2];
        }
#pragma unroll
        for (int k2 = 0; k2 < Y2; k2++) Dft<Z1, 1, float>::run(d[k2]);
#pragma unroll
        for (int c1 = 1; c1 < Z1; c1++) {
            const cpx<float> tw = TZ[c1 * Z2 + jz];
#pragma unroll
            for (int k2 = 0; k2 < Y2; k2++) d[k2][c1] = ctw<1>(d[k2][c1], tw);
        }
#pragma unroll
        for (int k2 = 0; k2 < Y2; k2++)
#pragma unroll
            for (int c1 = 0; c1 < Z1; c1++) P[(k1l + K1B * k2) * KP + C::pos(jz + Z2 * c1)] = d[k2][c1];
    }
    __syncthreads();

    // ---- S3 (local): DFT-Z2 over jz, x g, inverse DFT-Z2; rows in natural y
    {
        const float gx = __ldg(a.gx + x);
#pragma unroll 1
        for (int u = t; u < S::NS3; u += S::NT) {
            const int lr = u / Z1, c1 = u % Z1;
            const int y = K1B * r + (lr % K1B) + Y1 * (lr / K1B);
            cpx<float> *row = P + lr * KP;
            const float gy = __ldg(a.gy + y);
            float gg[Z2];
#pragma unroll
            for (int c2 = 0; c2 < Z2; c2++) gg[c2] = gx * (gy * GZ[c1 + Z1 * c2]);
            cpx<float> g[Z2];
            p3_ld16(row + C::pos(Z2 * c1), g);
            Dft<Z2, 1, float>::run(g);
#pragma unroll
            for (int c2 = 0; c2 < Z2; c2++) g[c2] = {g[c2].x * gg[c2], g[c2].y * gg[c2]};
            Dft<Z2, -1, float>::run(g);
            p3_st16(row + C::pos(Z2 * c1), g);
        }
    }
    __syncthreads();

    // ---- S2 forward: loads (local), then the transforms while the other CTAs
    // finish theirs, then pushes to the S1 owners in layout A
    {
        cpx<float> d[Y2][Z1];
#pragma unroll
        for (int k2 = 0; k2 < Y2; k2++)
#pragma unroll
            for (int c1 = 0; c1 < Z1; c1++) d[k2][c1] = P[(k1l + K1B * k2) * KP + C::pos(jz + Z2 * c1)];
        cluster_arrive();  // this CTA's layout-B reads are done
#pragma unroll
        for (int c1 = 1; c1 < Z1; c1++) {
            const cpx<float> tw = TZ[c1 * Z2 + jz];
#pragma unroll
            for (int k2 = 0; k2 < Y2; k2++) d[k2][c1] = ctw<-1>(d[k2][c1], tw);
        }
#pragma unroll
        for (int k2 = 0; k2 < Y2; k2++) Dft<Z1, -1, float>::run(d[k2]);
#pragma unroll
        for (int b = 0; b < Z1; b++) {
            cpx<float> u[Y2];
#pragma unroll
            for (int k2 = 0; k2 < Y2; k2++) u[k2] = d[k2][b];
            Dft<Y2, -1, float>::run(u);
#pragma unroll
            for (int j2 = 0; j2 < Y2; j2++) d[j2][b] = u[j2];
        }
#pragma unroll
        for (int j2 = 1; j2 < Y2; j2++) {
            const cpx<float> tw = TY[j2 * Y1 + k1];
#pragma unroll
            for (int b = 0; b < Z1; b++) d[j2][b] = ctw<-1>(d[j2][b], tw);
        }
        cluster_wait();  // every CTA's layout-B reads are done: layout A may be written
#pragma unroll
        for (int j2 = 0; j2 < Y2; j2++)
#pragma unroll
            for (int b = 0; b < Z1; b++)
                st_cluster(cluster_addr(Pa + 8u * (uint32_t)((k1 + Y1 * j2) * KZB + jz), (uint32_t)b), d[j2][b]);
    }
    cluster_arrive();
    cluster_wait();

    // ---- S1 forward (local, layout A): DFT-Y1 over k1, to global rows ky = j2 + Y2 a
    {
        const int kzl = t % KZB, j2 = t / KZB, kz = KZB * r + kzl;
        cpx<float> v[Y1];
#pragma unroll
        for (int kk = 0; kk < Y1; kk++) v[kk] = P[(kk + Y1 * j2) * KZB + kzl];
        Dft<Y1, -1, float>::run(v);
#pragma unroll
        for (int aa = 0; aa < Y1; aa++) Sg[(j2 + Y2 * aa) * NZ + kz] = v[aa];
    }
}

}  // namespace lfts
