// Adjoint of ln Q with respect to the box lengths (FP64).
//
// With q_{i+1} = h_{i+1} .* G q_i, G = F^-1 diag(g) F (real, symmetric: g is
// real and even) and Q = (1/M) sum_r q_N(r), the complementary propagator of
// the reference (q^, src/diblock.cc:19-24: q^_i = h_i .* G q^_{i+1}, q^_N = hB)
// is exactly the adjoint chain, so
//     dQ/dtheta = (1/M) sum_{i=1}^{N-1} q^_{i+1}^T (dG/dtheta) q_i
//               = (1/M) sum_i sum_k dg(k)/dtheta Re[ qhat_i(k) conj(qhat^_{i+1}(k)) ]
// (full-spectrum sum; on the half spectrum every kz other than 0 and mz/2
// counts twice).  For theta = L_alpha, dg/dL_alpha = g 4 pi^2 k_alpha^2 /
// (3 N L_alpha^3); this kernel accumulates, per alpha,
//     S_alpha = sum_i sum_k w(kz) g(k) k_alpha^2 Re[qhat_i conj(qhat^_{i+1})]
// and the host applies the constant.  The yz-plane forward transforms of the
// pair (q_i, q^_{i+1}) come from plane_kernel (PLANE_INIT_Q, chains 0 and 1);
// this x-pencil variant transforms both chains' columns of a tile and forms the
// products in registers.
#pragma once
#include "fft_kernels.cuh"

namespace lfts {

struct AdjArgs {
    const cpx<double> *spec;  // chain 0 at spec, chain 1 at spec + mx*ncol
    const cpx<double> *twx;
    const double *gx, *gy, *gz;  // factorised g (1/M in gz)
    int ncol, KZ, mx, my, mz;
    double *partial;  // [gridDim.x][3], accumulated over launches
};

template <int NX, int CW>
struct AdjCfg {
    static constexpr int R1 = Plan<NX>::R1, R2 = Plan<NX>::R2;
    static constexpr int NT = 128;
    static constexpr size_t SMEM = sizeof(cpx<double>) * (size_t)(2 * NX * CW + NX);
    static_assert(CW * R2 <= NT, "one stage-A task per thread and chain");
};

__device__ __forceinline__ int signed_idx(int K, int m) { return (K <= m / 2) ? K : K - m; }

template <int NX, int CW>
__global__ void __launch_bounds__(AdjCfg<NX, CW>::NT) pencil_adj_kernel(AdjArgs a)
{
    using C = AdjCfg<NX, CW>;
    constexpr int R1 = C::R1, R2 = C::R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<double> *T0 = reinterpret_cast<cpx<double> *>(smem_raw);
    cpx<double> *T1 = T0 + NX * CW;
    cpx<double> *twx = T1 + NX * CW;
    __shared__ double red[3][C::NT / 32];

    const int col0 = blockIdx.x * CW, ncol = a.ncol;
    for (int t = threadIdx.x; t < NX; t += C::NT) twx[t] = a.twx[t];
    __syncthreads();

    // stage A of both chains: strided rows from global, DFT, twiddle, to smem
    {
        const int t = threadIdx.x;
        const int cl = t % CW, j2 = t / CW, col = col0 + cl;
        if (t < CW * R2 && col < ncol) {
#pragma unroll
            for (int ch = 0; ch < 2; ch++) {
                const cpx<double> *Sg = a.spec + (long long)ch * a.mx * ncol;
                cpx<double> *Tl = ch ? T1 : T0;
                cpx<double> v[R1];
#pragma unroll
                for (int s = 0; s < R1; s++) v[s] = Sg[(long long)(j2 + R2 * s) * ncol + col];
                Dft<R1, -1, double>::run(v);
#pragma unroll
                for (int k1 = 0; k1 < R1; k1++)
                    Tl[(j2 + R2 * k1) * CW + cl] = ctw<-1>(v[k1], twx[(j2 * k1) % NX]);
            }
        }
    }
    __syncthreads();

    // stage B of both chains -> X[kx = k1 + R1 k2]; products weighted by k^2
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int t = threadIdx.x; t < CW * R1; t += C::NT) {
        const int cl = t % CW, k1 = t / CW, col = col0 + cl;
        if (col >= ncol) continue;
        cpx<double> u[R2], v[R2];
#pragma unroll
        for (int s = 0; s < R2; s++) {
            u[s] = T0[(R2 * k1 + s) * CW + cl];
            v[s] = T1[(R2 * k1 + s) * CW + cl];
        }
        Dft<R2, -1, double>::run(u);
        Dft<R2, -1, double>::run(v);
        const int Ky = col / a.KZ, kz = col % a.KZ;
        const int ky = signed_idx(Ky, a.my);
        const double wz = (kz == 0 || 2 * kz == a.mz) ? 1.0 : 2.0;
        const double gyz = a.gy[Ky] * a.gz[kz] * wz;
#pragma unroll
        for (int k2 = 0; k2 < R2; k2++) {
            const int Kx = k1 + R1 * k2;
            const int kx = signed_idx(Kx, a.mx);
            const double p = a.gx[Kx] * gyz * (u[k2].x * v[k2].x + u[k2].y * v[k2].y);  // Re(u conj v)
            sx += p * (double)(kx * kx);
            sy += p * (double)(ky * ky);
            sz += p * (double)(kz * kz);
        }
    }
    double s3[3] = {sx, sy, sz};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double v = s3[d];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[d][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0.0;
        for (int w = 0; w < C::NT / 32; w++) v += red[threadIdx.x][w];
        a.partial[blockIdx.x * 3 + threadIdx.x] += v;
    }
}

}  // namespace lfts
