// Streaming kernels around the contour steps: concentrations (with the
// Anderson residual and its dot products fused in), the Anderson w+ update,
// the Langevin W- update, S(k) spherical binning and the H sums.
//
// The element-wise updates reproduce the reference's expression trees with
// explicitly rounded operations (__dadd_rn etc.), so no multiply-add is
// contracted and a GPU element equals the reference's element bit for bit
// given equal inputs.  Reductions are deterministic: fixed grid, fixed
// per-block tree, fixed-order final pass.
#pragma once
#include <cuda_runtime.h>

namespace lfts {

constexpr int kMaxHist = 10;          // anderson(M_, 10) (src/lfts_simulation.cc:34)
constexpr int kRedWidth = kMaxHist + 1;
constexpr int kRedThreads = 256;

// Anderson history buffers; their element type is the context's propagator
// type (FP64, or FP32 in the FP32-mixed path, where only the least squares,
// Q and H are kept in FP64)
struct HistPtrs {
    const void *p[kMaxHist];
};
struct Coefs {
    double c[kMaxHist];
};

// sum of v over the block; result valid in thread 0
__device__ __forceinline__ double block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += sh[i];
    return s;
}

// Q = sum(qpart)/M and ln Q (src/diblock.cc:46-48,59)
static __global__ void q_finalize_kernel(const double *qpart, int n, long long M, double *Q_out)
{
    __shared__ double sh[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += qpart[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
        const double Q = s / (double)M;
        Q_out[0] = Q;
        Q_out[1] = log(Q);
    }
}

// Per-plane sums of chain 1's last propagator q_N (the first component of the
// stored FP32 pairs), one CTA per x-plane in a fixed order: the partials
// q_finalize_kernel reduces, for the chain that stores q in the x-pencil.
// (body: plane x of one field; the ensemble's batched launch calls it per replica)
__device__ __forceinline__ void plane_q_sums_body(const float2 *__restrict__ qN, long long plane, double *qpart,
                                                  const int x)
{
    __shared__ double sh[32];
    const float2 *p = qN + x * plane;
    double s = 0.0;
    for (long long i = threadIdx.x; i < plane; i += blockDim.x) s += (double)p[i].x;
    s = block_sum(s, sh);
    if (threadIdx.x == 0) qpart[x] = s;
}

static __global__ void __launch_bounds__(256) plane_q_sums_kernel(const float2 *__restrict__ qN, long long plane,
                                                                  double *qpart)
{
    plane_q_sums_body(qN, plane, qpart, blockIdx.x);
}

template <typename T, int V>
struct VecOf;
template <> struct VecOf<float, 4> { using type = float4; };
template <> struct VecOf<double, 2> { using type = double2; };

template <typename T, int V>
__device__ __forceinline__ void vload(const T *p, T (&out)[V])
{
    using VT = typename VecOf<T, V>::type;
    const VT v = *reinterpret_cast<const VT *>(p);
    const T *e = reinterpret_cast<const T *>(&v);
#pragma unroll
    for (int j = 0; j < V; j++) out[j] = e[j];
}

// phi-/phi+ (src/diblock.cc:50-57, 85-95) and, when Dh0 != nullptr, the
// Anderson residual Dh0 = phi+ - 1 with partial sums of Dh0*Dh0 and
// Dh0*Dh_m, m = 1..nh (src/anderson.cc:35-55).  Each thread handles V
// consecutive mesh points with vector loads; h comes from slot 1 (= [hA|hB]).
// body of block `blk` of `nblk` (the grid-stride partition fixes the order of
// the dot-product partial sums, so a replica's result does not depend on how
// its blocks are launched)
template <typename T>
__device__ __forceinline__ void concentrations_body(
    const T *__restrict__ q, long long M, int N, int NA, const double *__restrict__ w,
    double *__restrict__ phim, double *__restrict__ phip, const double *__restrict__ Qd,
    T *__restrict__ Dh0, int nh, const HistPtrs &hist, double *__restrict__ partials, const int blk,
    const int nblk)
{
    constexpr int V = sizeof(T) == 4 ? 4 : 2;
    using VT = typename VecOf<T, V>::type;
    __shared__ double sh[kRedThreads / 32];
    const double Q = Qd[0];
    const double NQ = __dmul_rn((double)N, Q);
    double acc[kRedWidth];
#pragma unroll
    for (int m = 0; m < kRedWidth; m++) acc[m] = 0.0;
    const long long nvec = M / V;
    const long long stride = (long long)nblk * blockDim.x;
    for (long long g = (long long)blk * blockDim.x + threadIdx.x; g < nvec; g += stride) {
        const long long r0 = g * V;
        // slot i holds [q_i | q^_{N+1-i}] (src/diblock.cc:19-24); slot i at q + (i-1)*2M
        double sA[V], sB[V];
#pragma unroll
        for (int j = 0; j < V; j++) sA[j] = sB[j] = 0.0;
        T hA[V], hB[V];
        if constexpr (sizeof(T) == 4) {
            // FP32 packed layout: slot i holds pairs (q_i, q^_{N+1-i}) (fft_packed.cuh),
            // so slots i and j = N+1-i together give q_i q^_i and q_j q^_j
#pragma unroll 4
            for (int i = 1; 2 * i <= N + 1; i++) {
                const int j = N + 1 - i;
                T a[2 * V], b[2 * V];
                vload<T, V>(q + (long long)(i - 1) * 2 * M + 2 * r0, *reinterpret_cast<T(*)[V]>(a));
                vload<T, V>(q + (long long)(i - 1) * 2 * M + 2 * r0 + V, *reinterpret_cast<T(*)[V]>(a + V));
                vload<T, V>(q + (long long)(j - 1) * 2 * M + 2 * r0, *reinterpret_cast<T(*)[V]>(b));
                vload<T, V>(q + (long long)(j - 1) * 2 * M + 2 * r0 + V, *reinterpret_cast<T(*)[V]>(b + V));
#pragma unroll
                for (int p = 0; p < V; p++) {
                    const double pi = __dmul_rn((double)a[2 * p], (double)b[2 * p + 1]);  // q_i q^_i
                    if (i <= NA)
                        sA[p] = __dadd_rn(sA[p], pi);
                    else
                        sB[p] = __dadd_rn(sB[p], pi);
                    if (j != i) {
                        const double pj = __dmul_rn((double)b[2 * p], (double)a[2 * p + 1]);  // q_j q^_j
                        if (j <= NA)
                            sA[p] = __dadd_rn(sA[p], pj);
                        else
                            sB[p] = __dadd_rn(sB[p], pj);
                    }
                }
            }
            T h[2 * V];
            vload<T, V>(q + 2 * r0, *reinterpret_cast<T(*)[V]>(h));
            vload<T, V>(q + 2 * r0 + V, *reinterpret_cast<T(*)[V]>(h + V));
#pragma unroll
            for (int p = 0; p < V; p++) {
                hA[p] = h[2 * p];
                hB[p] = h[2 * p + 1];
            }
        } else {
#pragma unroll 8
            for (int i = 1; i <= N; i++) {
                T a[V], b[V];
                vload<T, V>(q + (long long)(i - 1) * 2 * M + r0, a);
                vload<T, V>(q + (long long)(N - i) * 2 * M + M + r0, b);
                if (i <= NA) {
#pragma unroll
                    for (int j = 0; j < V; j++) sA[j] = __dadd_rn(sA[j], __dmul_rn((double)a[j], (double)b[j]));
                } else {
#pragma unroll
                    for (int j = 0; j < V; j++) sB[j] = __dadd_rn(sB[j], __dmul_rn((double)a[j], (double)b[j]));
                }
            }
            vload<T, V>(q + r0, hA);
            vload<T, V>(q + M + r0, hB);
        }
        double pm[V], pp[V];
#pragma unroll
        for (int j = 0; j < V; j++) {
            const double fA = sA[j] / __dmul_rn(NQ, (double)hA[j]);
            const double fB = sB[j] / __dmul_rn(NQ, (double)hB[j]);
            pm[j] = __dsub_rn(fA, fB);
            pp[j] = __dadd_rn(fA, fB);
        }
#pragma unroll
        for (int j = 0; j < V; j += 2) {
            *reinterpret_cast<double2 *>(phim + r0 + j) = make_double2(pm[j], pm[j + 1]);
            *reinterpret_cast<double2 *>(phip + r0 + j) = make_double2(pp[j], pp[j + 1]);
        }
        if (Dh0) {
            double d[V];
#pragma unroll
            for (int j = 0; j < V; j++) {
                d[j] = __dsub_rn(pp[j], 1.0);
                acc[0] = __dadd_rn(acc[0], __dmul_rn(d[j], d[j]));
            }
            {
                VT dv;
                T *e = reinterpret_cast<T *>(&dv);
#pragma unroll
                for (int j = 0; j < V; j++) e[j] = (T)d[j];
                *reinterpret_cast<VT *>(Dh0 + r0) = dv;
            }
#pragma unroll
            for (int m = 1; m < kRedWidth; m++) {
                if (m <= nh) {
                    T hv[V];
                    vload<T, V>(static_cast<const T *>(hist.p[m - 1]) + r0, hv);
#pragma unroll
                    for (int j = 0; j < V; j++) acc[m] = __dadd_rn(acc[m], __dmul_rn(d[j], (double)hv[j]));
                }
            }
        }
    }
    (void)w;
    if (!Dh0) return;
#pragma unroll
    for (int m = 0; m < kRedWidth; m++) {
        if (m > nh) break;
        const double s = block_sum(acc[m], sh);
        if (threadIdx.x == 0) partials[(long long)blk * kRedWidth + m] = s;
    }
}

// The same with the sums over the monomers already formed by the contour chain
// (the x-pencil's PENCIL_HA modes, FP32 packed path): acc[r] = (sum over A
// monomers of q_i q^_i, sum over B monomers), h = slot 1 = (hA, hB).  Two mesh
// points per thread and iteration; the dot-product partition is fixed by
// (blk, nblk) as in concentrations_body.
__device__ __forceinline__ void concentrations_acc_body(
    const float *__restrict__ acc, const float *__restrict__ h, long long M, int N, double *__restrict__ phim,
    double *__restrict__ phip, const double *__restrict__ Qd, float *__restrict__ Dh0, int nh, const HistPtrs &hist,
    double *__restrict__ partials, const int blk, const int nblk)
{
    __shared__ double sh[kRedThreads / 32];
    const double NQ = __dmul_rn((double)N, Qd[0]);
    double dots[kRedWidth];
#pragma unroll
    for (int m = 0; m < kRedWidth; m++) dots[m] = 0.0;
    const long long npair = M / 2;
    const long long stride = (long long)nblk * blockDim.x;
    for (long long g = (long long)blk * blockDim.x + threadIdx.x; g < npair; g += stride) {
        const long long r0 = 2 * g;
        const float4 s = *reinterpret_cast<const float4 *>(acc + 2 * r0);
        const float4 hh = *reinterpret_cast<const float4 *>(h + 2 * r0);
        const double sA[2] = {(double)s.x, (double)s.z}, sB[2] = {(double)s.y, (double)s.w};
        const double hA[2] = {(double)hh.x, (double)hh.z}, hB[2] = {(double)hh.y, (double)hh.w};
        double pm[2], pp[2];
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const double fA = sA[j] / __dmul_rn(NQ, hA[j]);
            const double fB = sB[j] / __dmul_rn(NQ, hB[j]);
            pm[j] = __dsub_rn(fA, fB);
            pp[j] = __dadd_rn(fA, fB);
        }
        *reinterpret_cast<double2 *>(phim + r0) = make_double2(pm[0], pm[1]);
        *reinterpret_cast<double2 *>(phip + r0) = make_double2(pp[0], pp[1]);
        if (Dh0) {
            double d[2];
#pragma unroll
            for (int j = 0; j < 2; j++) {
                d[j] = __dsub_rn(pp[j], 1.0);
                dots[0] = __dadd_rn(dots[0], __dmul_rn(d[j], d[j]));
            }
            *reinterpret_cast<float2 *>(Dh0 + r0) = make_float2((float)d[0], (float)d[1]);
#pragma unroll
            for (int m = 1; m < kRedWidth; m++) {
                if (m <= nh) {
                    const float2 hv = *reinterpret_cast<const float2 *>(static_cast<const float *>(hist.p[m - 1]) + r0);
                    dots[m] = __dadd_rn(dots[m], __dmul_rn(d[0], (double)hv.x));
                    dots[m] = __dadd_rn(dots[m], __dmul_rn(d[1], (double)hv.y));
                }
            }
        }
    }
    if (!Dh0) return;
#pragma unroll
    for (int m = 0; m < kRedWidth; m++) {
        if (m > nh) break;
        const double s = block_sum(dots[m], sh);
        if (threadIdx.x == 0) partials[(long long)blk * kRedWidth + m] = s;
    }
}

static __global__ void __launch_bounds__(kRedThreads, 4) concentrations_acc_kernel(
    const float *__restrict__ acc, const float *__restrict__ h, long long M, int N, double *__restrict__ phim,
    double *__restrict__ phip, const double *__restrict__ Qd, float *__restrict__ Dh0, int nh, HistPtrs hist,
    double *__restrict__ partials)
{
    concentrations_acc_body(acc, h, M, N, phim, phip, Qd, Dh0, nh, hist, partials, blockIdx.x, gridDim.x);
}

template <typename T>
static __global__ void __launch_bounds__(kRedThreads, 4) concentrations_kernel(
    const T *__restrict__ q, long long M, int N, int NA, const double *__restrict__ w,
    double *__restrict__ phim, double *__restrict__ phip, const double *__restrict__ Qd,
    T *__restrict__ Dh0, int nh, HistPtrs hist, double *__restrict__ partials)
{
    concentrations_body<T>(q, M, N, NA, w, phim, phip, Qd, Dh0, nh, hist, partials, blockIdx.x, gridDim.x);
}

// out[m] = sum over blocks of partials[b][m], fixed order; block m < width
// reduces column m (launch width blocks of 256 threads: every column's sum
// is formed in the same order as by one block looping over the columns)
static __global__ void reduce_partials_kernel(const double *partials, int nblocks, int width, double *out)
{
    __shared__ double sh[32];
    const int m = blockIdx.x;
    if (m >= width) return;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[(long long)b * kRedWidth + m];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) out[m] = s;
}

// w+ update of one Anderson iteration (src/anderson.cc:57-79) and the copy
// of the pre-update w+ into the current history slot (wh_[0], :38).
template <typename H>
__device__ __forceinline__ void anderson_update_body(double *__restrict__ wp, H *__restrict__ wh0,
                                                     const H *__restrict__ Dh0, long long M, double lambda,
                                                     int nh, int simple, const HistPtrs &Dh, const HistPtrs &wh,
                                                     const double *c, const int blk, const int nblk)
{
    const long long stride = (long long)nblk * blockDim.x;
    for (long long r = (long long)blk * blockDim.x + threadIdx.x; r < M; r += stride) {
        const double old = wp[r];
        const double d0 = (double)Dh0[r];
        wh0[r] = (H)old;
        const double base = __dadd_rn(old, __dmul_rn(lambda, d0));
        double acc = base;
        if (!simple) {
#pragma unroll
            for (int n = 0; n < kMaxHist; n++) {
                if (n < nh) {
                    const double whn = (double)static_cast<const H *>(wh.p[n])[r];
                    const double dhn = (double)static_cast<const H *>(Dh.p[n])[r];
                    const double hn = __dadd_rn(whn, __dmul_rn(lambda, dhn));
                    acc = __dadd_rn(acc, __dmul_rn(c[n], __dsub_rn(hn, base)));
                }
            }
        }
        wp[r] = acc;
    }
}

template <typename H>
static __global__ void anderson_update_kernel(double *__restrict__ wp, H *__restrict__ wh0,
                                              const H *__restrict__ Dh0, long long M, double lambda, int nh,
                                              int simple, HistPtrs Dh, HistPtrs wh, Coefs C)
{
    anderson_update_body<H>(wp, wh0, Dh0, M, lambda, nh, simple, Dh, wh, C.c, blockIdx.x, gridDim.x);
}

// W- += -(phi- + 2 W-/XbN) dt + (eta_prev + eta_new)/2   (src/langevin.cc:31)
static __global__ void langevin_kernel(double *__restrict__ w, long long M, const double *__restrict__ eta_prev,
                                const double *__restrict__ eta_new, double XbN, double dt)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < M; r += stride) {
        const double wm = w[r], pm = w[2 * M + r];
        const double drift = __dmul_rn(-__dadd_rn(pm, __ddiv_rn(__dmul_rn(2.0, wm), XbN)), dt);
        const double noise = __dmul_rn(0.5, __dadd_rn(eta_prev[r], eta_new[r]));
        w[r] = __dadd_rn(wm, __dadd_rn(drift, noise));
    }
}

// partial sums of w+ and W-^2 (src/lfts_simulation.cc:129-131)
static __global__ void __launch_bounds__(kRedThreads) h_sums_kernel(const double *__restrict__ w, long long M,
                                                             double *partials)
{
    __shared__ double sh[kRedThreads / 32];
    double sp = 0.0, s2 = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < M; r += stride) {
        const double wm = w[r];
        sp += w[M + r];
        s2 += wm * wm;
    }
    sp = block_sum(sp, sh);
    if (threadIdx.x == 0) partials[(long long)blockIdx.x * kRedWidth + 0] = sp;
    s2 = block_sum(s2, sh);
    if (threadIdx.x == 0) partials[(long long)blockIdx.x * kRedWidth + 1] = s2;
}

// Spherical average of S(k) (src/strFunc.cc:50-76): one thread per |K| bin,
// summing its wavevectors in the reference's stable-sorted order.
static __global__ void sk_bin_kernel(const double *__restrict__ S, const int *__restrict__ order,
                              const int *__restrict__ wt, const int *__restrict__ bin_start, int nbins,
                              double coeff_over_ns, double half_over_chi, double *__restrict__ out)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbins) return;
    double s = 0.0;
    int n = 0;
    for (int k = bin_start[b]; k < bin_start[b + 1]; k++) {
        const int p = order[k];
        const double term = __dsub_rn(__dmul_rn(coeff_over_ns, S[p]), half_over_chi);
        s = __dadd_rn(s, __dmul_rn((double)wt[p], term));
        n += wt[p];
    }
    out[b] = s / (double)n;
}

// [a | b] halves (M each) <-> M pairs (a, b): the FP32 packed path stores h
// and the propagators as pairs
template <typename Tin, typename Tout>
static __global__ void to_pairs_kernel(const Tin *__restrict__ in, Tout *__restrict__ out, long long M)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < M; r += stride) {
        out[2 * r] = (Tout)in[r];
        out[2 * r + 1] = (Tout)in[M + r];
    }
}
template <typename Tin, typename Tout>
static __global__ void from_pairs_kernel(const Tin *__restrict__ in, Tout *__restrict__ out, long long M)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < M; r += stride) {
        out[r] = (Tout)in[2 * r];
        out[M + r] = (Tout)in[2 * r + 1];
    }
}

template <typename Tin, typename Tout>
static __global__ void convert_kernel(const Tin *__restrict__ in, Tout *__restrict__ out, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = (Tout)in[i];
}

}  // namespace lfts
