// The scalar part of anderson::mix on the device (src/anderson.cc:35-89 and
// the LU solve of :106-127), shared by the replica ensemble
// (ensemble_kernels.cuh) and a single context's device-side Anderson loop
// (lfts_capi.cu): one block reduces the residual dot products in a fixed
// order, one warp builds and solves the least-squares system and does the
// history bookkeeping, so both produce bit for bit what the host-driven loop
// (anderson_mix_host in lfts_capi.cu) produces.
#pragma once
#include "field_kernels.cuh"

namespace lfts {

__device__ __forceinline__ int anderson_nh(int k) { return (k < kMaxHist + 1) ? k - 1 : kMaxHist; }

// GSL-style LU with partial pivoting and the two triangular solves
// (src/anderson.cc:106-127) on one warp: lane i holds row i of the n x n
// matrix (n <= kMaxHist) in registers and y[i].  Every matrix element goes
// through the same operations in the same order as in the sequential
// algorithm, each rounded separately (no fused multiply-adds), so x equals
// the host's result bit for bit.  Returns false (all lanes) for an exactly
// singular matrix.  x is valid in lane i for i < n.
__device__ __forceinline__ bool lu_solve_warp(double (&a)[kMaxHist], double y, double &x, int n)
{
    const int lane = threadIdx.x & 31;
    int perm = lane;  // original row now at this position
#pragma unroll
    for (int j = 0; j < kMaxHist; j++) {
        if (j >= n) break;
        // first maximal |a_ij|, i >= j (scan in row order, as sequentially)
        int piv = j;
        double amax = fabs(__shfl_sync(0xffffffffu, a[j], j));
        for (int i = j + 1; i < n; i++) {
            const double v = fabs(__shfl_sync(0xffffffffu, a[j], i));
            if (v > amax) {
                amax = v;
                piv = i;
            }
        }
        if (piv != j) {
            const int src = lane == j ? piv : (lane == piv ? j : lane);
#pragma unroll
            for (int k = 0; k < kMaxHist; k++) a[k] = __shfl_sync(0xffffffffu, a[k], src);
            perm = __shfl_sync(0xffffffffu, perm, src);
        }
        if (j + 1 < n) {
            const double ajj = __shfl_sync(0xffffffffu, a[j], j);
            if (lane > j && lane < n) {
                if (fabs(ajj) >= 2.2250738585072014e-308)
                    a[j] = __dmul_rn(a[j], __ddiv_rn(1.0, ajj));
                else
                    a[j] = __ddiv_rn(a[j], ajj);
            }
#pragma unroll
            for (int k = 0; k < kMaxHist; k++) {
                if (k > j && k < n) {
                    const double ajk = __shfl_sync(0xffffffffu, a[k], j);
                    if (lane > j && lane < n) a[k] = __dsub_rn(a[k], __dmul_rn(a[j], ajk));
                }
            }
        }
    }
    double diag = 1.0;
#pragma unroll
    for (int k = 0; k < kMaxHist; k++)
        if (k == lane) diag = a[k];
    if (__any_sync(0xffffffffu, lane < n && diag == 0.0)) return false;
    // forward substitution (unit lower), x_j broadcast as it becomes final
    double t = __shfl_sync(0xffffffffu, y, perm);
#pragma unroll
    for (int j = 0; j < kMaxHist; j++) {
        if (j >= n) break;
        const double xj = __shfl_sync(0xffffffffu, t, j);
        if (lane > j && lane < n) t = __dsub_rn(t, __dmul_rn(a[j], xj));
    }
    // back substitution: row i subtracts a_ij x_j for j = i+1 .. n-1 in order
    x = t;
    for (int i = n - 1; i >= 0; i--) {
        double ti = x;
#pragma unroll
        for (int j = 0; j < kMaxHist; j++) {
            if (j > i && j < n) {
                const double xj = __shfl_sync(0xffffffffu, x, j);
                if (lane == i) ti = __dsub_rn(ti, __dmul_rn(a[j], xj));
            }
        }
        if (lane == i) x = __ddiv_rn(ti, diag);
    }
    return true;
}

// One Anderson iteration's scalar step for loop state R (a struct with the
// fields used below: k, DD, coef, simple, go, stopped, singular, notconv,
// nonfinite), run by a whole block of 256 threads: the reduction of the
// per-block partial dot products (as reduce_partials_kernel, fixed order),
// then on one warp the row DD[0][0..nh], the least-squares coefficients
// (k >= 2), the DD bookkeeping and whether the loop goes on (err > tol and
// k + 1 < maxIter).
template <typename St>
__device__ __forceinline__ void anderson_reduce_solve(St &R, const double *__restrict__ partials, int red_blocks,
                                                      long long M, double tol, int maxIter)
{
    __shared__ double sh[32];
    __shared__ double dd0[kRedWidth];
    const int k = R.k, nh = anderson_nh(k);
    for (int m = 0; m <= nh; m++) {
        double v = 0.0;
        for (int b = threadIdx.x; b < red_blocks; b += blockDim.x) v += partials[(long long)b * kRedWidth + m];
        v = block_sum(v, sh);
        if (threadIdx.x == 0) dd0[m] = v;
    }
    __syncthreads();
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    if (lane <= nh) R.DD[0][lane] = dd0[lane];
    __syncwarp();
    const double DD00 = dd0[0];
    bool ok = true;
    if (k >= 2) {
        // U_mn = DD00 - DD0m - DD0n + DD_nm (upper triangle), V_m = DD00 - DD0m
        double a[kMaxHist];
        const int m = lane + 1;  // this lane's row
#pragma unroll
        for (int c = 0; c < kMaxHist; c++) {
            const int n = c + 1;
            a[c] = 0.0;
            if (m <= nh && n <= nh) {
                const int lo = m < n ? m : n, hi = m < n ? n : m;
                a[c] = __dadd_rn(__dsub_rn(__dsub_rn(DD00, dd0[hi]), dd0[lo]), R.DD[lo][hi]);
            }
        }
        const double v = m <= nh ? __dsub_rn(DD00, dd0[m]) : 0.0;
        double x = 0.0;
        ok = lu_solve_warp(a, v, x, nh);
        if (ok && lane < nh) R.coef[lane] = x;
    }
    __syncwarp();
    if (lane == 0) {
        R.simple = k < 2;
        // err = (S1/M)^(1/2) (the reference takes pow(., 0.5); sqrt is the
        // correctly rounded value of the same)
        const double err = sqrt(__ddiv_rn(DD00, (double)M));
        if (!isfinite(err)) {
            // a NaN or infinite residual: stop before w+ is updated with it
            // (the reference would update and then leave the loop, as NaN > tol
            // is false)
            R.nonfinite = 1;
            R.stopped = 1;
            R.go = 0;
        } else if (!ok) {
            R.singular = 1;
            R.stopped = 1;
            R.go = 0;
        } else {
            R.go = 1;
            // the current deviation becomes history slot n (src/anderson.cc:82-89)
            const int n = 1 + (k - 1) % kMaxHist;
            R.DD[n][n] = DD00;
            for (int c = 1; c < n; c++) R.DD[c][n] = dd0[c];
            for (int c = n + 1; c <= nh; c++) R.DD[n][c] = dd0[c];
            if (!(err > tol) || !(k + 1 < maxIter)) {
                R.stopped = 1;
                R.notconv = err > tol;  // the loop ends at the cap, above the tolerance
            }
        }
    }
}

// ---- one context's Anderson loop on the device --------------------------------
// anderson::mix as a CUDA graph: begin -> WHILE { contour chain, concentrations
// with the residual dot products, reduce + solve, w+ update, control }, no
// host round trip per iteration.  The state lives in device memory; maxIter
// and tol are written into it before each launch.
struct MixState {
    long long M;
    int red_blocks;
    int maxIter;
    double tol;
    double *w;              // fields [W-, w+, phi-, phi+]
    double *partials;       // per-block dot products
    const double *lambda;   // 1 - 0.9^k, k <= maxIter
    void *Dh[kRedWidth], *wh[kRedWidth];  // history ring, the context's propagator type
    int phys[kRedWidth];    // logical history slot -> physical buffer
    int cur;                // physical buffer of the current iteration
    int k, stopped, go, simple, singular, notconv, nonfinite, iters, guard;
    double coef[kMaxHist];
    double DD[kRedWidth][kRedWidth];
};

static __global__ void mix_begin_kernel(MixState *S)
{
    if (threadIdx.x != 0) return;
    S->k = 1;
    S->stopped = S->go = S->singular = S->notconv = S->nonfinite = S->guard = 0;
    S->iters = 0;
}

// the concentrations of this iteration with Dh0 and its dot products
// against the nh history slots (src/diblock.cc:50-60, src/anderson.cc:35-55)
template <typename T>
__global__ void __launch_bounds__(kRedThreads, 4)
    mix_conc_kernel(const MixState *__restrict__ S, const T *__restrict__ q, int N, int NA, const double *__restrict__ Qd)
{
    const int nh = anderson_nh(S->k);
    HistPtrs hist{};
    for (int m = 1; m <= nh; m++) hist.p[m - 1] = S->Dh[S->phys[m]];
    const long long M = S->M;
    concentrations_body<T>(q, M, N, NA, S->w, S->w + 2 * M, S->w + 3 * M, Qd, static_cast<T *>(S->Dh[S->cur]), nh,
                           hist, S->partials, blockIdx.x, gridDim.x);
}

// the same from the concentration sums the contour chain formed (PENCIL_HA)
static __global__ void __launch_bounds__(kRedThreads, 4)
    mix_conc_acc_kernel(const MixState *__restrict__ S, const float *__restrict__ acc, const float *__restrict__ h,
                        int N, const double *__restrict__ Qd)
{
    const int nh = anderson_nh(S->k);
    HistPtrs hist{};
    for (int m = 1; m <= nh; m++) hist.p[m - 1] = S->Dh[S->phys[m]];
    const long long M = S->M;
    concentrations_acc_body(acc, h, M, N, S->w + 2 * M, S->w + 3 * M, Qd, static_cast<float *>(S->Dh[S->cur]), nh,
                            hist, S->partials, blockIdx.x, gridDim.x);
}

static __global__ void __launch_bounds__(256) mix_solve_kernel(MixState *S)
{
    anderson_reduce_solve(*S, S->partials, S->red_blocks, S->M, S->tol, S->maxIter);
}

// w+ update (src/anderson.cc:57-79)
template <typename T>
__global__ void __launch_bounds__(256) mix_update_kernel(const MixState *__restrict__ S)
{
    if (!S->go) return;
    const int nh = anderson_nh(S->k);
    HistPtrs Dhp{}, whp{};
    for (int m = 1; m <= nh; m++) {
        Dhp.p[m - 1] = S->Dh[S->phys[m]];
        whp.p[m - 1] = S->wh[S->phys[m]];
    }
    anderson_update_body<T>(S->w + S->M, static_cast<T *>(S->wh[S->cur]), static_cast<const T *>(S->Dh[S->cur]), S->M,
                            S->lambda[S->k], nh, S->simple, Dhp, whp, S->coef, blockIdx.x, gridDim.x);
}

// history rotation (src/anderson.cc:82-89) and the next iteration number;
// ends the WHILE loop once this iteration stopped it (k is then the value
// anderson::mix returns), and in any case past maxIter + 2 iterations
static __global__ void mix_control_kernel(MixState *S, cudaGraphConditionalHandle loop)
{
    if (threadIdx.x != 0) return;
    if (S->go) {
        const int n = 1 + (S->k - 1) % kMaxHist;
        const int evicted = S->phys[n];
        S->phys[n] = S->cur;
        S->cur = evicted;
    }
    S->k++;
    const bool cut = ++S->guard >= S->maxIter + 2;
    if (cut) S->notconv = 1;
    if (S->stopped || cut) {
        S->iters = S->k;
        cudaGraphSetConditional(loop, 0u);
    } else {
        cudaGraphSetConditional(loop, 1u);
    }
}

}  // namespace lfts
