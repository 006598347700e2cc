// Batched kernels of the replica ensemble (lfts_ensemble.cu): many
// independent FP32-mixed L-FTS systems, grouped by mesh, advanced by one CUDA
// graph launch per Langevin step.  Every replica's arithmetic is that of a
// single FP32-mixed context (the same kernel bodies, the same reduction
// partitions), so a replica reproduces a single context fed the same noise.
//
// The Anderson loop runs on the device, per replica: each body iteration of
// the graph's WHILE node runs the contour chain, the concentrations with the
// residual dot products, the reduction and least-squares solve, the w+
// update and the control step.  A replica whose loop has stopped runs one
// more chain + concentrations (the reference's extra calc_concs after mix,
// src/lfts_simulation.cc:69-76) and then idles (its CTAs return at once)
// until every replica is done; the control kernel ends the WHILE loop then.
#pragma once
#include "fft_packed.cuh"
#include "fft_plane3.cuh"
#include "anderson_device.cuh"
#include "field_kernels.cuh"
#include "philox.cuh"

namespace lfts {

// device-resident descriptor of one replica (buffers owned by its context)
struct EnsRep {
    int mx, my, mz, N, NA, NB;
    long long M;
    int red_blocks;
    double XbN, dt, sigma;
    unsigned long long seed;
    double *w;
    float *q;
    cpx<float> *spec;
    const cpx<float> *tw[3];
    const float *g[3];
    double *qpart, *Qd, *partials;
    float *acc;  // (A, B) concentration sums formed in the chain (h-in-pencil groups with phi_in_chain), or null
    float *Dh[kRedWidth], *wh[kRedWidth];  // FP32 history (the FP32-mixed context's)
    // Anderson loop state
    int phys[kRedWidth];  // logical history slot -> physical buffer
    int cur;              // physical buffer of the current iteration
    int k;                // iteration number (src/anderson.cc:31)
    int active, stopped, done, go, simple, singular;
    int notconv, nonfinite;  // loop ended at maxIter above tol; NaN or infinite residual
    int sticky;              // OR over the mixes of one host call: 1 notconv, 2 singular, 4 nonfinite
    int iters;            // k at loop exit (the value anderson::mix returns)
    double coef[kMaxHist];
    double DD[kRedWidth][kRedWidth];
};

__device__ __forceinline__ int ens_nh(int k) { return anderson_nh(k); }

template <int NY, int NZ, int MODE>
__global__ void __launch_bounds__(PlaneCCfg<float, NY, NZ>::NT, 1)
    ens_plane_kernel(EnsRep *__restrict__ reps, const int *__restrict__ members, int i)
{
    const EnsRep &R = reps[members[blockIdx.y]];
    if (!R.active) return;
    PlaneArgs<float> a{};
    a.w = R.w;
    a.spec = R.spec;
    a.twy = R.tw[1];
    a.twz = R.tw[2];
    a.qpart = R.qpart;
    a.nchains = 2;
    a.Nd = (double)R.N;
    if (MODE == PLANE_INIT_W) {
        a.qout = R.q;  // slot 1 = [hA | hB]
    } else {
        a.h = R.q;
        a.qout = R.q + (long long)i * 2 * R.M;    // slot i+1
        a.hsel0 = i < R.NA ? 0 : 1;               // src/step.cc:53-57
        a.hsel1 = i < R.NB ? 1 : 0;               // src/step.cc:60-64
    }
    plane_c_body<float, NY, NZ, MODE>(a, blockIdx.x, R.mx);
}

// the three-stage plane body (64, 96, 128 planes), as the single context uses
template <typename C3, int MODE>
__global__ void __launch_bounds__(C3::NT, 1)
    ens_plane3_kernel(EnsRep *__restrict__ reps, const int *__restrict__ members, int i)
{
    const EnsRep &R = reps[members[blockIdx.y]];
    if (!R.active) return;
    PlaneArgs<float> a{};
    a.w = R.w;
    a.spec = R.spec;
    a.twy = R.tw[1];
    a.twz = R.tw[2];
    a.qpart = R.qpart;
    a.nchains = 2;
    a.Nd = (double)R.N;
    if (MODE == PLANE_INIT_W) {
        a.qout = R.q;
    } else if (MODE == PLANE_G) {
        // the h-in-pencil chain's plane (enqueue_chain_launches): g from the
        // separable tables; ahead of a summing pencil, its partner slot to L2
        a.gx = R.g[0];
        a.gy = R.g[1];
        a.gz = R.g[2];
        if (R.acc && R.N - i < i + 1) a.pf = R.q + (long long)(R.N - i - 1) * 2 * R.M;
    } else {
        a.h = R.q;
        a.qout = R.q + (long long)i * 2 * R.M;
        a.hsel0 = i < R.NA ? 0 : 1;
        a.hsel1 = i < R.NB ? 1 : 0;
    }
    plane3_body<C3, MODE>(a, blockIdx.x, R.mx);
}

// The h-in-pencil chain's x-pencils (the single context's
// enqueue_chain_launches, same arguments): INIT_W (h from the fields, stored
// as slot 1), H (store slot i+1), and, from the middle of the chain on when
// the replica forms its concentration sums in the chain (R.acc), HA / HA_LAST
// (add the slot's products with its stored partner slot N-i).
template <int NX, int CW, int MODE>
__global__ void __launch_bounds__(PencilCfg<float, NX, CW>::NT)
    ens_pencil_x_kernel(EnsRep *__restrict__ reps, const int *__restrict__ members, int i)
{
    const EnsRep &R = reps[members[blockIdx.y]];
    if (!R.active) return;
    PencilArgs<float> a{};
    a.spec = R.spec;
    a.twx = R.tw[0];
    a.gx = R.g[0];
    a.gy = R.g[1];
    a.gz = R.g[2];
    a.ncol = R.my * R.mz;
    a.KZ = R.mz;
    a.w = R.w;
    a.h = R.q;  // slot 1: the (hA, hB) pairs
    a.M = R.M;
    a.Nd = (double)R.N;
    if (MODE == PENCIL_INIT_W) {
        a.qout = R.q;
    } else {
        a.qout = R.q + (long long)i * 2 * R.M;  // slot i+1
        a.hsel0 = i < R.NA ? 0 : 1;              // src/step.cc:53-57
        a.hsel1 = i < R.NB ? 1 : 0;              // src/step.cc:60-64
        if (MODE == PENCIL_HA || MODE == PENCIL_HA_LAST) {
            const int p = R.N - i;  // partner slot
            a.partner = p < i + 1 ? R.q + (long long)(p - 1) * 2 * R.M : nullptr;
            a.acc = R.acc;
            a.acc_init = i == (R.N - 1 + 1) / 2 ? 1 : 0;  // the first step with p <= i + 1
            a.a_is_A = i + 1 <= R.NA;
            a.b_is_A = p <= R.NA;
        }
    }
    pencil_body<float, NX, CW, MODE>(a, blockIdx.x, 0);
}

// Q's per-plane partials from slot N of every member (plane_q_sums_kernel
// per replica): grid (mx, members)
__global__ void __launch_bounds__(256) ens_plane_q_sums_kernel(EnsRep *__restrict__ reps, const int *__restrict__ members)
{
    const EnsRep &R = reps[members[blockIdx.y]];
    if (!R.active || (int)blockIdx.x >= R.mx) return;
    plane_q_sums_body(reinterpret_cast<const float2 *>(R.q + (long long)(R.N - 1) * 2 * R.M),
                      (long long)R.my * R.mz, R.qpart, blockIdx.x);
}

template <int NX, int CW>
__global__ void __launch_bounds__(PencilCfg<float, NX, CW>::NT)
    ens_pencil_kernel(EnsRep *__restrict__ reps, const int *__restrict__ members)
{
    const EnsRep &R = reps[members[blockIdx.y]];
    if (!R.active) return;
    PencilArgs<float> a{};
    a.spec = R.spec;
    a.twx = R.tw[0];
    a.gx = R.g[0];
    a.gy = R.g[1];
    a.gz = R.g[2];
    a.ncol = R.my * R.mz;
    a.KZ = R.mz;
    pencil_body<float, NX, CW, PENCIL_CONV>(a, blockIdx.x, 0);
}

// Q and ln Q of every active replica (as q_finalize_kernel, 256 threads)
__global__ void __launch_bounds__(256) ens_qfinal_kernel(EnsRep *__restrict__ reps)
{
    const EnsRep &R = reps[blockIdx.x];
    if (!R.active) return;
    __shared__ double sh[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < R.mx; i += blockDim.x) s += R.qpart[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
        const double Q = s / (double)R.M;
        R.Qd[0] = Q;
        R.Qd[1] = log(Q);
    }
}

// phi, the residual Dh0 and its dot products: grid (max red_blocks, nrep), or
// (max red_blocks, group size) over `members`
__global__ void __launch_bounds__(kRedThreads, 4) ens_conc_kernel(EnsRep *__restrict__ reps,
                                                                  const int *__restrict__ members)
{
    const EnsRep &R = reps[members ? members[blockIdx.y] : blockIdx.y];
    if (!R.active || (int)blockIdx.x >= R.red_blocks) return;
    const int nh = ens_nh(R.k);
    HistPtrs hist{};
    for (int m = 1; m <= nh; m++) hist.p[m - 1] = R.Dh[R.phys[m]];
    if (R.acc)  // phi from the sums the chain formed (concentrations_acc_kernel)
        concentrations_acc_body(R.acc, R.q, R.M, R.N, R.w + 2 * R.M, R.w + 3 * R.M, R.Qd, R.Dh[R.cur], nh, hist,
                                R.partials, blockIdx.x, R.red_blocks);
    else
        concentrations_body<float>(R.q, R.M, R.N, R.NA, R.w, R.w + 2 * R.M, R.w + 3 * R.M, R.Qd, R.Dh[R.cur], nh,
                                   hist, R.partials, blockIdx.x, R.red_blocks);
}

// One replica per block: the reduction of its dot products (as
// reduce_partials_kernel, 256 threads, fixed order), then on one warp the
// scalar part of the Anderson iteration (src/anderson.cc:35-89): the row
// DD[0][0..nh], the least-squares coefficients (k >= 2), the DD bookkeeping
// and whether the loop goes on (err > tol and k + 1 < maxIter).  In the
// iteration after the loop stopped (the extra calc_concs) it only marks the
// replica done.
__global__ void __launch_bounds__(256) ens_reduce_solve_kernel(EnsRep *__restrict__ reps, double tol, int maxIter)
{
    EnsRep &R = reps[blockIdx.x];
    if (!R.active) return;
    if (R.stopped) {
        if (threadIdx.x == 0) {
            R.go = 0;
            R.done = 1;
        }
        return;
    }
    anderson_reduce_solve(R, R.partials, R.red_blocks, R.M, tol, maxIter);
}

// w+ update (src/anderson.cc:57-79): grid (max red_blocks, nrep); lambda[k] =
// 1 - 0.9^k from the host
__global__ void __launch_bounds__(256) ens_update_kernel(EnsRep *__restrict__ reps, const double *__restrict__ lambda)
{
    const EnsRep &R = reps[blockIdx.y];
    if (!R.active || !R.go || (int)blockIdx.x >= R.red_blocks) return;
    const int nh = ens_nh(R.k);
    HistPtrs Dhp{}, whp{};
    for (int m = 1; m <= nh; m++) {
        Dhp.p[m - 1] = R.Dh[R.phys[m]];
        whp.p[m - 1] = R.wh[R.phys[m]];
    }
    anderson_update_body<float>(R.w + R.M, R.wh[R.cur], R.Dh[R.cur], R.M, lambda[R.k], nh, R.simple, Dhp, whp, R.coef,
                         blockIdx.x, R.red_blocks);
}

// After each body iteration: history rotation (src/anderson.cc:82-89) and
// the next iteration number of every active replica; replicas whose extra
// iteration just ran become idle.  Ends the WHILE loop when none is active.
// guard[0] counts the body iterations of this mix; past `cap` (more than any
// replica's loop can take: maxIter + 2) the loop ends regardless and the
// replicas still active are marked (sticky bit 8), so no error in the
// bookkeeping above can keep the WHILE node running.
__global__ void ens_control_kernel(EnsRep *__restrict__ reps, int nrep, cudaGraphConditionalHandle loop, int *guard,
                                   int cap)
{
    __shared__ int any, cut;
    if (threadIdx.x == 0) {
        any = 0;
        cut = ++guard[0] >= cap;
    }
    __syncthreads();
    if (cut) {
        for (int r = threadIdx.x; r < nrep; r += blockDim.x) {
            EnsRep &R = reps[r];
            if (!R.active) continue;
            R.active = 0;
            R.iters = R.k;
            R.sticky |= 8;
        }
        __syncthreads();
        if (threadIdx.x == 0) cudaGraphSetConditional(loop, 0u);
        return;
    }
    for (int r = threadIdx.x; r < nrep; r += blockDim.x) {
        EnsRep &R = reps[r];
        if (!R.active) continue;
        if (R.done) {
            R.active = 0;
            R.iters = R.k;
            R.sticky |= (R.notconv ? 1 : 0) | (R.singular ? 2 : 0) | (R.nonfinite ? 4 : 0);
            continue;
        }
        if (R.go) {
            const int n = 1 + (R.k - 1) % kMaxHist;
            const int evicted = R.phys[n];
            R.phys[n] = R.cur;
            R.cur = evicted;
        }
        R.k++;
        any = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) cudaGraphSetConditional(loop, any ? 1u : 0u);
}

// start of a mix: every replica active at iteration 1, the iteration guard
// at zero; with advance, the Langevin step counter moves on (after this
// step's update used it); with set_inner (a mix nested in a run's step
// loop), the mix's WHILE condition is raised again for this step
__global__ void ens_begin_kernel(EnsRep *__restrict__ reps, int nrep, long long *step, int advance, int *guard,
                                 int set_inner, cudaGraphConditionalHandle inner)
{
    for (int r = threadIdx.x; r < nrep; r += blockDim.x) {
        EnsRep &R = reps[r];
        R.k = 1;
        R.active = 1;
        R.stopped = R.done = R.go = R.singular = R.notconv = R.nonfinite = 0;
    }
    if (threadIdx.x == 0) {
        if (advance) *step += 1;
        if (guard) guard[0] = 0;
        if (set_inner) cudaGraphSetConditional(inner, 1u);
    }
}

// end of one step of a run: records every replica's Anderson count for this
// step (kbuf[step][replica]), counts the step and keeps the step loop going
// while run[0] (steps done) < run[1] (steps asked for)
__global__ void ens_step_end_kernel(const EnsRep *__restrict__ reps, int nrep, int *run, int *kbuf,
                                    cudaGraphConditionalHandle outer)
{
    const int s = run[0];
    for (int r = threadIdx.x; r < nrep; r += blockDim.x) kbuf[(long long)s * nrep + r] = reps[r].iters;
    __syncthreads();
    if (threadIdx.x == 0) {
        run[0] = s + 1;
        cudaGraphSetConditional(outer, s + 1 < run[1] ? 1u : 0u);
    }
}

// clears the replicas' status bits at the start of a host call (mix or run)
__global__ void ens_clear_status_kernel(EnsRep *__restrict__ reps, int nrep)
{
    for (int r = threadIdx.x; r < nrep; r += blockDim.x) reps[r].sticky = 0;
}

// W- += -(phi- + 2 W-/XbN) dt + (eta_prev + eta_new)/2 (src/langevin.cc:31),
// the noise of steps s-1 and s regenerated from the counter: grid (blocks, nrep)
__global__ void __launch_bounds__(256) ens_langevin_kernel(EnsRep *__restrict__ reps, const long long *step)
{
    const EnsRep &R = reps[blockIdx.y];
    const long long s = *step;
    double *w = R.w;
    const long long M = R.M;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < M; r += stride) {
        const double ep = philox_noise(R.seed, s - 1, r, R.sigma);
        const double en = philox_noise(R.seed, s, r, R.sigma);
        const double wm = w[r], pm = w[2 * M + r];
        const double drift = __dmul_rn(-__dadd_rn(pm, __ddiv_rn(__dmul_rn(2.0, wm), R.XbN)), R.dt);
        const double noise = __dmul_rn(0.5, __dadd_rn(ep, en));
        w[r] = __dadd_rn(wm, __dadd_rn(drift, noise));
    }
}

// the noise sigma * z of points [0, n) of step s (for callers that feed it to
// a single context, and for tests)
__global__ void philox_noise_kernel(unsigned long long seed, long long s, long long n, double sigma, double *out)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride)
        out[r] = philox_noise(seed, s, r, sigma);
}

}  // namespace lfts
