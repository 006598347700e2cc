// C ABI of the B200 L-FTS step (include/lfts_b200.h): device state, launch
// orchestration and the small host-side pieces (Anderson least squares,
// S(k) bin tables) around the kernels in fft_kernels.cuh / field_kernels.cuh.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <tuple>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lfts_b200.h"
#include "anderson_device.cuh"
#include "ctx.h"
#include "fft_dispatch.h"
#include "field_kernels.cuh"

using namespace lfts;

namespace {

thread_local std::string g_last_error = "";

int cuda_fail(cudaError_t e, const char *what)
{
    char buf[512];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    g_last_error = buf;
    return LFTS_ERR_CUDA;
}

#define CK(call)                                           \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

constexpr double kTwoPi = 6.283185307179586476925286766559005768;
// x-pencil tile widths used when autotuning is off (the usual winners at 128^3)
constexpr int kDefaultCwFp32 = 16, kDefaultCwFp64 = 32;

// Gaussian elimination with partial pivoting (first maximal |pivot|,
// reciprocal scaling of the sub-column, right-looking rank-1 updates), then
// forward/back substitution: the LU solve the reference does with GSL at
// src/anderson.cc:106-127.  Returns false for an exactly singular matrix,
// where GSL's solve reports an error.
bool lu_solve(std::vector<double> A, std::vector<double> y, double *x, int n)
{
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    for (int j = 0; j < n; j++) {
        int piv = j;
        double amax = std::fabs(A[j * n + j]);
        for (int i = j + 1; i < n; i++) {
            double v = std::fabs(A[i * n + j]);
            if (v > amax) { amax = v; piv = i; }
        }
        if (piv != j) {
            for (int k = 0; k < n; k++) std::swap(A[j * n + k], A[piv * n + k]);
            std::swap(perm[j], perm[piv]);
        }
        if (j + 1 < n) {
            const double ajj = A[j * n + j];
            if (std::fabs(ajj) >= 2.2250738585072014e-308) {
                const double inv = 1.0 / ajj;
                for (int i = j + 1; i < n; i++) A[i * n + j] *= inv;
            } else {
                for (int i = j + 1; i < n; i++) A[i * n + j] /= ajj;
            }
            for (int i = j + 1; i < n; i++) {
                const double lij = A[i * n + j];
                for (int k = j + 1; k < n; k++) A[i * n + k] -= lij * A[j * n + k];
            }
        }
    }
    for (int i = 0; i < n; i++)
        if (A[i * n + i] == 0.0) return false;
    for (int i = 0; i < n; i++) x[i] = y[perm[i]];
    for (int i = 0; i < n; i++) {
        double t = x[i];
        for (int j = 0; j < i; j++) t -= A[i * n + j] * x[j];
        x[i] = t;
    }
    for (int i = n - 1; i >= 0; i--) {
        double t = x[i];
        for (int j = i + 1; j < n; j++) t -= A[i * n + j] * x[j];
        x[i] = t / A[i * n + i];
    }
    return true;
}

// signed wavenumber of index K in [0, m): -(m-1)/2 .. m/2 (src/step.cc:69-79)
inline int signed_k(int K, int m) { return (K <= m / 2) ? K : K - m; }

}  // namespace

// shared with lfts_noalloc.cu, which reports through lfts_last_error_string
void lfts_internal_set_error(const char *msg) { g_last_error = msg; }


namespace {

template <typename T>
PlaneKernels<T> &plane_of(lfts_ctx *c);
template <>
PlaneKernels<double> &plane_of<double>(lfts_ctx *c) { return c->pl64; }
template <>
PlaneKernels<float> &plane_of<float>(lfts_ctx *c) { return c->pl32; }
template <typename T>
PencilKernels<T> &pencil_of(lfts_ctx *c);
template <>
PencilKernels<double> &pencil_of<double>(lfts_ctx *c) { return c->pe64; }
template <>
PencilKernels<float> &pencil_of<float>(lfts_ctx *c) { return c->pe32; }

template <typename T>
int set_smem_attrs(const PlaneKernels<T> &pl, const PencilKernels<T> &pe)
{
    for (int m = 0; m < kPlaneModes; m++)
        if (pl.fn[m]) CK(cudaFuncSetAttribute(pl.fn[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem));
    for (int m = 0; m < kPencilModes; m++)
        if (pe.fn[m]) CK(cudaFuncSetAttribute(pe.fn[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pe.smem));
    return LFTS_OK;
}

template <typename T>
int upload_tables(lfts_ctx *c, void **tw, void **gt)
{
    const int m[3] = {c->mx, c->my, c->mz};
    for (int d = 0; d < 3; d++) {
        std::vector<cpx<T>> t(m[d]);
        for (int k = 0; k < m[d]; k++) {
            long double a = -(long double)kTwoPi * (long double)k / (long double)m[d];
            t[k].x = (T)(double)cosl(a);
            t[k].y = (T)(double)sinl(a);
        }
        CK(cudaMalloc(&tw[d], sizeof(cpx<T>) * m[d]));
        CK(cudaMemcpy(tw[d], t.data(), sizeof(cpx<T>) * m[d], cudaMemcpyHostToDevice));
    }
    if (!gt) return LFTS_OK;
    // g = exp(-(2 pi)^2 (kx^2/Lx^2 + ky^2/Ly^2 + kz^2/Lz^2)/(6N)) / M, factorised;
    // the packed (full complex) spectrum needs kz over [0, mz), signed
    const int n[3] = {c->mx, c->my, c->packed ? c->mz : c->KZ};
    for (int d = 0; d < 3; d++) {
        std::vector<T> g(n[d]);
        for (int K = 0; K < n[d]; K++) {
            const int k = (d == 2 && !c->packed) ? K : signed_k(K, m[d]);
            const double ksq = (double)k * k / (c->p.L[d] * c->p.L[d]);
            double v = std::exp(-kTwoPi * kTwoPi * ksq / (6.0 * c->N));
            if (d == 2) v /= (double)c->M;
            g[K] = (T)v;
        }
        CK(cudaMalloc(&gt[d], sizeof(T) * n[d]));
        CK(cudaMemcpy(gt[d], g.data(), sizeof(T) * n[d], cudaMemcpyHostToDevice));
    }
    return LFTS_OK;
}

inline dim3 stream_grid(const lfts_ctx *c) { return dim3(c->red_blocks); }
// element-wise passes with no cross-block reduction (the Anderson w+ update,
// the Langevin update): a full wave of 256-thread CTAs, so more loads are in
// flight per SM
inline dim3 update_grid(const lfts_ctx *c) { return dim3(c->sms * 8); }

// ---- contour chain ----------------------------------------------------------
template <typename T>
PlaneArgs<T> plane_args(lfts_ctx *c)
{
    PlaneArgs<T> a{};
    a.w = c->w;
    a.spec = static_cast<cpx<T> *>(c->spec);
    a.twy = static_cast<const cpx<T> *>(c->tw[1]);
    a.twz = static_cast<const cpx<T> *>(c->tw[2]);
    a.qpart = c->qpart;
    a.nchains = 2;
    a.Nd = (double)c->N;
    a.gx = static_cast<const T *>(c->gtab[0]);
    a.gy = static_cast<const T *>(c->gtab[1]);
    a.gz = static_cast<const T *>(c->gtab[2]);
    return a;
}

template <typename T>
PencilArgs<T> pencil_args(lfts_ctx *c)
{
    PencilArgs<T> a{};
    a.spec = static_cast<cpx<T> *>(c->spec);
    a.twx = static_cast<const cpx<T> *>(c->tw[0]);
    a.gx = static_cast<const T *>(c->gtab[0]);
    a.gy = static_cast<const T *>(c->gtab[1]);
    a.gz = static_cast<const T *>(c->gtab[2]);
    a.ncol = c->my * (c->packed ? c->mz : c->KZ);
    a.KZ = c->packed ? c->mz : c->KZ;
    a.w = c->w;
    a.h = static_cast<const T *>(c->q);  // slot 1: the (hA, hB) pairs
    a.M = c->M;
    a.Nd = (double)c->N;
    return a;
}

// Chain kernels go out with programmatic stream serialisation (see pdl_wait in
// fft_kernels.cuh): each may be scheduled while its predecessor drains.
template <typename K, typename A>
void launch_pdl(lfts_ctx *c, K kernel, dim3 grid, int nt, size_t smem, const A &args, cudaStream_t st = nullptr)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(nt);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st ? st : c->st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = c->use_pdl ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args);
    c->launches++;
}

// In packed mode one launch covers both chains (gridDim.y = 1).
template <typename T>
void launch_plane(lfts_ctx *c, int mode, const PlaneArgs<T> &a, int nchains, cudaStream_t st = nullptr)
{
    if constexpr (sizeof(T) == sizeof(float)) {
        if (mode == PLANE_G && c->plane_split > 1) {
            launch_pdl(c, c->psplit.fn, dim3(c->mx * c->psplit.cl), c->psplit.nt, c->psplit.smem, a, st);
            return;
        }
    }
    const PlaneKernels<T> &pl = plane_of<T>(c);
    const int extra = mode == PLANE_G ? a.pf_ctas : 0;
    launch_pdl(c, pl.fn[mode], dim3(c->mx + extra, c->packed ? 1 : nchains), pl.nt, pl.smem, a, st);
}

template <typename T>
void launch_pencil(lfts_ctx *c, int mode, const PencilArgs<T> &a, int nchains, cudaStream_t st = nullptr)
{
    const PencilKernels<T> &pe = pencil_of<T>(c);
    launch_pdl(c, pe.fn[mode], dim3((a.ncol + pe.cw - 1) / pe.cw, c->packed ? 1 : nchains), pe.nt, pe.smem, a,
               st);
}

inline int hsel_chain0(const lfts_ctx *c, int i) { return i < c->NA ? 0 : 1; }  // src/step.cc:53-57
inline int hsel_chain1(const lfts_ctx *c, int i) { return i < c->NB ? 1 : 0; }  // src/step.cc:60-64

template <typename T>
void enqueue_chain_launches(lfts_ctx *c);

// The chain's launches have fixed arguments for the life of the context, so
// they are captured once into a CUDA graph (programmatic-launch edges
// included) and replayed: one launch per calc_concs instead of ~2N.
template <typename T>
void enqueue_chain(lfts_ctx *c)
{
    if (!c->use_graph) {
        enqueue_chain_launches<T>(c);
        return;
    }
    if (!c->chain_exec) {
        const long long before = c->launches;
        cudaError_t e = cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            enqueue_chain_launches<T>(c);
            cudaGraph_t g = nullptr;
            e = cudaStreamEndCapture(c->st, &g);
            if (e == cudaSuccess && g) e = cudaGraphInstantiate(&c->chain_exec, g, 0);
            if (e == cudaSuccess && c->chain_exec) {
                c->chain_graph = g;
                c->chain_kernels = c->launches - before;
                // upload before the first replay and let both streams drain
                e = cudaGraphUpload(c->chain_exec, c->st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(c->st1);
            } else {
                if (g) cudaGraphDestroy(g);
                c->chain_exec = nullptr;
            }
        }
        if (e != cudaSuccess) cuda_fail(e, "chain graph capture");
        c->launches = before;
        cudaGetLastError();  // a failed capture falls back to direct launches below
        if (!c->chain_exec) {
            c->use_graph = false;
            enqueue_chain_launches<T>(c);
            return;
        }
    }
    cudaError_t e = cudaGraphLaunch(c->chain_exec, c->st);
    if (e != cudaSuccess) {
        cuda_fail(e, "cudaGraphLaunch(chain)");
        fprintf(stderr, "lfts: %s\n", g_last_error.c_str());
    }
    c->launches += c->chain_kernels;
}

// propagators of both chains for all N monomers, then Q (src/diblock.cc:36-48).
// The two chains (q and q^) are independent until the concentrations, so
// each runs its own launch sequence on its own stream (st: q, st1: q^) and
// one chain's kernels fill the other's tails; with one stream both chains
// share every launch.
template <typename T>
void enqueue_chain_launches(lfts_ctx *c)
{
    T *q = static_cast<T *>(c->q);
    const long long M = c->M;
    PlaneArgs<T> a = plane_args<T>(c);
    PencilArgs<T> pa = pencil_args<T>(c);
    if constexpr (sizeof(T) == sizeof(float)) {
        if (c->xh_chain) {
            // One step is q_{i+1} = h . F^-1[g . F[q_i]].  g is even in every
            // wavenumber, so F^-1[g F[q]] = F[g F^-1[q]]; with D_i = F_x^-1[q_i]
            // in the spectrum buffer a step is
            //   yz-plane (PLANE_G):  E_i = F_yz[g . F_yz^-1[D_i]]  (the STEP flow, g for h)
            //   x-pencil (PENCIL_H): q_{i+1} = h . F_x[E_i], stored; D_{i+1} = F_x^-1[q_{i+1}]
            // which puts the h loads and q stores in the pencil's several CTAs
            // per SM instead of the plane kernel's one.
            PencilArgs<T> pi = pa;
            pi.qout = q;  // slot 1 = (hA, hB)
            launch_pencil<T>(c, PENCIL_INIT_W, pi, 2);
            // With phi in the chain, the concentration sums are formed as the
            // slots are made: slot i+1 = (q_{i+1}, q^_{N-i}) pairs with slot
            // N-i = (q_{N-i}, q^_{i+1}).  From the middle of the chain on that
            // partner is already stored, so the pencil adds the two products
            // into acc and slot i+1 need not be stored (except slot N, for Q);
            // the middle slot of an odd chain pairs with itself.
            const bool acc = c->phi_in_chain;
            bool first_acc = true;
            for (int i = 1; i < c->N; i++) {
                PlaneArgs<T> ag = a;
                if (acc && c->N - i < i + 1) {
                    ag.pf = q + (long long)(c->N - i - 1) * 2 * M;  // the partner slot
                    if (c->plane_split == 1) ag.pf_ctas = c->pf_ctas;
                }
                launch_plane<T>(c, PLANE_G, ag, 2);
                PencilArgs<T> ph = pa;
                ph.qout = q + (long long)i * 2 * M;  // slot i+1
                ph.hsel0 = hsel_chain0(c, i);
                ph.hsel1 = hsel_chain1(c, i);
                const int p = c->N - i;  // partner slot
                if (!acc || p > i + 1) {
                    launch_pencil<T>(c, i + 1 < c->N ? PENCIL_H : PENCIL_H_LAST, ph, 2);
                    continue;
                }
                ph.partner = p < i + 1 ? q + (long long)(p - 1) * 2 * M : nullptr;
                ph.acc = static_cast<T *>(c->acc);
                ph.acc_init = first_acc ? 1 : 0;
                ph.a_is_A = i + 1 <= c->NA;
                ph.b_is_A = p <= c->NA;
                first_acc = false;
                launch_pencil<T>(c, i + 1 < c->N ? PENCIL_HA : PENCIL_HA_LAST, ph, 2);
            }
            plane_q_sums_kernel<<<c->mx, 256, 0, c->st>>>(
                reinterpret_cast<const float2 *>(q + (long long)(c->N - 1) * 2 * M), (long long)c->my * c->mz,
                c->qpart);
            q_finalize_kernel<<<1, 256, 0, c->st>>>(c->qpart, c->mx, M, c->Qd);
            c->launches += 2;
            return;
        }
    }
    if (!c->two_streams || c->packed) {
        a.qout = q;  // slot 1 = [hA | hB]
        launch_plane<T>(c, PLANE_INIT_W, a, 2);
        a.h = q;
        for (int i = 1; i < c->N; i++) {
            launch_pencil<T>(c, PENCIL_CONV, pa, 2);
            a.qout = q + (long long)i * 2 * M;  // slot i+1
            a.hsel0 = hsel_chain0(c, i);
            a.hsel1 = hsel_chain1(c, i);
            launch_plane<T>(c, i + 1 < c->N ? PLANE_STEP : PLANE_LAST, a, 2);
        }
    } else {
        cudaEventRecord(c->ev_fork, c->st);
        cudaStreamWaitEvent(c->st1, c->ev_fork, 0);
        cudaStream_t sc[2] = {c->st, c->st1};
        PlaneArgs<T> ac[2] = {a, a};
        PencilArgs<T> pc[2] = {pa, pa};
        for (int k = 0; k < 2; k++) {
            ac[k].cbase = k;
            pc[k].cbase = k;
            ac[k].qout = q;
            launch_plane<T>(c, PLANE_INIT_W, ac[k], 1, sc[k]);
            ac[k].h = q;
        }
        // Each stream's INIT_W writes its own half of h (hA from chain 1, hB from
        // chain 2), and each chain's steps read the other half once i >= NA
        // (chain 1) or i >= NB (chain 2): both halves are complete before either
        // chain's first step.
        for (int k = 0; k < 2; k++) cudaEventRecord(c->ev_h[k], sc[k]);
        for (int k = 0; k < 2; k++) cudaStreamWaitEvent(sc[k], c->ev_h[1 - k], 0);
        for (int i = 1; i < c->N; i++) {
            for (int k = 0; k < 2; k++) launch_pencil<T>(c, PENCIL_CONV, pc[k], 1, sc[k]);
            for (int k = 0; k < 2; k++) {
                ac[k].qout = q + (long long)i * 2 * M;
                ac[k].hsel0 = hsel_chain0(c, i);
                ac[k].hsel1 = hsel_chain1(c, i);
                launch_plane<T>(c, i + 1 < c->N ? PLANE_STEP : PLANE_LAST, ac[k], 1, sc[k]);
            }
        }
        cudaEventRecord(c->ev_join, c->st1);
        cudaStreamWaitEvent(c->st, c->ev_join, 0);
    }
    q_finalize_kernel<<<1, 256, 0, c->st>>>(c->qpart, c->mx, M, c->Qd);
    c->launches++;
}

template <typename T>
void enqueue_concs(lfts_ctx *c, void *Dh0, int nh, const HistPtrs &hist)
{
    enqueue_chain<T>(c);
    if (c->phi_in_chain)
        concentrations_acc_kernel<<<stream_grid(c), kRedThreads, 0, c->st>>>(
            static_cast<const float *>(c->acc), static_cast<const float *>(c->q), c->M, c->N, c->w + 2 * c->M,
            c->w + 3 * c->M, c->Qd, static_cast<float *>(Dh0), nh, hist, c->partials);
    else
        concentrations_kernel<T><<<stream_grid(c), kRedThreads, 0, c->st>>>(
            static_cast<const T *>(c->q), c->M, c->N, c->NA, c->w, c->w + 2 * c->M, c->w + 3 * c->M, c->Qd,
            static_cast<T *>(Dh0), nh, hist, c->partials);
    c->launches++;
    if (Dh0) {
        reduce_partials_kernel<<<nh + 1, 256, 0, c->st>>>(c->partials, c->red_blocks, nh + 1, c->red);
        c->launches++;
    }
}

void enqueue_chain_any(lfts_ctx *c)
{
    if (c->prec == LFTS_FP64)
        enqueue_chain<double>(c);
    else
        enqueue_chain<float>(c);
}

void enqueue_concs_any(lfts_ctx *c, void *Dh0, int nh, const HistPtrs &hist)
{
    if (c->prec == LFTS_FP64)
        enqueue_concs<double>(c, Dh0, nh, hist);
    else
        enqueue_concs<float>(c, Dh0, nh, hist);
}

// ---- tile choices and their autotuner ------------------------------------------
// A context's contour chain has these free choices, none of which changes what
// is computed (each is tested against the others at the precision's tolerance;
// the x-pencil width changes no column's arithmetic at all):
//   pencil_cw     x-pencil columns per CTA (8, 16, 32)
//   plane_stages  FP32-mixed yz-plane transform stages per axis: 3 (fft_plane3.cuh,
//                 64 / 96 / 128 square planes) or 2 (fft_packed.cuh)
//   h_in_pencil   FP32-mixed: h and the propagator stores in the x-pencil and g in
//                 the yz-plane kernel (96- and 128-point x lines, three-stage planes),
//                 or both in the yz-plane kernel
//   two_streams   FP64: each chain on its own stream, or both chains per launch
// autotune() times the whole chain for every valid combination on the
// context's own buffers (a tile's cost depends on how it overlaps its
// neighbours in the chain, so it is timed in place) and keeps the fastest,
// once per (precision, mesh) per process -- the reference's analogue is
// planning its FFTs with FFTW_PATIENT (src/step.cc:15-16).
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, lfts_tiles> g_tuned;

template <typename T>
int set_pencil(lfts_ctx *c, int cw)
{
    PencilKernels<T> pk{};
    if (!pencil_kernels(c->mx, cw, &pk)) return LFTS_ERR_UNSUPPORTED;
    for (int m = 0; m < kPencilModes; m++)
        if (pk.fn[m]) CK(cudaFuncSetAttribute(pk.fn[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pk.smem));
    pencil_of<T>(c) = pk;
    return LFTS_OK;
}

// the captured chain and the Anderson-loop graph that holds it (rebuilt on
// the next use with the new tiles)
void drop_chain_graph(lfts_ctx *c)
{
    if (c->chain_exec) cudaGraphExecDestroy(c->chain_exec);
    if (c->chain_graph) cudaGraphDestroy(c->chain_graph);
    c->chain_exec = nullptr;
    c->chain_graph = nullptr;
    if (c->mix_exec) cudaGraphExecDestroy(c->mix_exec);
    if (c->mix_graph) cudaGraphDestroy(c->mix_graph);
    c->mix_exec = nullptr;
    c->mix_graph = nullptr;
    if (c->mix_graph_state == 1) c->mix_graph_state = 0;
}

// installs a tile choice (validated); the chain graph is captured anew
int apply_tiles(lfts_ctx *c, const lfts_tiles &t)
{
    if (t.pencil_cw != 8 && t.pencil_cw != 16 && t.pencil_cw != 32) return LFTS_ERR_ARG;
    const int split = t.plane_split == 0 ? 1 : t.plane_split;
    if (split != 1 && split != 8) return LFTS_ERR_ARG;
    if (c->prec == LFTS_FP64) {
        if (t.plane_stages != 2 || t.h_in_pencil != 0 || (t.two_streams != 0 && t.two_streams != 1) ||
            t.phi_in_chain != 0 || split != 1)
            return LFTS_ERR_ARG;
        int rc = set_pencil<double>(c, t.pencil_cw);
        if (rc) return rc;
        c->two_streams = t.two_streams == 1;
    } else {
        if ((t.plane_stages != 2 && t.plane_stages != 3) || (t.h_in_pencil != 0 && t.h_in_pencil != 1) ||
            t.two_streams != 0 || (t.phi_in_chain != 0 && t.phi_in_chain != 1) || (t.phi_in_chain && !t.h_in_pencil))
            return LFTS_ERR_ARG;
        PlaneKernels<float> pl{};
        const bool ok = t.plane_stages == 3 ? plane3_kernels(c->my, c->mz, &pl) : plane_c_kernels(c->my, c->mz, &pl);
        if (!ok) return LFTS_ERR_UNSUPPORTED;
        PencilKernels<float> pk{};
        if (!pencil_kernels(c->mx, t.pencil_cw, &pk)) return LFTS_ERR_UNSUPPORTED;
        if (t.h_in_pencil && !(pl.fn[PLANE_G] && pk.fn[PENCIL_H])) return LFTS_ERR_UNSUPPORTED;
        if (t.phi_in_chain && !(pk.fn[PENCIL_HA] && pk.fn[PENCIL_HA_LAST])) return LFTS_ERR_UNSUPPORTED;
        PlaneSplitKernel ps{};
        if (split > 1) {
            // the cluster kernel replaces PLANE_G of the three-stage plane
            if (!(t.h_in_pencil && t.plane_stages == 3 && plane_split_kernel(c->my, c->mz, &ps) && ps.cl == split))
                return LFTS_ERR_UNSUPPORTED;
            CK(cudaFuncSetAttribute(ps.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps.smem));
        }
        if (t.phi_in_chain && !c->acc) {
            // the (A, B) concentration sums, FP32 pairs per mesh point
            cudaError_t e = cudaMalloc(&c->acc, sizeof(float) * 2 * (size_t)c->M);
            if (e != cudaSuccess) {
                cudaGetLastError();
                c->acc = nullptr;
                g_last_error = "device allocation of the concentration sums failed";
                return LFTS_ERR_NOMEM;
            }
        }
        for (int m = 0; m < kPlaneModes; m++)
            if (pl.fn[m]) CK(cudaFuncSetAttribute(pl.fn[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem));
        int rc = set_pencil<float>(c, t.pencil_cw);
        if (rc) return rc;
        c->pl32 = pl;
        c->psplit = ps;
        c->plane_split = split;
        c->plane_stages = t.plane_stages;
        c->xh_chain = t.h_in_pencil == 1;
        c->phi_in_chain = t.phi_in_chain == 1;
    }
    drop_chain_graph(c);
    return LFTS_OK;
}

lfts_tiles current_tiles(const lfts_ctx *c)
{
    lfts_tiles t{};
    const bool fp64 = c->prec == LFTS_FP64;
    t.pencil_cw = fp64 ? c->pe64.cw : c->pe32.cw;
    t.plane_stages = fp64 ? 2 : c->plane_stages;
    t.h_in_pencil = (!fp64 && c->xh_chain) ? 1 : 0;
    t.two_streams = (fp64 && c->two_streams) ? 1 : 0;
    t.phi_in_chain = (!fp64 && c->phi_in_chain) ? 1 : 0;
    t.plane_split = fp64 ? 1 : c->plane_split;
    return t;
}

// every valid combination for this context, restricted by the environment
// (LFTS_PENCIL_CW, LFTS_XH_CHAIN, LFTS_ONE_STREAM, LFTS_PHI_IN_CHAIN fix one
// choice each)
std::vector<lfts_tiles> tile_candidates(const lfts_ctx *c)
{
    std::vector<lfts_tiles> out;
    const char *fcw = std::getenv("LFTS_PENCIL_CW");
    const char *fxh = std::getenv("LFTS_XH_CHAIN");
    const char *fone = std::getenv("LFTS_ONE_STREAM");
    const char *fphi = std::getenv("LFTS_PHI_IN_CHAIN");
    const char *fsplit = std::getenv("LFTS_PLANE_SPLIT");
    const int split_forced = fsplit ? std::atoi(fsplit) : 0;
    PlaneSplitKernel ps{};
    const bool has_split = c->prec != LFTS_FP64 && plane_split_kernel(c->my, c->mz, &ps);
    const int cw_forced = fcw ? std::atoi(fcw) : 0;
    for (int cw : {8, 16, 32}) {
        if (cw_forced > 0 && cw != cw_forced) continue;
        if (c->prec == LFTS_FP64) {
            for (int two : {1, 0}) {
                if (fone && ((fone[0] == '1') == (two == 1))) continue;
                out.push_back({cw, 2, 0, two, 0, 1});
            }
            continue;
        }
        PlaneKernels<float> p3{};
        PencilKernels<float> pk{};
        const bool has3 = plane3_kernels(c->my, c->mz, &p3);
        const bool hasx = has3 && p3.fn[PLANE_G] && pencil_kernels(c->mx, cw, &pk) && pk.fn[PENCIL_H];
        const bool hasa = hasx && pk.fn[PENCIL_HA] && pk.fn[PENCIL_HA_LAST];
        for (int st : {3, 2}) {
            if (st == 3 && !has3) continue;
            for (int xh : {1, 0}) {
                if (xh && (st != 3 || !hasx)) continue;
                if (fxh && ((fxh[0] != '0') != (xh == 1))) continue;
                for (int phi : {0, 1}) {
                    if (phi && (!xh || !hasa)) continue;
                    if (fphi && ((fphi[0] != '0') != (phi == 1))) continue;
                    // LFTS_PLANE_SPLIT applies where the cluster kernel does
                    const bool can_split = xh && has_split && ps.cl == 8;
                    for (int split : {1, 8}) {
                        if (split > 1 && !can_split) continue;
                        if (split_forced > 0 && can_split && split != split_forced) continue;
                        out.push_back({cw, st, xh, 0, phi, split});
                    }
                }
            }
        }
    }
    return out;
}

// the choice used when autotuning is off: three-stage planes and h in the
// x-pencil where compiled, the usual pencil winners, two FP64 streams
lfts_tiles default_tiles(const lfts_ctx *c)
{
    std::vector<lfts_tiles> cand = tile_candidates(c);
    const int cw = c->prec == LFTS_FP64 ? kDefaultCwFp64 : kDefaultCwFp32;
    for (const lfts_tiles &t : cand)
        if (t.pencil_cw == cw) return t;  // candidates come best-guess first
    return cand.empty() ? lfts_tiles{cw, 2, 0, c->prec == LFTS_FP64 ? 1 : 0, 0, 1} : cand.front();
}

// one calc_concs without the Anderson dot products: the chain, then the
// concentrations from the stored slots or from the sums the chain formed
template <typename T>
void enqueue_calc(lfts_ctx *c)
{
    enqueue_chain_launches<T>(c);
    if (c->phi_in_chain)
        concentrations_acc_kernel<<<stream_grid(c), kRedThreads, 0, c->st>>>(
            static_cast<const float *>(c->acc), static_cast<const float *>(c->q), c->M, c->N, c->w + 2 * c->M,
            c->w + 3 * c->M, c->Qd, nullptr, 0, HistPtrs{}, c->partials);
    else
        concentrations_kernel<T><<<stream_grid(c), kRedThreads, 0, c->st>>>(
            static_cast<const T *>(c->q), c->M, c->N, c->NA, c->w, c->w + 2 * c->M, c->w + 3 * c->M, c->Qd, nullptr,
            0, HistPtrs{}, c->partials);
}

// a tile choice is timed on whole calc_concs (chain + concentrations): the
// choices differ in how the concentration work is split between them
template <typename T>
int time_chain(lfts_ctx *c, cudaEvent_t e0, cudaEvent_t e1, float *ms)
{
    enqueue_calc<T>(c);  // warm-up
    CK(cudaEventRecord(e0, c->st));
    for (int r = 0; r < 3; r++) enqueue_calc<T>(c);
    CK(cudaEventRecord(e1, c->st));
    CK(cudaEventSynchronize(e1));
    CK(cudaGetLastError());
    CK(cudaEventElapsedTime(ms, e0, e1));
    return LFTS_OK;
}

int tune_tiles(lfts_ctx *c, lfts_tiles *best)
{
    const long long launches0 = c->launches;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best_ms = 0.f;
    bool found = false;
    int rc = LFTS_OK;
    for (const lfts_tiles &t : tile_candidates(c)) {
        if (apply_tiles(c, t) != LFTS_OK) continue;
        float ms = 0.f;
        rc = c->prec == LFTS_FP64 ? time_chain<double>(c, e0, e1, &ms) : time_chain<float>(c, e0, e1, &ms);
        if (rc) break;
        if (!found || ms < best_ms) {
            best_ms = ms;
            *best = t;
            found = true;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->launches = launches0;
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->st));
    CK(cudaStreamSynchronize(c->st1));
    return found ? LFTS_OK : LFTS_ERR_UNSUPPORTED;
}

int autotune(lfts_ctx *c)
{
    lfts_tiles t = default_tiles(c);
    const char *e = std::getenv("LFTS_AUTOTUNE");
    if (!(e && e[0] == '0')) {
        const auto key = std::make_tuple(c->prec, c->mx, c->my, c->mz);
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            t = it->second;
        } else {
            int rc = tune_tiles(c, &t);
            if (rc) return rc;
            g_tuned[key] = t;
        }
    }
    return apply_tiles(c, t);
}

// One chain on one stream with CUDA events around every contour-step kernel
// (mean duration of a yz-plane STEP and an x-pencil CONV launch, both chains
// per launch), then the production chain timed as a whole (first launch to Q).
template <typename T>
int profile_chain(lfts_ctx *c, double *ms_plane, double *ms_pencil, double *ms_chain)
{
    const int n = c->N - 1;
    std::vector<cudaEvent_t> ev(4 * n + 2);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    T *q = static_cast<T *>(c->q);
    const long long M = c->M;
    PlaneArgs<T> a = plane_args<T>(c);
    PencilArgs<T> pa = pencil_args<T>(c);
    // per step j: pencil between ev[4j] and ev[4j+1], plane between ev[4j+2] and ev[4j+3]
    CK(cudaEventRecord(ev[4 * n], c->st));
    if (c->xh_chain) {
        // the chain of enqueue_chain_launches: pencil INIT_W, (N-1) x (plane G, pencil H)
        PencilArgs<T> pi = pa;
        pi.qout = q;
        launch_pencil<T>(c, PENCIL_INIT_W, pi, 2);
        for (int i = 1; i < c->N; i++) {
            const int j = i - 1;
            CK(cudaEventRecord(ev[4 * j + 2], c->st));
            launch_plane<T>(c, PLANE_G, a, 2);
            CK(cudaEventRecord(ev[4 * j + 3], c->st));
            PencilArgs<T> ph = pa;
            ph.qout = q + (long long)i * 2 * M;
            ph.hsel0 = hsel_chain0(c, i);
            ph.hsel1 = hsel_chain1(c, i);
            CK(cudaEventRecord(ev[4 * j], c->st));
            launch_pencil<T>(c, i + 1 < c->N ? PENCIL_H : PENCIL_H_LAST, ph, 2);
            CK(cudaEventRecord(ev[4 * j + 1], c->st));
        }
        if constexpr (sizeof(T) == sizeof(float))
            plane_q_sums_kernel<<<c->mx, 256, 0, c->st>>>(
                reinterpret_cast<const float2 *>(q + (long long)(c->N - 1) * 2 * M), (long long)c->my * c->mz,
                c->qpart);
    } else {
        a.qout = q;
        launch_plane<T>(c, PLANE_INIT_W, a, 2);
        a.h = q;
        for (int i = 1; i < c->N; i++) {
            const int j = i - 1;
            CK(cudaEventRecord(ev[4 * j], c->st));
            launch_pencil<T>(c, PENCIL_CONV, pa, 2);
            CK(cudaEventRecord(ev[4 * j + 1], c->st));
            a.qout = q + (long long)i * 2 * M;
            a.hsel0 = hsel_chain0(c, i);
            a.hsel1 = hsel_chain1(c, i);
            CK(cudaEventRecord(ev[4 * j + 2], c->st));
            launch_plane<T>(c, i + 1 < c->N ? PLANE_STEP : PLANE_LAST, a, 2);
            CK(cudaEventRecord(ev[4 * j + 3], c->st));
        }
    }
    q_finalize_kernel<<<1, 256, 0, c->st>>>(c->qpart, c->mx, M, c->Qd);
    c->launches += c->xh_chain ? 2 : 1;
    CK(cudaEventRecord(ev[4 * n + 1], c->st));
    CK(cudaEventSynchronize(ev[4 * n + 1]));
    // means over the full-step launches (the last step's short launch left out)
    double pl = 0.0, pe = 0.0;
    int npl = 0, npe = 0;
    for (int j = 0; j < n; j++) {
        float t = 0.f;
        if (j + 1 < n || !c->xh_chain) {
            CK(cudaEventElapsedTime(&t, ev[4 * j], ev[4 * j + 1]));
            pe += t;
            npe++;
        }
        if (j + 1 < n || c->xh_chain) {
            CK(cudaEventElapsedTime(&t, ev[4 * j + 2], ev[4 * j + 3]));
            pl += t;
            npl++;
        }
    }
    // the production chain (both streams, PDL), timed as a whole
    CK(cudaEventRecord(ev[0], c->st));
    enqueue_chain<T>(c);
    CK(cudaEventRecord(ev[1], c->st));
    CK(cudaEventSynchronize(ev[1]));
    float tc = 0.f;
    CK(cudaEventElapsedTime(&tc, ev[0], ev[1]));
    for (auto &e : ev) cudaEventDestroy(e);
    *ms_pencil = npe ? pe / npe : 0.0;
    *ms_plane = npl ? pl / npl : 0.0;
    *ms_chain = tc;
    return LFTS_OK;
}

int calc_concs_sync(lfts_ctx *c, double *lnQ)
{
    HistPtrs none{};
    enqueue_concs_any(c, nullptr, 0, none);
    CK(cudaGetLastError());
    if (lnQ) {
        CK(cudaMemcpyAsync(c->red_host, c->Qd, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        *lnQ = c->red_host[1];
    }
    c->have_concs = true;
    return LFTS_OK;
}

// anderson::mix (src/anderson.cc:24-93) with the history kept as a ring of
// physical buffers addressed through the reference's logical slot numbers:
// the host-driven loop (one round trip per iteration for the dot products and
// the least squares).  anderson_mix below runs the same loop on the device.
int anderson_mix_host(lfts_ctx *c, int maxIter, double errTol, int *k_out)
{
    const int nhMax = kMaxHist;
    const long long M = c->M;
    double err = 1.0;
    int k;
    for (k = 1; k < maxIter && err > errTol; k++) {
        const int nh = (k < nhMax + 1) ? k - 1 : nhMax;
        HistPtrs Dhp{}, whp{};
        for (int m = 1; m <= nh; m++) {
            Dhp.p[m - 1] = c->Dh[c->phys[m]];
            whp.p[m - 1] = c->wh[c->phys[m]];
        }
        void *Dh0 = c->Dh[c->cur];
        enqueue_concs_any(c, Dh0, nh, Dhp);
        CK(cudaMemcpyAsync(c->red_host, c->red, (nh + 1) * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        const double S1 = c->red_host[0];
        err = std::pow(S1 / (double)M, 0.5);
        if (!std::isfinite(err)) {
            // stop before w+ is updated with it; k_out is what the reference's
            // loop would return (NaN > tol ends it after this iteration)
            g_last_error = "NaN or infinite Anderson residual (non-finite fields or concentrations)";
            c->mix_calls++;
            if (k_out) *k_out = k + 1;
            return LFTS_ERR_NONFINITE;
        }
        const double lambda = 1.0 - std::pow(0.9, double(k));
        for (int m = 0; m <= nh; m++) c->DD[0][m] = c->red_host[m];

        Coefs C{};
        int simple = 1;
        if (k >= 2) {
            simple = 0;
            std::vector<double> U((size_t)nh * nh), V(nh);
            for (int m = 1; m <= nh; m++) {
                V[m - 1] = c->DD[0][0] - c->DD[0][m];
                for (int n = 1; n <= m; n++) {
                    const double u = c->DD[0][0] - c->DD[0][m] - c->DD[0][n] + c->DD[n][m];
                    U[(m - 1) * nh + n - 1] = u;
                    U[(n - 1) * nh + m - 1] = u;
                }
            }
            if (!lu_solve(U, V, C.c, nh)) {
                g_last_error = "Anderson least-squares matrix is singular";
                return LFTS_ERR_SINGULAR;
            }
        }
        if (c->prec == LFTS_FP64)
            anderson_update_kernel<double><<<update_grid(c), 256, 0, c->st>>>(
                c->w + M, static_cast<double *>(c->wh[c->cur]), static_cast<const double *>(Dh0), M, lambda, nh,
                simple, Dhp, whp, C);
        else
            anderson_update_kernel<float><<<update_grid(c), 256, 0, c->st>>>(
                c->w + M, static_cast<float *>(c->wh[c->cur]), static_cast<const float *>(Dh0), M, lambda, nh,
                simple, Dhp, whp, C);
        c->launches++;
        CK(cudaGetLastError());

        // the current field and deviation become history slot n (src/anderson.cc:82-89)
        const int n = 1 + (k - 1) % nhMax;
        const int evicted = c->phys[n];
        c->phys[n] = c->cur;
        c->cur = evicted;
        c->DD[n][n] = c->DD[0][0];
        for (int m = 1; m < n; m++) c->DD[m][n] = c->DD[0][m];
        for (int m = n + 1; m <= nh; m++) c->DD[n][m] = c->DD[0][m];
        c->mix_iters++;
    }
    c->mix_calls++;
    if (k_out) *k_out = k;
    c->have_concs = true;
    if (err > errTol) {  // the loop ended at maxIter
        g_last_error = "Anderson mixing stopped at maxIter with the error above the tolerance";
        return LFTS_ERR_NOTCONV;
    }
    return LFTS_OK;
}

// ---- the Anderson loop on the device ---------------------------------------------
// One graph per context: begin -> WHILE { contour chain (the chain's own
// launches, programmatic edges included), concentrations + dot products,
// reduce + least squares (one warp, the host LU's operation order), w+
// update, control }.  Bit for bit what anderson_mix_host computes; the host
// sees the loop once per mix (state in, state out) instead of once per
// iteration.
template <typename T>
int capture_mix_graph(lfts_ctx *c, cudaGraph_t *g_out)
{
    MixState *S = static_cast<MixState *>(c->d_mix);
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    auto fail = [&](cudaError_t e, const char *what) {
        cudaGraphDestroy(g);
        cudaGetLastError();
        return cuda_fail(e, what);
    };
    cudaGraphConditionalHandle loop;
    cudaError_t e = cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return fail(e, "conditional handle");
    e = cudaStreamBeginCaptureToGraph(c->st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail(e, "mix graph capture");
    mix_begin_kernel<<<1, 32, 0, c->st>>>(S);
    cudaGraph_t cap = nullptr;
    e = cudaStreamEndCapture(c->st, &cap);
    if (e != cudaSuccess) return fail(e, "mix graph capture");
    size_t nn = 1;
    cudaGraphNode_t begin = nullptr;
    e = cudaGraphGetNodes(g, &begin, &nn);
    if (e != cudaSuccess) return fail(e, "mix graph nodes");
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cond = nullptr;
    e = cudaGraphAddNode(&cond, g, &begin, 1, &cp);
    if (e != cudaSuccess) return fail(e, "mix graph WHILE node");
    e = cudaStreamBeginCaptureToGraph(c->st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail(e, "mix graph body capture");
    const long long launches0 = c->launches;
    enqueue_chain_launches<T>(c);
    if (c->phi_in_chain)
        mix_conc_acc_kernel<<<stream_grid(c), kRedThreads, 0, c->st>>>(S, static_cast<const float *>(c->acc),
                                                                        static_cast<const float *>(c->q), c->N, c->Qd);
    else
        mix_conc_kernel<T><<<stream_grid(c), kRedThreads, 0, c->st>>>(S, static_cast<const T *>(c->q), c->N, c->NA,
                                                                        c->Qd);
    mix_solve_kernel<<<1, 256, 0, c->st>>>(S);
    mix_update_kernel<T><<<update_grid(c), 256, 0, c->st>>>(S);
    mix_control_kernel<<<1, 32, 0, c->st>>>(S, loop);
    c->mix_body_kernels = c->launches - launches0 + 4;
    c->launches = launches0;
    e = cudaStreamEndCapture(c->st, &cap);
    if (e != cudaSuccess) return fail(e, "mix graph body capture");
    *g_out = g;
    return LFTS_OK;
}

// builds the graph (with the chain's programmatic edges; without them if the
// body refuses them); on failure the context keeps the host loop
int ensure_mix_graph(lfts_ctx *c, int maxIter)
{
    if (c->mix_graph_state < 0) return LFTS_ERR_UNSUPPORTED;
    if (!c->d_mix) CK(cudaMalloc(&c->d_mix, sizeof(MixState)));
    if (maxIter + 2 > c->lambda_cap) {
        // lambda_k = 1 - 0.9^k (src/anderson.cc:44), host pow as in anderson_mix_host
        const int cap = std::max(maxIter + 2, 256);
        std::vector<double> lam(cap);
        for (int k = 0; k < cap; k++) lam[k] = 1.0 - std::pow(0.9, double(k));
        cudaFree(c->d_lambda);
        c->d_lambda = nullptr;
        CK(cudaMalloc(&c->d_lambda, sizeof(double) * cap));
        CK(cudaMemcpy(c->d_lambda, lam.data(), sizeof(double) * cap, cudaMemcpyHostToDevice));
        c->lambda_cap = cap;
    }
    if (c->mix_graph_state == 1) return LFTS_OK;
    const bool pdl = c->use_pdl;
    int rc = LFTS_ERR_CUDA;
    for (int attempt = 0; attempt < 2 && rc; attempt++) {
        c->use_pdl = pdl && attempt == 0;
        cudaGraph_t g = nullptr;
        rc = c->prec == LFTS_FP64 ? capture_mix_graph<double>(c, &g) : capture_mix_graph<float>(c, &g);
        if (!rc) {
            cudaError_t e = cudaGraphInstantiate(&c->mix_exec, g, 0);
            if (e == cudaSuccess) e = cudaGraphUpload(c->mix_exec, c->st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
            if (e != cudaSuccess) {
                if (c->mix_exec) cudaGraphExecDestroy(c->mix_exec);
                c->mix_exec = nullptr;
                cudaGraphDestroy(g);
                cudaGetLastError();
                rc = cuda_fail(e, "mix graph instantiate");
            } else {
                c->mix_graph = g;
                c->mix_pdl = c->use_pdl;
            }
        }
    }
    c->use_pdl = pdl;
    c->mix_graph_state = rc ? -1 : 1;
    if (const char *v = getenv("LFTS_VERBOSE"))
        if (v[0] == '1')
            fprintf(stderr, "lfts: Anderson-loop graph %s%s\n", rc ? "not built: " : "built, chain ",
                    rc ? g_last_error.c_str() : (c->mix_pdl ? "with programmatic edges" : "without programmatic edges"));
    return rc;
}

int anderson_mix(lfts_ctx *c, int maxIter, double errTol, int *k_out)
{
    if (!c->mix_on_device || maxIter < 2 || ensure_mix_graph(c, maxIter) != LFTS_OK)
        return anderson_mix_host(c, maxIter, errTol, k_out);
    MixState h{};
    h.M = c->M;
    h.red_blocks = c->red_blocks;
    h.maxIter = maxIter;
    h.tol = errTol;
    h.w = c->w;
    h.partials = c->partials;
    h.lambda = c->d_lambda;
    for (int i = 0; i < kRedWidth; i++) {
        h.Dh[i] = c->Dh[i];
        h.wh[i] = c->wh[i];
        h.phys[i] = c->phys[i];
    }
    h.cur = c->cur;
    MixState *S = static_cast<MixState *>(c->d_mix);
    CK(cudaMemcpyAsync(S, &h, sizeof(MixState), cudaMemcpyHostToDevice, c->st));
    CK(cudaGraphLaunch(c->mix_exec, c->st));
    CK(cudaMemcpyAsync(&h, S, sizeof(MixState), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int i = 0; i < kRedWidth; i++) c->phys[i] = h.phys[i];
    c->cur = h.cur;
    std::memcpy(c->DD, h.DD, sizeof(c->DD));
    const bool failed = h.nonfinite || h.singular;
    c->mix_iters += h.iters - 1 - (failed ? 1 : 0);
    c->mix_calls++;
    c->launches += (long long)(h.iters - 1) * c->mix_body_kernels + 1;
    if (h.nonfinite) {
        g_last_error = "NaN or infinite Anderson residual (non-finite fields or concentrations)";
        if (k_out) *k_out = h.iters;
        return LFTS_ERR_NONFINITE;
    }
    if (h.singular) {
        g_last_error = "Anderson least-squares matrix is singular";
        return LFTS_ERR_SINGULAR;
    }
    if (k_out) *k_out = h.iters;
    c->have_concs = true;
    if (h.notconv) {
        g_last_error = "Anderson mixing stopped at maxIter with the error above the tolerance";
        return LFTS_ERR_NOTCONV;
    }
    return LFTS_OK;
}

// ---- structure function -------------------------------------------------------
int sk_sample(lfts_ctx *c)
{
    PlaneArgs<double> a{};
    a.src64 = c->w;  // W-
    a.src_stride = 0;
    a.spec = static_cast<cpx<double> *>(c->skspec);
    const bool fp64 = c->prec == LFTS_FP64;
    a.twy = static_cast<const cpx<double> *>(fp64 ? c->tw[1] : c->sktw[1]);
    a.twz = static_cast<const cpx<double> *>(fp64 ? c->tw[2] : c->sktw[2]);
    a.Nd = (double)c->N;
    c->pl64.fn[PLANE_INIT_Q]<<<dim3(c->mx, 1), c->pl64.nt, c->pl64.smem, c->st>>>(a);
    PencilArgs<double> pa{};
    pa.spec = a.spec;
    pa.twx = static_cast<const cpx<double> *>(fp64 ? c->tw[0] : c->sktw[0]);
    pa.S = c->S;
    pa.ncol = c->my * c->KZ;
    pa.KZ = c->KZ;
    const int ncol = pa.ncol;
    c->pe64.fn[PENCIL_POWER]<<<dim3((ncol + c->pe64.cw - 1) / c->pe64.cw, 1), c->pe64.nt, c->pe64.smem, c->st>>>(pa);
    c->launches += 2;
    CK(cudaGetLastError());
    c->nsamples++;
    return LFTS_OK;
}

// |K| of every half-spectrum index (src/strFunc.cc:80-103) and bin tables
int sk_prepare_bins(lfts_ctx *c, double dK)
{
    const int m[3] = {c->mx, c->my, c->mz};
    const double *L = c->p.L;
    const long long Mk = c->Mk;
    std::vector<double> K(Mk);
    std::vector<int> wt(Mk, 2), P(Mk);
    for (int k0 = -(m[0] - 1) / 2; k0 <= m[0] / 2; k0++) {
        const int K0 = (k0 < 0) ? (k0 + m[0]) : k0;
        const double kx_sq = k0 * k0 / (L[0] * L[0]);
        for (int k1 = -(m[1] - 1) / 2; k1 <= m[1] / 2; k1++) {
            const int K1 = (k1 < 0) ? (k1 + m[1]) : k1;
            const double ky_sq = k1 * k1 / (L[1] * L[1]);
            for (int k2 = 0; k2 <= m[2] / 2; k2++) {
                const double kz_sq = k2 * k2 / (L[2] * L[2]);
                const long long k = k2 + (long long)(m[2] / 2 + 1) * (K1 + (long long)m[1] * K0);
                K[k] = kTwoPi * std::pow(kx_sq + ky_sq + kz_sq, 0.5);
                if (k2 == 0 || k2 == m[2] / 2) wt[k] = 1;
            }
        }
    }
    std::iota(P.begin(), P.end(), 0);
    std::stable_sort(P.begin(), P.end(), [&](int i, int j) { return K[i] < K[j]; });
    std::vector<int> bins;
    c->sk_K.clear();
    bins.push_back(0);
    for (long long k = 0; k < Mk; k++) {
        if (k == Mk - 1 || std::fabs(K[P[k + 1]] - K[P[k]]) > dK) {
            bins.push_back((int)k + 1);
            c->sk_K.push_back(K[P[k]]);
        }
    }
    cudaFree(c->sk_order);
    cudaFree(c->sk_wt);
    cudaFree(c->sk_bins);
    cudaFree(c->sk_out);
    c->sk_nbins = (int)bins.size() - 1;
    CK(cudaMalloc(&c->sk_order, sizeof(int) * Mk));
    CK(cudaMalloc(&c->sk_wt, sizeof(int) * Mk));
    CK(cudaMalloc(&c->sk_bins, sizeof(int) * bins.size()));
    CK(cudaMalloc(&c->sk_out, sizeof(double) * c->sk_nbins));
    CK(cudaMemcpy(c->sk_order, P.data(), sizeof(int) * Mk, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->sk_wt, wt.data(), sizeof(int) * Mk, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->sk_bins, bins.data(), sizeof(int) * bins.size(), cudaMemcpyHostToDevice));
    c->sk_dK = dK;
    return LFTS_OK;
}

int ctx_alloc(lfts_ctx *c)
{
    const long long M = c->M;
    CK(cudaMalloc(&c->w, sizeof(double) * 4 * M));
    CK(cudaMemset(c->w, 0, sizeof(double) * 4 * M));
    CK(cudaMalloc(&c->q, c->tsize * 2 * M * (size_t)c->N));
    CK(cudaMalloc(&c->spec, c->tsize * 2 * 2 * (size_t)c->mx * c->my * c->KZ));
    CK(cudaMalloc(&c->qpart, sizeof(double) * c->mx));
    CK(cudaMalloc(&c->Qd, sizeof(double) * 2));
    CK(cudaMalloc(&c->partials, sizeof(double) * kRedWidth * c->red_blocks));
    CK(cudaMalloc(&c->red, sizeof(double) * kRedWidth));
    CK(cudaMallocHost(&c->red_host, sizeof(double) * kRedWidth));
    for (int i = 0; i < 2; i++) {
        CK(cudaMalloc(&c->eta[i], sizeof(double) * M));
        CK(cudaMemset(c->eta[i], 0, sizeof(double) * M));
    }
    for (int i = 0; i < kRedWidth; i++) {
        CK(cudaMalloc(&c->Dh[i], c->tsize * M));
        CK(cudaMalloc(&c->wh[i], c->tsize * M));
        CK(cudaMemset(c->Dh[i], 0, c->tsize * M));
        CK(cudaMemset(c->wh[i], 0, c->tsize * M));
    }
    // logical slots 1..10 -> buffers 1..10, buffer 0 is the first current one
    for (int i = 0; i < kRedWidth; i++) c->phys[i] = i;
    c->cur = 0;
    CK(cudaMalloc(&c->S, sizeof(double) * c->Mk));
    CK(cudaMemset(c->S, 0, sizeof(double) * c->Mk));
    if (c->prec == LFTS_FP64) {
        c->skspec = c->spec;
    } else {
        CK(cudaMalloc(&c->skspec, sizeof(cpx<double>) * (size_t)c->Mk));
        c->sk_own_spec = true;
    }
    return LFTS_OK;
}

void ctx_free(lfts_ctx *c)
{
    if (c->st) cudaStreamSynchronize(c->st);
    cudaFree(c->w);
    cudaFree(c->q);
    cudaFree(c->spec);
    for (int d = 0; d < 3; d++) {
        cudaFree(c->tw[d]);
        cudaFree(c->gtab[d]);
        cudaFree(c->sktw[d]);
    }
    cudaFree(c->qpart);
    cudaFree(c->Qd);
    cudaFree(c->partials);
    cudaFree(c->red);
    if (c->red_host) cudaFreeHost(c->red_host);
    for (int i = 0; i < 2; i++) cudaFree(c->eta[i]);
    for (int i = 0; i < kRedWidth; i++) {
        cudaFree(c->Dh[i]);
        cudaFree(c->wh[i]);
    }
    cudaFree(c->S);
    if (c->sk_own_spec) cudaFree(c->skspec);
    cudaFree(c->sk_order);
    cudaFree(c->sk_wt);
    cudaFree(c->sk_bins);
    cudaFree(c->sk_out);
    cudaFree(c->sf_buf);
    cudaFree(c->adj_partial);
    cudaFree(c->adj_buf);
    drop_chain_graph(c);
    cudaFree(c->acc);
    cudaFree(c->d_mix);
    cudaFree(c->d_lambda);
    if (c->st1) cudaStreamSynchronize(c->st1);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    for (int k = 0; k < 2; k++)
        if (c->ev_h[k]) cudaEventDestroy(c->ev_h[k]);
    if (c->st1) cudaStreamDestroy(c->st1);
    if (c->st) cudaStreamDestroy(c->st);
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

namespace {
template <typename T>
int step_fwd_impl(lfts_ctx *c, const double *q_in, double *q_out, const double *h, int i)
{
    const long long M = c->M;
    double *dq = static_cast<double *>(c->sf_buf);
    double *dout = dq + 2 * M, *dh = dq + 4 * M;
    T *tq = reinterpret_cast<T *>(dh + 2 * M);  // T copies when T != double
    T *th = tq + 2 * M;
    T *tout = th + 2 * M;
    CK(cudaMemcpyAsync(dq, q_in, sizeof(double) * 2 * M, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(dh, h, sizeof(double) * 2 * M, cudaMemcpyHostToDevice, c->st));
    const T *src = reinterpret_cast<const T *>(dq), *hh = reinterpret_cast<const T *>(dh);
    T *dst = reinterpret_cast<T *>(dout);
    if (sizeof(T) != sizeof(double)) {
        convert_kernel<double, T><<<stream_grid(c), 256, 0, c->st>>>(dq, tq, 2 * M);
        to_pairs_kernel<double, T><<<stream_grid(c), 256, 0, c->st>>>(dh, th, M);  // packed-path layout
        c->launches += 2;
        src = tq;
        hh = th;
        dst = tout;
    }
    PlaneArgs<T> a = plane_args<T>(c);
    a.src = src;
    a.src_stride = M;
    launch_plane<T>(c, PLANE_INIT_Q, a, 2);
    launch_pencil<T>(c, PENCIL_CONV, pencil_args<T>(c), 2);
    a.qout = dst;
    a.h = hh;
    a.hsel0 = hsel_chain0(c, i);
    a.hsel1 = hsel_chain1(c, i);
    launch_plane<T>(c, PLANE_LAST, a, 2);
    if (sizeof(T) != sizeof(double)) {
        from_pairs_kernel<T, double><<<stream_grid(c), 256, 0, c->st>>>(tout, dout, M);
        c->launches++;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(q_out, dout, sizeof(double) * 2 * M, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return LFTS_OK;
}

}  // namespace

namespace {

// One adjoint term: forward transforms of q_i (chain 0) and q^_{i+1}
// (chain 1), then the k^2-weighted products summed into c->adj_partial.
int adjoint_term(lfts_ctx *c, const double *q_i, const double *qh_ip1)
{
    PlaneArgs<double> a = plane_args<double>(c);
    a.src = q_i;
    a.src_stride = (long long)(qh_ip1 - q_i);
    launch_plane<double>(c, PLANE_INIT_Q, a, 2);
    AdjArgs aa{};
    aa.spec = static_cast<const cpx<double> *>(c->spec);
    aa.twx = static_cast<const cpx<double> *>(c->tw[0]);
    aa.gx = static_cast<const double *>(c->gtab[0]);
    aa.gy = static_cast<const double *>(c->gtab[1]);
    aa.gz = static_cast<const double *>(c->gtab[2]);
    aa.ncol = c->my * c->KZ;
    aa.KZ = c->KZ;
    aa.mx = c->mx;
    aa.my = c->my;
    aa.mz = c->mz;
    aa.partial = c->adj_partial;
    c->adj.fn<<<(aa.ncol + c->adj.cw - 1) / c->adj.cw, c->adj.nt, c->adj.smem, c->st>>>(aa);
    c->launches++;
    return LFTS_OK;
}

// Propagators of both chains with q stored only at monomers 1, 1+K, 1+2K, ...
// (q^ in full); returns after Q is reduced.  Chains run as separate launches
// so each output can be placed independently.
int chain_checkpointed(lfts_ctx *c, int K)
{
    double *q = static_cast<double *>(c->q);
    const long long M = c->M;
    double *discard = c->adj_buf + (long long)K * M;
    PlaneArgs<double> a = plane_args<double>(c);
    PencilArgs<double> pa = pencil_args<double>(c);
    a.qout = q;
    launch_plane<double>(c, PLANE_INIT_W, a, 2);  // slot 1 = [hA | hB]
    a.h = q;
    PlaneArgs<double> a0 = a, a1 = a;
    PencilArgs<double> p0 = pa, p1 = pa;
    a0.cbase = 0;
    a1.cbase = 1;
    p0.cbase = 0;
    p1.cbase = 1;
    for (int i = 1; i < c->N; i++) {
        launch_pencil<double>(c, PENCIL_CONV, p0, 1);
        launch_pencil<double>(c, PENCIL_CONV, p1, 1);
        const int mode = i + 1 < c->N ? PLANE_STEP : PLANE_LAST;
        a0.hsel0 = a1.hsel0 = hsel_chain0(c, i);
        a0.hsel1 = a1.hsel1 = hsel_chain1(c, i);
        // q_{i+1}: a checkpoint slot or the discard row (chain 0 writes qout + 0)
        a0.qout = (i % K == 0) ? q + (long long)i * 2 * M : discard;
        a1.qout = q + (long long)i * 2 * M;  // q^_{N-i}: second half of slot i+1
        launch_plane<double>(c, mode, a0, 1);
        launch_plane<double>(c, mode, a1, 1);
    }
    q_finalize_kernel<<<1, 256, 0, c->st>>>(c->qpart, c->mx, M, c->Qd);
    c->launches++;
    return LFTS_OK;
}

// q_{c0+1} .. q_{c0+n} recomputed from the checkpoint q_{c0} into adj_buf rows 1..n
void recompute_segment(lfts_ctx *c, const double *q_c0, int c0, int n)
{
    const long long M = c->M;
    PlaneArgs<double> a = plane_args<double>(c);
    PencilArgs<double> pa = pencil_args<double>(c);
    a.cbase = 0;
    pa.cbase = 0;
    a.src = q_c0;
    a.src_stride = 0;
    launch_plane<double>(c, PLANE_INIT_Q, a, 1);
    a.h = static_cast<double *>(c->q);
    for (int j = 1; j <= n; j++) {
        const int i = c0 + j - 1;  // step i makes q_{i+1}
        launch_pencil<double>(c, PENCIL_CONV, pa, 1);
        a.hsel0 = hsel_chain0(c, i);
        a.qout = c->adj_buf + (long long)j * M;
        launch_plane<double>(c, PLANE_STEP, a, 1);
    }
}

}  // namespace

}  // namespace

// =============================================================================
extern "C" {

const char *lfts_version(void) { return "lfts_b200 0.1 (sm_100a)"; }

const char *lfts_status_string(int s)
{
    switch (s) {
        case LFTS_OK: return "ok";
        case LFTS_ERR_ARG: return "invalid argument";
        case LFTS_ERR_UNSUPPORTED: return "mesh size not supported by the FFT kernels";
        case LFTS_ERR_CUDA: return "CUDA error";
        case LFTS_ERR_NOMEM: return "device allocation failed";
        case LFTS_ERR_SINGULAR: return "Anderson least-squares matrix singular";
        case LFTS_ERR_STATE: return "call out of order";
        case LFTS_ERR_NOTCONV: return "Anderson iteration cap reached above the tolerance";
        case LFTS_ERR_NONFINITE: return "non-finite Anderson residual";
        default: return "unknown status";
    }
}

const char *lfts_last_error_string(void) { return g_last_error.c_str(); }

int lfts_mesh_supported(int n) { return fft_length_supported(n) ? 1 : 0; }

int lfts_create(const lfts_params *p, int precision, int device, lfts_ctx **out)
{
    if (!p || !out) return LFTS_ERR_ARG;
    *out = nullptr;
    if (p->N < 2 || p->NA < 0 || p->NA > p->N || p->C <= 0.0 || p->XbN == 0.0) return LFTS_ERR_ARG;
    if (precision != LFTS_FP64 && precision != LFTS_FP32_MIXED) return LFTS_ERR_ARG;
    for (int d = 0; d < 3; d++)
        if (p->m[d] < 1 || !(p->L[d] > 0.0)) return LFTS_ERR_ARG;
    // even my and mz (row pairs, packed Nyquist column) also make M a multiple
    // of 4, which the vectorised concentration pass relies on
    if (!fft_length_supported(p->m[0]) || !plane_pair_supported(p->m[1], p->m[2]) || (p->m[1] % 2) ||
        (p->m[2] % 2)) {
        g_last_error = "mesh not supported: each dimension must be one of the compiled FFT lengths";
        return LFTS_ERR_UNSUPPORTED;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        g_last_error = "no CUDA device";
        return LFTS_ERR_CUDA;
    }
    DeviceGuard g(device);
    lfts_ctx *c = new lfts_ctx;
    c->p = *p;
    c->prec = precision;
    c->dev = device;
    c->N = p->N;
    c->NA = p->NA;
    c->NB = p->N - p->NA;
    c->mx = p->m[0];
    c->my = p->m[1];
    c->mz = p->m[2];
    c->KZ = c->mz / 2 + 1;
    c->M = (long long)c->mx * c->my * c->mz;
    c->Mk = (long long)c->mx * c->my * c->KZ;
    c->tsize = precision == LFTS_FP64 ? sizeof(double) : sizeof(float);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->sms = prop.multiProcessorCount;
    c->red_blocks = c->sms * 4;
    if (const char *e = getenv("LFTS_NO_PDL")) c->use_pdl = !(e[0] == '1');
    // SMs the one-CTA-per-plane PLANE_G leaves idle take its L2 prefetch of the
    // partner slot (LFTS_PREFETCH_CTAS=0: the plane CTAs issue it themselves).
    // Only for 128 x 128 planes, whose CTA fills an SM's shared memory: at 96 x 96
    // two plane CTAs share an SM and the extra CTAs measured slower
    c->pf_ctas = (c->my == 128 && c->mz == 128 && c->sms > c->mx) ? std::min(c->sms - c->mx, 64) : 0;
    if (const char *e = getenv("LFTS_PREFETCH_CTAS")) c->pf_ctas = std::max(0, std::min(std::atoi(e), c->pf_ctas));
    if (const char *e = getenv("LFTS_ONE_STREAM")) c->two_streams = !(e[0] == '1');
    if (const char *e = getenv("LFTS_NO_GRAPH")) c->use_graph = !(e[0] == '1');
    if (const char *e = getenv("LFTS_DEVICE_MIX")) c->mix_on_device = e[0] == '1';
    if (!c->use_graph) c->mix_on_device = false;
    int rc = LFTS_OK;
    auto fail = [&](int code) {
        ctx_free(c);
        delete c;
        return code;
    };
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->st1, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_h[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_h[1], cudaEventDisableTiming) != cudaSuccess)
        return fail(LFTS_ERR_CUDA);
    if (!plane_kernels(c->my, c->mz, &c->pl64) || !pencil_kernels(c->mx, &c->pe64)) return fail(LFTS_ERR_UNSUPPORTED);
    if ((rc = set_smem_attrs(c->pl64, c->pe64))) return fail(rc);
    if (precision == LFTS_FP32_MIXED) {
        c->packed = true;
        if (plane3_kernels(c->my, c->mz, &c->pl32))
            c->plane_stages = 3;
        else if (!plane_c_kernels(c->my, c->mz, &c->pl32))
            return fail(LFTS_ERR_UNSUPPORTED);
        if (!pencil_kernels(c->mx, kDefaultCwFp32, &c->pe32)) return fail(LFTS_ERR_UNSUPPORTED);
        // h and the stored propagators in the x-pencil where both kernels have
        // those modes (128^3); LFTS_XH_CHAIN=0 keeps them in the yz-plane kernel
        const char *xh = getenv("LFTS_XH_CHAIN");
        c->xh_chain = c->pl32.fn[PLANE_G] && c->pe32.fn[PENCIL_H] && !(xh && xh[0] == '0');
        if ((rc = set_smem_attrs(c->pl32, c->pe32))) return fail(rc);
    }
    if ((rc = ctx_alloc(c))) return fail(rc == LFTS_ERR_CUDA ? LFTS_ERR_NOMEM : rc);
    if (precision == LFTS_FP64)
        rc = upload_tables<double>(c, c->tw, c->gtab);
    else {
        rc = upload_tables<float>(c, c->tw, c->gtab);
        if (!rc) rc = upload_tables<double>(c, c->sktw, nullptr);
    }
    if (rc) return fail(rc);
    if ((rc = autotune(c))) return fail(rc);
    *out = c;
    return LFTS_OK;
}

int lfts_destroy(lfts_ctx *c)
{
    if (!c) return LFTS_OK;
    DeviceGuard g(c->dev);
    ctx_free(c);
    delete c;
    return LFTS_OK;
}

int lfts_device_bytes(const lfts_ctx *c, size_t *bytes)
{
    if (!c || !bytes) return LFTS_ERR_ARG;
    const size_t M = c->M;
    size_t b = 4 * M * 8 + c->tsize * 2 * M * c->N + c->tsize * 4 * (size_t)c->mx * c->my * c->KZ;
    b += 2 * M * 8 + 2 * kRedWidth * M * c->tsize + c->Mk * 8;
    if (c->sk_own_spec) b += c->Mk * 16;
    if (c->acc) b += 8 * M;
    *bytes = b;
    return LFTS_OK;
}

int lfts_set_fields(lfts_ctx *c, const double *w_host)
{
    if (!c || !w_host) return LFTS_ERR_ARG;
    DeviceGuard g(c->dev);
    CK(cudaMemcpyAsync(c->w, w_host, sizeof(double) * 2 * c->M, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->fields_set = true;
    return LFTS_OK;
}

int lfts_get_fields(lfts_ctx *c, double *w_host)
{
    if (!c || !w_host) return LFTS_ERR_ARG;
    DeviceGuard g(c->dev);
    CK(cudaMemcpyAsync(w_host, c->w, sizeof(double) * 4 * c->M, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return LFTS_OK;
}

int lfts_fields_device(lfts_ctx *c, double **w_dev)
{
    if (!c || !w_dev) return LFTS_ERR_ARG;
    *w_dev = c->w;
    c->fields_set = true;  // the caller may fill the array directly
    return LFTS_OK;
}

int lfts_calc_concs(lfts_ctx *c, double *lnQ)
{
    if (!c) return LFTS_ERR_ARG;
    if (!c->fields_set) return LFTS_ERR_STATE;
    DeviceGuard g(c->dev);
    return calc_concs_sync(c, lnQ);
}

int lfts_anderson_mix(lfts_ctx *c, int maxIter, double errTol, int *k_out)
{
    if (!c) return LFTS_ERR_ARG;
    if (!c->fields_set) return LFTS_ERR_STATE;
    DeviceGuard g(c->dev);
    return anderson_mix(c, maxIter, errTol, k_out);
}

int lfts_langevin_init(lfts_ctx *c, const double *noise_prev_host)
{
    if (!c || !noise_prev_host) return LFTS_ERR_ARG;
    DeviceGuard g(c->dev);
    c->eta_prev = 0;
    CK(cudaMemcpyAsync(c->eta[0], noise_prev_host, sizeof(double) * c->M, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->eta_set = true;
    return LFTS_OK;
}

static int langevin_device(lfts_ctx *c, const double *eta_new_dev)
{
    const int nb = 1 - c->eta_prev;
    if (eta_new_dev != c->eta[nb])
        CK(cudaMemcpyAsync(c->eta[nb], eta_new_dev, sizeof(double) * c->M, cudaMemcpyDeviceToDevice, c->st));
    langevin_kernel<<<update_grid(c), 256, 0, c->st>>>(c->w, c->M, c->eta[c->eta_prev], c->eta[nb], c->p.XbN,
                                                       c->p.dt);
    c->launches++;
    CK(cudaGetLastError());
    c->eta_prev = nb;  // the new noise is the next step's previous noise (src/langevin.cc:34-36)
    return LFTS_OK;
}

int lfts_langevin_step(lfts_ctx *c, const double *noise_new_host)
{
    if (!c || !noise_new_host) return LFTS_ERR_ARG;
    if (!c->fields_set || !c->eta_set || !c->have_concs) return LFTS_ERR_STATE;
    DeviceGuard g(c->dev);
    const int nb = 1 - c->eta_prev;
    CK(cudaMemcpyAsync(c->eta[nb], noise_new_host, sizeof(double) * c->M, cudaMemcpyHostToDevice, c->st));
    int rc = langevin_device(c, c->eta[nb]);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->st));
    return LFTS_OK;
}

int lfts_langevin_step_device(lfts_ctx *c, const double *noise_new_dev)
{
    if (!c || !noise_new_dev) return LFTS_ERR_ARG;
    if (!c->fields_set || !c->eta_set || !c->have_concs) return LFTS_ERR_STATE;
    DeviceGuard g(c->dev);
    return langevin_device(c, noise_new_dev);
}

int lfts_langevin_full_step(lfts_ctx *c, const double *noise_new_dev, int maxIter, double errTol, int *k_out,
                            double *lnQ)
{
    if (!c || !noise_new_dev) return LFTS_ERR_ARG;
    if (!c->fields_set || !c->eta_set || !c->have_concs) return LFTS_ERR_STATE;
    DeviceGuard g(c->dev);
    int rc = langevin_device(c, noise_new_dev);
    if (rc) return rc;
    rc = anderson_mix(c, maxIter, errTol, k_out);
    if (rc && rc != LFTS_ERR_NOTCONV) return rc;
    const int rc2 = calc_concs_sync(c, lnQ);  // the step completes past the cap, as in the reference
    return rc2 ? rc2 : rc;
}

int lfts_sk_sample(lfts_ctx *c)
{
    if (!c) return LFTS_ERR_ARG;
    if (!c->fields_set) return LFTS_ERR_STATE;
    DeviceGuard g(c->dev);
    int rc = sk_sample(c);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->st));
    return LFTS_OK;
}

int lfts_sk_get(lfts_ctx *c, double *S_host, int *nsamples)
{
    if (!c) return LFTS_ERR_ARG;
    DeviceGuard g(c->dev);
    if (S_host) {
        CK(cudaMemcpyAsync(S_host, c->S, sizeof(double) * c->Mk, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
    }
    if (nsamples) *nsamples = c->nsamples;
    return LFTS_OK;
}

int lfts_sk_reset(lfts_ctx *c)
{
    if (!c) return LFTS_ERR_ARG;
    DeviceGuard g(c->dev);
    CK(cudaMemsetAsync(c->S, 0, sizeof(double) * c->Mk, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->nsamples = 0;
    return LFTS_OK;
}

int lfts_sk_bin(lfts_ctx *c, double dK, double *K_out, double *S_out, int *nbins)
{
    // with no samples the averages come out NaN, as the reference's division
    // by nsamples_ = 0 does
    if (!c || !K_out || !S_out || !nbins || !(dK >= 0.0)) return LFTS_ERR_ARG;
    DeviceGuard g(c->dev);
    if (dK != c->sk_dK) {
        int rc = sk_prepare_bins(c, dK);
        if (rc) return rc;
    }
    // coeff_ = CV/(chi_b^2 M^2) (src/strFunc.cc:21), with CV = C*V
    const double V = c->p.L[0] * c->p.L[1] * c->p.L[2];
    const double CV = c->p.C * V;
    const double M = (double)c->M;
    const double coeff = CV / (c->p.XbN * c->p.XbN * M * M);
    sk_bin_kernel<<<(c->sk_nbins + 127) / 128, 128, 0, c->st>>>(c->S, c->sk_order, c->sk_wt, c->sk_bins,
                                                               c->sk_nbins, coeff / (double)c->nsamples,
                                                               0.5 / c->p.XbN, c->sk_out);
    c->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(S_out, c->sk_out, sizeof(double) * c->sk_nbins, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    std::memcpy(K_out, c->sk_K.data(), sizeof(double) * c->sk_nbins);
    *nbins = c->sk_nbins;
    return LFTS_OK;
}

int lfts_get_H(lfts_ctx *c, double *H)
{
    if (!c || !H) return LFTS_ERR_ARG;
    if (!c->fields_set) return LFTS_ERR_STATE;
    DeviceGuard g(c->dev);
    double lnQ = 0.0;
    int rc = calc_concs_sync(c, &lnQ);
    if (rc) return rc;
    h_sums_kernel<<<stream_grid(c), kRedThreads, 0, c->st>>>(c->w, c->M, c->partials);
    reduce_partials_kernel<<<2, 256, 0, c->st>>>(c->partials, c->red_blocks, 2, c->red);
    c->launches += 2;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->red_host, c->red, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    const double wp_sum = c->red_host[0], wm2_sum = c->red_host[1];
    *H = -lnQ + (wm2_sum / c->p.XbN - wp_sum) / (double)c->M;
    return LFTS_OK;
}

int lfts_step_fwd(lfts_ctx *c, const double *q_in, double *q_out, const double *h, int i)
{
    if (!c || !q_in || !q_out || !h || i < 1 || i >= c->N) return LFTS_ERR_ARG;
    DeviceGuard g(c->dev);
    if (!c->sf_buf) CK(cudaMalloc(&c->sf_buf, sizeof(double) * 6 * c->M + c->tsize * 6 * c->M));
    if (c->prec == LFTS_FP64) return step_fwd_impl<double>(c, q_in, q_out, h, i);
    return step_fwd_impl<float>(c, q_in, q_out, h, i);
}

int lfts_g_lookup(lfts_ctx *c, double *g_host)
{
    if (!c || !g_host) return LFTS_ERR_ARG;
    // the factorised weights the kernels multiply by, expanded to the Mk layout
    const int m[3] = {c->mx, c->my, c->mz};
    std::vector<double> g[3];
    const int n[3] = {c->mx, c->my, c->KZ};
    for (int d = 0; d < 3; d++) {
        g[d].resize(n[d]);
        for (int K = 0; K < n[d]; K++) {
            const int k = (d == 2) ? K : signed_k(K, m[d]);
            const double ksq = (double)k * k / (c->p.L[d] * c->p.L[d]);
            double v = std::exp(-kTwoPi * kTwoPi * ksq / (6.0 * c->N));
            if (d == 2) v /= (double)c->M;
            g[d][K] = (c->prec == LFTS_FP64) ? v : (double)(float)v;
        }
    }
    for (int a = 0; a < c->mx; a++)
        for (int b = 0; b < c->my; b++)
            for (int k = 0; k < c->KZ; k++)
                g_host[((long long)a * c->my + b) * c->KZ + k] = g[0][a] * g[1][b] * g[2][k];
    return LFTS_OK;
}

int lfts_backward(lfts_ctx *c, int ckpt_every, double *dH_dL, double *dH_dXbN, double *H)
{
    if (!c || !dH_dL || ckpt_every < 0) return LFTS_ERR_ARG;
    if (!c->fields_set) return LFTS_ERR_STATE;
    if (c->prec != LFTS_FP64) {
        g_last_error = "the adjoint runs on FP64 contexts";
        return LFTS_ERR_UNSUPPORTED;
    }
    DeviceGuard g(c->dev);
    if (!c->adj.fn && !adjoint_kernel(c->mx, &c->adj)) return LFTS_ERR_UNSUPPORTED;
    CK(cudaFuncSetAttribute(c->adj.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->adj.smem));
    const long long M = c->M;
    const int nblk = (c->my * c->KZ + c->adj.cw - 1) / c->adj.cw;
    if (!c->adj_partial) CK(cudaMalloc(&c->adj_partial, sizeof(double) * 3 * nblk));
    CK(cudaMemsetAsync(c->adj_partial, 0, sizeof(double) * 3 * nblk, c->st));
    double *q = static_cast<double *>(c->q);
    const int N = c->N;
    // q_i is the first half of slot i, q^_{i+1} the second half of slot N-i
    auto qh = [&](int i1) { return q + (long long)(N - i1) * 2 * M + M; };  // q^_{i1}
    if (ckpt_every == 0) {
        int rc = calc_concs_sync(c, nullptr);
        if (rc) return rc;
        for (int i = 1; i < N; i++) adjoint_term(c, q + (long long)(i - 1) * 2 * M, qh(i + 1));
    } else {
        const int K = ckpt_every;
        if (c->adj_buf_slots < K + 1) {
            cudaFree(c->adj_buf);
            c->adj_buf = nullptr;
            CK(cudaMalloc(&c->adj_buf, sizeof(double) * (size_t)(K + 1) * M));
            c->adj_buf_slots = K + 1;
        }
        chain_checkpointed(c, K);
        for (int c0 = 1; c0 < N; c0 += K) {
            const int last = std::min(c0 + K - 1, N - 1);  // terms i = c0 .. last
            const double *qc = q + (long long)(c0 - 1) * 2 * M;
            if (last > c0) recompute_segment(c, qc, c0, last - c0);
            for (int i = c0; i <= last; i++)
                adjoint_term(c, i == c0 ? qc : c->adj_buf + (long long)(i - c0) * M, qh(i + 1));
        }
        c->have_concs = false;  // phi was not recomputed
    }
    CK(cudaGetLastError());
    std::vector<double> part(3 * (size_t)nblk);
    CK(cudaMemcpyAsync(part.data(), c->adj_partial, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(c->red_host, c->Qd, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    const double Q = c->red_host[0], lnQ = c->red_host[1];
    double S[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < nblk; b++)
        for (int d = 0; d < 3; d++) S[d] += part[3 * (size_t)b + d];
    // dH/dL = -(1/Q) dQ/dL, dQ/dL_a = (1/M) 4 pi^2 S_a / (3 N L_a^3)
    for (int d = 0; d < 3; d++) {
        const double L = c->p.L[d];
        dH_dL[d] = -(kTwoPi * kTwoPi * S[d] / (3.0 * N * L * L * L)) / ((double)M * Q);
    }
    h_sums_kernel<<<stream_grid(c), kRedThreads, 0, c->st>>>(c->w, M, c->partials);
    reduce_partials_kernel<<<2, 256, 0, c->st>>>(c->partials, c->red_blocks, 2, c->red);
    c->launches += 2;
    CK(cudaMemcpyAsync(c->red_host, c->red, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    const double wp_sum = c->red_host[0], wm2_sum = c->red_host[1];
    const double X = c->p.XbN;
    if (dH_dXbN) *dH_dXbN = -wm2_sum / (X * X * (double)M);
    if (H) *H = -lnQ + (wm2_sum / X - wp_sum) / (double)M;
    return LFTS_OK;
}

void *lfts_stream(lfts_ctx *c) { return c ? (void *)c->st : nullptr; }

int lfts_profile_chain(lfts_ctx *c, double *ms_plane, double *ms_pencil, double *ms_chain)
{
    if (!c || !ms_plane || !ms_pencil || !ms_chain) return LFTS_ERR_ARG;
    if (!c->fields_set) return LFTS_ERR_STATE;
    DeviceGuard g(c->dev);
    CK(cudaStreamSynchronize(c->st));
    if (c->prec == LFTS_FP64) return profile_chain<double>(c, ms_plane, ms_pencil, ms_chain);
    return profile_chain<float>(c, ms_plane, ms_pencil, ms_chain);
}

int lfts_profile_iteration(lfts_ctx *c, int reps, double *ms_chain, double *ms_concs, double *ms_update)
{
    if (!c || reps < 1 || !ms_chain || !ms_concs || !ms_update) return LFTS_ERR_ARG;
    if (!c->fields_set) return LFTS_ERR_STATE;
    DeviceGuard g(c->dev);
    CK(cudaStreamSynchronize(c->st));
    const long long M = c->M;
    // a full history: every ring buffer in use, as from the 11th iteration on
    HistPtrs Dhp{}, whp{};
    for (int m = 1; m <= kMaxHist; m++) {
        Dhp.p[m - 1] = c->Dh[c->phys[m]];
        whp.p[m - 1] = c->wh[c->phys[m]];
    }
    Coefs zero{};  // lambda = 0 and zero coefficients leave w+ bitwise unchanged
    cudaEvent_t ev[4];
    for (auto &e : ev) CK(cudaEventCreate(&e));
    enqueue_chain_any(c);  // warm
    CK(cudaEventRecord(ev[0], c->st));
    for (int r = 0; r < reps; r++) enqueue_chain_any(c);
    CK(cudaEventRecord(ev[1], c->st));
    for (int r = 0; r < reps; r++) {
        if (c->prec == LFTS_FP64)
            concentrations_kernel<double><<<stream_grid(c), kRedThreads, 0, c->st>>>(
                static_cast<const double *>(c->q), M, c->N, c->NA, c->w, c->w + 2 * M, c->w + 3 * M, c->Qd,
                static_cast<double *>(c->Dh[c->cur]), kMaxHist, Dhp, c->partials);
        else if (c->phi_in_chain)
            concentrations_acc_kernel<<<stream_grid(c), kRedThreads, 0, c->st>>>(
                static_cast<const float *>(c->acc), static_cast<const float *>(c->q), M, c->N, c->w + 2 * M,
                c->w + 3 * M, c->Qd, static_cast<float *>(c->Dh[c->cur]), kMaxHist, Dhp, c->partials);
        else
            concentrations_kernel<float><<<stream_grid(c), kRedThreads, 0, c->st>>>(
                static_cast<const float *>(c->q), M, c->N, c->NA, c->w, c->w + 2 * M, c->w + 3 * M, c->Qd,
                static_cast<float *>(c->Dh[c->cur]), kMaxHist, Dhp, c->partials);
        reduce_partials_kernel<<<kRedWidth, 256, 0, c->st>>>(c->partials, c->red_blocks, kRedWidth, c->red);
    }
    CK(cudaEventRecord(ev[2], c->st));
    for (int r = 0; r < reps; r++) {
        if (c->prec == LFTS_FP64)
            anderson_update_kernel<double><<<update_grid(c), 256, 0, c->st>>>(
                c->w + M, static_cast<double *>(c->wh[c->cur]), static_cast<const double *>(c->Dh[c->cur]), M, 0.0,
                kMaxHist, 0, Dhp, whp, zero);
        else
            anderson_update_kernel<float><<<update_grid(c), 256, 0, c->st>>>(
                c->w + M, static_cast<float *>(c->wh[c->cur]), static_cast<const float *>(c->Dh[c->cur]), M, 0.0,
                kMaxHist, 0, Dhp, whp, zero);
    }
    CK(cudaEventRecord(ev[3], c->st));
    CK(cudaEventSynchronize(ev[3]));
    CK(cudaGetLastError());
    float t[3];
    for (int i = 0; i < 3; i++) CK(cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]));
    for (auto &e : ev) cudaEventDestroy(e);
    c->launches += (long long)reps * 3;
    *ms_chain = t[0] / reps;
    *ms_concs = t[1] / reps;
    *ms_update = t[2] / reps;
    return LFTS_OK;
}

int lfts_get_tiles(const lfts_ctx *c, lfts_tiles *out)
{
    if (!c || !out) return LFTS_ERR_ARG;
    *out = current_tiles(c);
    return LFTS_OK;
}

int lfts_set_tiles(lfts_ctx *c, const lfts_tiles *t)
{
    if (!c || !t) return LFTS_ERR_ARG;
    DeviceGuard g(c->dev);
    CK(cudaStreamSynchronize(c->st));
    CK(cudaStreamSynchronize(c->st1));
    const lfts_tiles old = current_tiles(c);
    int rc = apply_tiles(c, *t);
    if (rc) {
        apply_tiles(c, old);  // leave the context as it was
        g_last_error = "tile choice not valid for this context's precision and mesh";
    }
    return rc;
}

int lfts_tuning(const lfts_ctx *c, int *pencil_cw, int *plane_stages)
{
    if (!c) return LFTS_ERR_ARG;
    if (pencil_cw) *pencil_cw = c->prec == LFTS_FP64 ? c->pe64.cw : c->pe32.cw;
    if (plane_stages) *plane_stages = c->prec == LFTS_FP64 ? 2 : c->plane_stages;
    return LFTS_OK;
}

long long lfts_kernel_launches(const lfts_ctx *c) { return c ? c->launches : 0; }

int lfts_anderson_stats(const lfts_ctx *c, long long *calls, long long *iterations)
{
    if (!c) return LFTS_ERR_ARG;
    if (calls) *calls = c->mix_calls;
    if (iterations) *iterations = c->mix_iters;
    return LFTS_OK;
}

int lfts_get_propagators(lfts_ctx *c, double *q_host)
{
    if (!c || !q_host) return LFTS_ERR_ARG;
    DeviceGuard g(c->dev);
    const long long n = 2 * c->M * (long long)c->N;
    std::memset(q_host, 0, sizeof(double) * 2 * c->M);
    if (c->prec == LFTS_FP64) {
        CK(cudaMemcpyAsync(q_host + 2 * c->M, c->q, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
    } else {
        if (c->phi_in_chain && c->fields_set) {
            // the chain that forms the concentration sums leaves the later slots
            // unstored: run the storing chain on the same fields
            c->phi_in_chain = false;
            enqueue_chain_launches<float>(c);
            c->phi_in_chain = true;
            CK(cudaGetLastError());
        }
        // FP32 slots hold (q_i, q^_{N+1-i}) pairs: back to the [q_i | q^] halves
        std::vector<float> tmp(n);
        CK(cudaMemcpyAsync(tmp.data(), c->q, sizeof(float) * n, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        const long long M = c->M;
        for (int sl = 0; sl < c->N; sl++) {
            const float *src = tmp.data() + (long long)sl * 2 * M;
            double *dst = q_host + (long long)(sl + 1) * 2 * M;
            for (long long r = 0; r < M; r++) {
                dst[r] = src[2 * r];
                dst[M + r] = src[2 * r + 1];
            }
        }
    }
    return LFTS_OK;
}

}  // extern "C"
