// Internal state of one L-FTS context (the opaque lfts_ctx of the C ABI),
// shared by the C ABI (lfts_capi.cu) and the ensemble (lfts_ensemble.cu).
#pragma once
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lfts_b200.h"
#include "fft_dispatch.h"
#include "field_kernels.cuh"

using namespace lfts;

struct lfts_ctx {
    lfts_params p{};
    int prec = 0, dev = 0;
    int N = 0, NA = 0, NB = 0;
    int mx = 0, my = 0, mz = 0, KZ = 0;
    long long M = 0, Mk = 0;
    size_t tsize = 8;  // bytes of the propagator type
    cudaStream_t st = nullptr;
    cudaStream_t st1 = nullptr;         // chain 1 of the contour chain runs here
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_h[2] = {};  // each chain's half of h written (two-stream FP64 chain)
    int sms = 148;

    double *w = nullptr;       // 4M: W-, w+, phi-, phi+
    void *q = nullptr;         // N slots x 2M, slot i at (i-1)*2M
    void *spec = nullptr;      // 2 x mx x my x KZ complex
    void *tw[3] = {};          // exp(-2 pi i t/m) per dimension
    void *gtab[3] = {};        // gx[mx], gy[my], gz[KZ] (gz carries 1/M)
    double *qpart = nullptr;   // mx per-plane sums of q_N
    double *Qd = nullptr;      // Q, ln Q
    double *partials = nullptr;
    double *red = nullptr;     // kRedWidth reduced values (device)
    double *red_host = nullptr;  // pinned copy
    int red_blocks = 0;

    double *eta[2] = {};       // Langevin noise: prev, new
    int eta_prev = 0;
    bool eta_set = false;

    void *Dh[kRedWidth] = {}, *wh[kRedWidth] = {};  // Anderson ring (physical buffers, propagator type)
    int phys[kRedWidth] = {};  // logical history slot -> physical buffer
    int cur = 0;               // physical buffer of the current iteration
    double DD[kRedWidth][kRedWidth] = {};

    double *S = nullptr;       // S(k) accumulator (Mk)
    void *skspec = nullptr;    // FP64 spectrum scratch for S(k)
    bool sk_own_spec = false;
    void *sktw[3] = {};        // FP64 twiddles (FP32 contexts only)
    int nsamples = 0;
    double sk_dK = -1.0;
    int sk_nbins = 0;
    int *sk_order = nullptr, *sk_wt = nullptr, *sk_bins = nullptr;
    double *sk_out = nullptr;
    std::vector<double> sk_K;  // K value reported for each bin

    void *sf_buf = nullptr;    // step_fwd scratch: q_in, q_out, h (2M each, FP64)
    double *adj_partial = nullptr;  // adjoint block partials [blocks][3]
    double *adj_buf = nullptr;      // checkpointed adjoint: recomputed q segment + discard row
    int adj_buf_slots = 0;
    AdjKernel adj{};

    PlaneKernels<double> pl64{};
    PencilKernels<double> pe64{};
    PlaneKernels<float> pl32{};
    PencilKernels<float> pe32{};
    int plane_stages = 2;     // yz-plane transform stages per axis (3: fft_plane3.cuh)
    int plane_split = 1;      // CTAs per x-plane of PLANE_G (8: the cluster kernel, fft_plane3c.cuh)
    int pf_ctas = 0;          // PLANE_G ahead of a summing pencil: prefetching CTAs past the planes
    PlaneSplitKernel psplit{};

    bool fields_set = false;
    bool have_concs = false;
    bool packed = false;      // FP32: both chains as one complex field (fft_packed.cuh)
    bool xh_chain = false;    // FP32 128^3: h and the q stores in the x-pencil (enqueue_chain_launches)
    bool phi_in_chain = false;  // with xh_chain: the concentration sums formed in the chain (PENCIL_HA)
    void *acc = nullptr;      // their (A, B) sums per mesh point, FP32 pairs
    bool use_graph = true;    // LFTS_NO_GRAPH=1: launch the chain kernel by kernel
    cudaGraph_t chain_graph = nullptr;
    cudaGraphExec_t chain_exec = nullptr;
    long long chain_kernels = 0;  // kernels in one replay of chain_exec
    // the device-side Anderson loop (anderson_device.cuh): one graph launch per
    // mix, selected by LFTS_DEVICE_MIX=1 (measured slower than the host-driven
    // loop on B200: each WHILE-node iteration costs more than a host round trip)
    bool mix_on_device = false;
    int mix_graph_state = 0;  // 0 not built, 1 built, -1 building failed (host loop)
    void *d_mix = nullptr;    // MixState
    double *d_lambda = nullptr;
    int lambda_cap = 0;       // largest maxIter the lambda table covers
    cudaGraph_t mix_graph = nullptr;
    cudaGraphExec_t mix_exec = nullptr;
    long long mix_body_kernels = 0;  // kernels per iteration of the mix graph's body
    bool mix_pdl = false;            // the body kept the chain's programmatic edges
    bool use_pdl = true;      // LFTS_NO_PDL=1 in the environment turns it off
    bool two_streams = true;  // LFTS_ONE_STREAM=1 runs both chains in each launch
    long long launches = 0;
    long long mix_calls = 0, mix_iters = 0;
};
