// lfts_step_fwd_noalloc: the contour step (step::fwd) for callers that must
// not allocate device memory -- code running where cudaMalloc is off limits
// (a host framework that owns every device allocation through its own pool,
// a real-time loop that may not call into the allocator, or a library layered
// under an allocator-free API).  The caller passes device inputs and outputs;
// the step's scratch (the two chains' half spectra, the per-plane Q partial
// sums and the twiddle / Boltzmann-weight tables) lives in one file-scope
// device array of fixed size, so this path makes no allocation at all.
//
// Limits and sharing rules, stated once here and in include/lfts_b200.h:
//  * FP64 only; 2 * mx * my * (mz/2 + 1) <= LFTS_NOALLOC_MAX_SPECTRUM complex
//    values (covers every mesh up to 64^3); each dimension one of the compiled
//    FFT lengths (<= 128).
//  * The array is one per device and shared by every call: two calls whose
//    kernels overlap on a GPU (different streams, or different host threads)
//    race on it.  Serialise them (one stream, or events).
//  * Nothing in the array has to start at zero: every call rewrites the tables
//    and the spectrum before reading them, and each plane's Q partial is
//    written before it is read.  The array keeps the last call's contents.
//  * The first call on a device looks up the array's device address (with
//    that device current); make that first call before any stream capture.
#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/lfts_b200.h"
#include "fft_dispatch.h"

using namespace lfts;

// error text reported by lfts_last_error_string (lfts_capi.cu)
void lfts_internal_set_error(const char *msg);

namespace {

constexpr long long kMaxSpec = LFTS_NOALLOC_MAX_SPECTRUM;  // complex values, both chains
constexpr int kMaxLen = 128;                               // largest compiled FFT length

struct NoallocLayout {
    static constexpr size_t spec = 0;
    static constexpr size_t tw = spec + sizeof(cpx<double>) * kMaxSpec;      // 3 x kMaxLen complex
    static constexpr size_t g = tw + sizeof(cpx<double>) * 3 * kMaxLen;      // 3 x kMaxLen doubles
    static constexpr size_t qpart = g + sizeof(double) * 3 * kMaxLen;        // kMaxLen doubles
    static constexpr size_t bytes = qpart + sizeof(double) * kMaxLen;
};

// the scratch: one per device, shared by all calls (see the rules above)
static __device__ __align__(256) unsigned char g_step_scratch[NoallocLayout::bytes];

constexpr int kMaxDevices = 64;
// device address of g_step_scratch per device, looked up once per device
// (std::call_once: host threads making their first calls together wait for
// one lookup).  The address belongs to the device's primary context: after
// cudaDeviceReset on a device it is stale, like every other handle of this
// library on that device.
unsigned char *g_scratch_addr[kMaxDevices] = {};
std::once_flag g_scratch_once[kMaxDevices];
cudaError_t g_scratch_err[kMaxDevices] = {};

// twiddles exp(-2 pi i t/n) and the factorised Boltzmann weight of
// src/step.cc:69-89 (1/M folded into the z factor), computed on the device
__global__ void noalloc_tables_kernel(cpx<double> *tw, double *g, int mx, int my, int mz, double Lx, double Ly,
                                      double Lz, int N, double M)
{
    const int n[3] = {mx, my, mz};
    const double L[3] = {Lx, Ly, Lz};
    const double two_pi = 6.283185307179586476925286766559005768;
    for (int d = 0; d < 3; d++) {
        for (int t = threadIdx.x; t < n[d]; t += blockDim.x) {
            double s, c;
            sincospi(-2.0 * t / n[d], &s, &c);
            tw[d * kMaxLen + t] = {c, s};
        }
        const int len = (d == 2) ? n[2] / 2 + 1 : n[d];
        for (int K = threadIdx.x; K < len; K += blockDim.x) {
            const int k = (d == 2 || K <= n[d] / 2) ? K : K - n[d];
            const double ksq = (double)k * k / (L[d] * L[d]);
            double v = exp(-two_pi * two_pi * ksq / (6.0 * N));
            if (d == 2) v /= M;
            g[d * kMaxLen + K] = v;
        }
    }
}

int fail(int code, const char *msg)
{
    lfts_internal_set_error(msg);
    return code;
}

// Per-device set-up, done by the first call on each device with that device
// current: the scratch array's device address.  Then, every call, the
// dynamic shared-memory limits of the kernels this mesh uses.
int device_setup(int dev, const PlaneKernels<double> &pl, const PencilKernels<double> &pe)
{
    std::call_once(g_scratch_once[dev], [dev] {
        void *p = nullptr;
        g_scratch_err[dev] = cudaGetSymbolAddress(&p, g_step_scratch);
        if (g_scratch_err[dev] == cudaSuccess && p) g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    });
    if (g_scratch_err[dev] != cudaSuccess || !g_scratch_addr[dev])
        return fail(LFTS_ERR_CUDA, "cudaGetSymbolAddress(g_step_scratch) failed");
    for (int m = 0; m < 4; m++)
        if (cudaFuncSetAttribute(pl.fn[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem) != cudaSuccess)
            return fail(LFTS_ERR_CUDA, "cudaFuncSetAttribute failed");
    for (int m = 0; m < 2; m++)
        if (cudaFuncSetAttribute(pe.fn[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pe.smem) != cudaSuccess)
            return fail(LFTS_ERR_CUDA, "cudaFuncSetAttribute failed");
    return LFTS_OK;
}

}  // namespace

extern "C" {

int lfts_step_fwd_noalloc(const lfts_params *p, const double *q_in, double *q_out, const double *h, int i,
                          void *stream)
{
    if (!p || !q_in || !q_out || !h) return fail(LFTS_ERR_ARG, "null pointer");
    const int mx = p->m[0], my = p->m[1], mz = p->m[2];
    if (p->N < 2 || i < 1 || i >= p->N || p->NA < 0 || p->NA > p->N)
        return fail(LFTS_ERR_ARG, "chain lengths or monomer index out of range");
    if (mx < 1 || my < 1 || mz < 1 || mx > kMaxLen || my > kMaxLen || mz > kMaxLen)
        return fail(LFTS_ERR_ARG, "mesh dimension above the no-alloc limit of 128");
    for (int d = 0; d < 3; d++)
        if (!(p->L[d] > 0.0) || !std::isfinite(p->L[d]))
            return fail(LFTS_ERR_ARG, "box lengths must be positive and finite");
    const long long KZ = mz / 2 + 1;
    if (2LL * mx * my * KZ > kMaxSpec)
        return fail(LFTS_ERR_ARG, "mesh above the no-alloc scratch limit: 2*mx*my*(mz/2+1) must be <= "
                                  "LFTS_NOALLOC_MAX_SPECTRUM (64^3 meshes fit)");
    PlaneKernels<double> pl{};
    PencilKernels<double> pe{};
    if (!plane_kernels(my, mz, &pl) || !pencil_kernels(mx, &pe))
        return fail(LFTS_ERR_UNSUPPORTED, "mesh size without an FFT kernel");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(LFTS_ERR_CUDA, "no current CUDA device");
    int rc = device_setup(dev, pl, pe);
    if (rc) return rc;

    unsigned char *base = g_scratch_addr[dev];
    cpx<double> *spec = reinterpret_cast<cpx<double> *>(base + NoallocLayout::spec);
    cpx<double> *tw = reinterpret_cast<cpx<double> *>(base + NoallocLayout::tw);
    double *g = reinterpret_cast<double *>(base + NoallocLayout::g);
    double *qpart = reinterpret_cast<double *>(base + NoallocLayout::qpart);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long M = (long long)mx * my * mz;
    const int NB = p->N - p->NA;

    noalloc_tables_kernel<<<1, 128, 0, st>>>(tw, g, mx, my, mz, p->L[0], p->L[1], p->L[2], p->N, (double)M);

    PlaneArgs<double> a{};
    a.src = q_in;
    a.src_stride = M;
    a.spec = spec;
    a.twy = tw + kMaxLen;
    a.twz = tw + 2 * kMaxLen;
    a.qpart = qpart;
    a.nchains = 2;
    a.Nd = (double)p->N;
    pl.fn[PLANE_INIT_Q]<<<dim3(mx, 2), pl.nt, pl.smem, st>>>(a);

    PencilArgs<double> pa{};
    pa.spec = spec;
    pa.twx = tw;
    pa.gx = g;
    pa.gy = g + kMaxLen;
    pa.gz = g + 2 * kMaxLen;
    pa.ncol = my * (int)KZ;
    pa.KZ = (int)KZ;
    pe.fn[PENCIL_CONV]<<<dim3((pa.ncol + pe.cw - 1) / pe.cw, 2), pe.nt, pe.smem, st>>>(pa);

    a.qout = q_out;
    a.h = h;
    a.hsel0 = i < p->NA ? 0 : 1;  // src/step.cc:53-57
    a.hsel1 = i < NB ? 1 : 0;     // src/step.cc:60-64
    pl.fn[PLANE_LAST]<<<dim3(mx, 2), pl.nt, pl.smem, st>>>(a);

    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(LFTS_ERR_CUDA, cudaGetErrorString(e));
    return LFTS_OK;
}

}  // extern "C"
