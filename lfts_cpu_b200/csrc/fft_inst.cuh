// Instantiation lists of the FFT kernels, shared by fft_fp64.cu / fft_fp32.cu.
#pragma once
#include "fft_dispatch.h"
#include "fft_packed.cuh"

// line lengths (each needs a Plan<> in dft.cuh)
#define LFTS_FOR_EACH_LEN(X) X(8) X(12) X(16) X(20) X(24) X(32) X(40) X(48) X(64) X(80) X(96) X(128)
// (ny, nz) plane pairs: the cubic ones plus a few boxes used by tests
#define LFTS_FOR_EACH_PAIR(X)                                                                  \
    X(8, 8) X(12, 12) X(16, 16) X(20, 20) X(24, 24) X(32, 32) X(40, 40) X(48, 48) X(64, 64)   \
    X(80, 80) X(96, 96) X(128, 128) X(12, 20) X(24, 16) X(16, 32) X(32, 64)

namespace lfts {

template <typename T, int NY, int NZ>
static void fill_plane(PlaneKernels<T> *o)
{
    using C = PlaneCfg<T, NY, NZ>;
    o->fn[PLANE_INIT_W] = plane_kernel<T, NY, NZ, PLANE_INIT_W>;
    o->fn[PLANE_INIT_Q] = plane_kernel<T, NY, NZ, PLANE_INIT_Q>;
    o->fn[PLANE_STEP] = plane_kernel<T, NY, NZ, PLANE_STEP>;
    o->fn[PLANE_LAST] = plane_kernel<T, NY, NZ, PLANE_LAST>;
    o->fn[PLANE_G] = nullptr;
    o->nt = C::NT;
    o->smem = C::SMEM;
}

template <typename T, int NY, int NZ>
static void fill_plane_c(PlaneKernels<T> *o)
{
    using C = PlaneCCfg<T, NY, NZ>;
    o->fn[PLANE_INIT_W] = plane_c_kernel<T, NY, NZ, PLANE_INIT_W>;
    o->fn[PLANE_INIT_Q] = plane_c_kernel<T, NY, NZ, PLANE_INIT_Q>;
    o->fn[PLANE_STEP] = plane_c_kernel<T, NY, NZ, PLANE_STEP>;
    o->fn[PLANE_LAST] = plane_c_kernel<T, NY, NZ, PLANE_LAST>;
    o->fn[PLANE_G] = nullptr;
    o->nt = C::NT;
    o->smem = C::SMEM;
}

template <typename T, int NX, int CW = 32>
static void fill_pencil(PencilKernels<T> *o)
{
    using C = PencilCfg<T, NX, CW>;
    o->fn[PENCIL_CONV] = pencil_kernel<T, NX, CW, PENCIL_CONV>;
    // S(k) samples run in FP64 in both precisions
    if constexpr (sizeof(T) == sizeof(double))
        o->fn[PENCIL_POWER] = pencil_kernel<T, NX, CW, PENCIL_POWER>;
    else
        o->fn[PENCIL_POWER] = nullptr;
    // the h-in-pencil chain: FP32 packed field, 96- and 128-point x lines (at 64
    // the pencil's added h and q traffic cost more than the plane kernel saves)
    if constexpr (sizeof(T) == sizeof(float) && (NX == 96 || NX == 128)) {
        o->fn[PENCIL_H] = pencil_kernel<T, NX, CW, PENCIL_H>;
        o->fn[PENCIL_H_LAST] = pencil_kernel<T, NX, CW, PENCIL_H_LAST>;
        o->fn[PENCIL_INIT_W] = pencil_kernel<T, NX, CW, PENCIL_INIT_W>;
        o->fn[PENCIL_HA] = pencil_kernel<T, NX, CW, PENCIL_HA>;
        o->fn[PENCIL_HA_LAST] = pencil_kernel<T, NX, CW, PENCIL_HA_LAST>;
    } else {
        o->fn[PENCIL_H] = o->fn[PENCIL_H_LAST] = o->fn[PENCIL_INIT_W] = nullptr;
        o->fn[PENCIL_HA] = o->fn[PENCIL_HA_LAST] = nullptr;
    }
    o->nt = C::NT;
    o->smem = C::SMEM;
    o->cw = CW;
}

}  // namespace lfts

// pencils of one precision (both); half-spectrum plane kernels (FP64 only:
// FP32 contexts use the packed-field kernels)
#define LFTS_DEFINE_PLANE_DISPATCH(T)                                                 \
    namespace lfts {                                                                  \
    bool plane_kernels(int ny, int nz, PlaneKernels<T> *o)                            \
    {                                                                                 \
        LFTS_FOR_EACH_PAIR(LFTS_PLANE_CASE_##T)                                       \
        return false;                                                                 \
    }                                                                                 \
    }
#define LFTS_DEFINE_DISPATCH(T)                                                       \
    namespace lfts {                                                                  \
    bool pencil_kernels(int nx, PencilKernels<T> *o)                                  \
    {                                                                                 \
        LFTS_FOR_EACH_LEN(LFTS_PENCIL_CASE_##T)                                       \
        return false;                                                                 \
    }                                                                                 \
    bool pencil_kernels(int nx, int cw, PencilKernels<T> *o)                          \
    {                                                                                 \
        LFTS_FOR_EACH_LEN(LFTS_PENCIL_CW_CASE_##T)                                    \
        return false;                                                                 \
    }                                                                                 \
    }
