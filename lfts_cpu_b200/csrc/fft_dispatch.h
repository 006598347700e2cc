// Lookup of the compiled FFT kernels by mesh size (one translation unit per
// precision instantiates them: fft_fp64.cu, fft_fp32.cu).
#pragma once
#include <cstddef>

#include "adjoint.cuh"
#include "fft_kernels.cuh"

namespace lfts {

template <typename T>
struct PlaneKernels {
    void (*fn[kPlaneModes])(PlaneArgs<T>);  // indexed by PlaneMode (null: not compiled)
    int nt;
    size_t smem;
};

template <typename T>
struct PencilKernels {
    void (*fn[kPencilModes])(PencilArgs<T>);  // indexed by PencilMode (null: not compiled)
    int nt;
    size_t smem;
    int cw;
};

// false when (ny, nz) / nx has no compiled instantiation
// packed-chain plane kernels (fft_packed.cuh), FP32
bool plane_c_kernels(int ny, int nz, PlaneKernels<float> *out);
// three-stage packed-chain plane kernels (fft_plane3.cuh), FP32: 64, 96, 128 square planes
bool plane3_kernels(int ny, int nz, PlaneKernels<float> *out);
// PLANE_G with each x-plane split over a thread-block cluster of cl CTAs
// (fft_plane3c.cuh), FP32: 128 x 128 planes
struct PlaneSplitKernel {
    void (*fn)(PlaneArgs<float>);
    int cl, nt;
    size_t smem;
};
bool plane_split_kernel(int ny, int nz, PlaneSplitKernel *out);
bool plane_kernels(int ny, int nz, PlaneKernels<double> *out);
bool pencil_kernels(int nx, PencilKernels<double> *out);
bool pencil_kernels(int nx, PencilKernels<float> *out);
// x-pencil kernels of tile width cw (columns per CTA: 8, 16 or 32); the tile
// width changes only the work split, not any column's arithmetic
bool pencil_kernels(int nx, int cw, PencilKernels<double> *out);
bool pencil_kernels(int nx, int cw, PencilKernels<float> *out);
struct AdjKernel {
    void (*fn)(AdjArgs);
    int nt;
    size_t smem;
    int cw;
};
// adjoint x-pencil (FP64) for line length nx
bool adjoint_kernel(int nx, AdjKernel *out);

// line lengths with a two-stage plan
bool fft_length_supported(int n);
// (ny, nz) plane pairs with an instantiation
bool plane_pair_supported(int ny, int nz);

}  // namespace lfts
