// FP32 instantiations of the contour-step FFT kernels (the FP32-mixed path).
#include "fft_inst.cuh"
#include "fft_plane3.cuh"
#include "fft_plane3c.cuh"

#define LFTS_PENCIL_CASE_float(a) \
    if (nx == a) { fill_pencil<float, a>(o); return true; }
#define LFTS_PENCIL_CW_CASE_float(a)                                   \
    if (nx == a) {                                                   \
        if (cw == 8) { fill_pencil<float, a, 8>(o); return true; }      \
        if (cw == 16) { fill_pencil<float, a, 16>(o); return true; }    \
        if (cw == 32) { fill_pencil<float, a, 32>(o); return true; }    \
        return false;                                                \
    }
LFTS_DEFINE_DISPATCH(float)

#define LFTS_PLANE_C_CASE(a, b) \
    if (ny == a && nz == b) { fill_plane_c<float, a, b>(o); return true; }
namespace lfts {
bool plane_c_kernels(int ny, int nz, PlaneKernels<float> *o)
{
    LFTS_FOR_EACH_PAIR(LFTS_PLANE_C_CASE)
    return false;
}
template <typename C>
static void fill_plane3(PlaneKernels<float> *o)
{
    o->fn[PLANE_INIT_W] = plane3_kernel<C, PLANE_INIT_W>;
    o->fn[PLANE_INIT_Q] = plane3_kernel<C, PLANE_INIT_Q>;
    o->fn[PLANE_STEP] = plane3_kernel<C, PLANE_STEP>;
    o->fn[PLANE_LAST] = plane3_kernel<C, PLANE_LAST>;
    // the h-in-pencil chain runs on 96 x 96 and 128 x 128 planes
    if constexpr (C::NY == 96 || C::NY == 128)
        o->fn[PLANE_G] = plane3_kernel<C, PLANE_G>;
    else
        o->fn[PLANE_G] = nullptr;
    o->nt = C::NT;
    o->smem = C::SMEM;
}
bool plane3_kernels(int ny, int nz, PlaneKernels<float> *o)
{
    if (ny != nz) return false;
    if (ny == 128) { fill_plane3<Plane3_128>(o); return true; }
    if (ny == 96) { fill_plane3<Plane3_96>(o); return true; }
    if (ny == 64) { fill_plane3<Plane3_64>(o); return true; }
    return false;
}
bool plane_split_kernel(int ny, int nz, PlaneSplitKernel *o)
{
    if (ny != 128 || nz != 128) return false;
    o->fn = plane3_split_g_kernel<Plane3Split128>;
    o->cl = Plane3Split128::CL;
    o->nt = Plane3Split128::NT;
    o->smem = Plane3Split128::SMEM;
    return true;
}
}  // namespace lfts
