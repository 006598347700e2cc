// FP32 instantiations of the contour-step FFT kernels (the FP32-mixed path).
#include "fft_inst.cuh"

#define LFTS_PLANE_CASE_float(a, b) \
    if (ny == a && nz == b) { fill_plane<float, a, b>(o); return true; }
#define LFTS_PENCIL_CASE_float(a) \
    if (nx == a) { fill_pencil<float, a>(o); return true; }
LFTS_DEFINE_DISPATCH(float)

#define LFTS_PLANE_C_CASE(a, b) \
    if (ny == a && nz == b) { fill_plane_c<float, a, b>(o); return true; }
namespace lfts {
bool plane_c_kernels(int ny, int nz, PlaneKernels<float> *o)
{
    LFTS_FOR_EACH_PAIR(LFTS_PLANE_C_CASE)
    return false;
}
}  // namespace lfts
