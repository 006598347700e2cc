// FP64 instantiations of the contour-step FFT kernels.
#include "fft_inst.cuh"

#define LFTS_PLANE_CASE_double(a, b) \
    if (ny == a && nz == b) { fill_plane<double, a, b>(o); return true; }
#define LFTS_PENCIL_CASE_double(a) \
    if (nx == a) { fill_pencil<double, a>(o); return true; }
#define LFTS_PENCIL_CW_CASE_double(a)                                   \
    if (nx == a) {                                                   \
        if (cw == 8) { fill_pencil<double, a, 8>(o); return true; }      \
        if (cw == 16) { fill_pencil<double, a, 16>(o); return true; }    \
        if (cw == 32) { fill_pencil<double, a, 32>(o); return true; }    \
        return false;                                                \
    }
LFTS_DEFINE_PLANE_DISPATCH(double)
LFTS_DEFINE_DISPATCH(double)

namespace lfts {
bool fft_length_supported(int n)
{
#define LFTS_LEN_CASE(a) if (n == a) return true;
    LFTS_FOR_EACH_LEN(LFTS_LEN_CASE)
#undef LFTS_LEN_CASE
    return false;
}
bool plane_pair_supported(int ny, int nz)
{
#define LFTS_PAIR_CASE(a, b) if (ny == a && nz == b) return true;
    LFTS_FOR_EACH_PAIR(LFTS_PAIR_CASE)
#undef LFTS_PAIR_CASE
    return false;
}
}  // namespace lfts

namespace lfts {
bool adjoint_kernel(int nx, AdjKernel *o)
{
    constexpr int CW = 16;
#define LFTS_ADJ_CASE(a)                                       \
    if (nx == a) {                                             \
        o->fn = pencil_adj_kernel<a, CW>;                      \
        o->nt = AdjCfg<a, CW>::NT;                             \
        o->smem = AdjCfg<a, CW>::SMEM;                         \
        o->cw = CW;                                            \
        return true;                                           \
    }
    LFTS_FOR_EACH_LEN(LFTS_ADJ_CASE)
#undef LFTS_ADJ_CASE
    return false;
}
}  // namespace lfts
