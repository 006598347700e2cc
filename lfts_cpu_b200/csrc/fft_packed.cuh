// Packed-chain yz-plane kernel (FP32-mixed path).
//
// Both chains are real and the Boltzmann weight g(k) is real and even, so the
// two propagators of a contour step travel as ONE complex field
//     Z = q_i + i q^_{N+1-i}
// through a full complex 3-D transform: FFT(Z) = FFT(q) + i FFT(q^), the
// product with g keeps that split, and after the inverse transform Re Z is
// chain 1 and Im Z is chain 2 (each then multiplied by its own h).  Compared
// with two half-spectrum real transforms (plane_kernel) this removes the
// row-pair packing/unpacking and the packed Nyquist column, at the same FFT
// count.  A 128x128 complex FP32 plane (139 KB with padding) fits one CTA.
//
// Stored propagators (FP32 packed path): slot i holds the M pairs
// (q_i(r), q^_{N+1-i}(r)), one 8-byte store per mesh point; slot 1 is
// (hA(r), hB(r)).
//
// Spectrum layout: full complex [x][ky][kz], kz in [0, mz); the x-pencil
// kernel runs on it unchanged with ncol = my*mz and an even kz weight table.
// Each CTA owns one x-plane; warps own whole z lines (rows) in the z section.
#pragma once
#include "fft_kernels.cuh"

namespace lfts {

template <typename T, int NY, int NZ>
struct PlaneCCfg {
    static constexpr int RY1 = Plan<NY>::R1, RY2 = Plan<NY>::R2;
    static constexpr int RZ1 = Plan<NZ>::R1, RZ2 = Plan<NZ>::R2;
    static constexpr int KC = NZ;  // columns of the y phases
    // one pad slot per 16 slots of a z line (stage-B blocks of RZ2 = 8 then hit
    // distinct banks); row pitch = 8 (mod 16) so a warp's rows alternate bank
    // halves
    static constexpr int ZSPAN = NZ + (NZ - 1) / 16;
    static constexpr int KP = (ZSPAN + 7) / 16 * 16 + 8;
    static constexpr int NT0 = KC * RY2 > NY * RZ2 / 4 ? KC * RY2 : NY * RZ2 / 4;
    static constexpr int NT = NT0 > 1024 ? 1024 : (NT0 + 127) / 128 * 128;
    static constexpr int NW = NT / 32;
    static constexpr int ROWS_PER_WARP = (NY + NW - 1) / NW;
    static constexpr int TAP = RZ1 + 1, TBP = RZ2 + 1;
    static constexpr int NTA = RZ2 * TAP, NTB = RZ1 * TBP;
    static constexpr size_t SMEM = sizeof(cpx<T>) * (size_t)(NY * KP + NY + NTA + NTB);
    static __device__ __forceinline__ int zpos(int s) { return s + s / 16; }
    static __device__ __forceinline__ int ymap(int p) { return p / RY2 + RY1 * (p % RY2); }
    static __device__ __forceinline__ int zmap(int p) { return p / RZ2 + RZ1 * (p % RZ2); }
    static __device__ __forceinline__ int ta(int j2, int k1) { return j2 * TAP + k1; }
    static __device__ __forceinline__ int tb(int k1, int u) { return k1 * TBP + u; }
    static_assert(KC * RY2 <= NT, "one y stage-A task per thread");
};

// rows owned by warp w in the z section
template <typename C>
__device__ __forceinline__ void warp_rows(int w, int &r0, int &nr)
{
    constexpr int NY = C::RY1 * C::RY2;
    r0 = (w * NY) / C::NW;
    nr = ((w + 1) * NY) / C::NW - r0;
}

// ------------------------------------------------------------------ y phases
// inverse stage A from the global spectrum (natural ky, natural kz)
template <typename C, typename T>
__device__ __forceinline__ void pc_y_invA_load(const cpx<T> *__restrict__ Sg, cpx<T> (&v)[C::RY1])
{
    constexpr int KC = C::KC, R1 = C::RY1, R2 = C::RY2;
    const int t = threadIdx.x;
    if (t < KC * R2) {
        const int col = t % KC, j2 = t / KC;
#pragma unroll
        for (int a = 0; a < R1; a++) v[a] = Sg[(j2 + R2 * a) * KC + col];
    }
}

template <typename C, typename T>
__device__ __forceinline__ void pc_y_A(cpx<T> *P, cpx<T> (&v)[C::RY1], const cpx<T> *twy, bool from_regs)
{
    // S = +1 (inverse, from_regs) writes w^-(j2 k1); forward from smem writes w^+(j2 k1)
    constexpr int KC = C::KC, KP = C::KP, R1 = C::RY1, R2 = C::RY2, NY = R1 * R2;
    const int t = threadIdx.x;
    if (t < KC * R2) {
        const int col = t % KC, j2 = t / KC, pc = C::zpos(col);
        if (from_regs) {
            Dft<R1, 1, T>::run(v);
#pragma unroll
            for (int k1 = 0; k1 < R1; k1++) P[(j2 + R2 * k1) * KP + pc] = ctw<1>(v[k1], twy[(j2 * k1) % NY]);
        } else {
#pragma unroll
            for (int a = 0; a < R1; a++) v[a] = P[(j2 + R2 * a) * KP + pc];
            Dft<R1, -1, T>::run(v);
#pragma unroll
            for (int k1 = 0; k1 < R1; k1++) P[(j2 + R2 * k1) * KP + pc] = ctw<-1>(v[k1], twy[(j2 * k1) % NY]);
        }
    }
}

// stage B in place with sign S; TW: twiddle w^(S j2 k1) after the DFT
template <typename C, int S, bool TW, typename T>
__device__ __forceinline__ void pc_y_B(cpx<T> *P, const cpx<T> *twy)
{
    constexpr int KC = C::KC, KP = C::KP, R1 = C::RY1, R2 = C::RY2, NY = R1 * R2;
    for (int t = threadIdx.x; t < KC * R1; t += C::NT) {
        const int col = t % KC, k1 = t / KC, pc = C::zpos(col);
        cpx<T> v[R2];
#pragma unroll
        for (int u = 0; u < R2; u++) v[u] = P[(R2 * k1 + u) * KP + pc];
        Dft<R2, S, T>::run(v);
#pragma unroll
        for (int u = 0; u < R2; u++) P[(R2 * k1 + u) * KP + pc] = TW ? ctw<S>(v[u], twy[(u * k1) % NY]) : v[u];
    }
}

// forward stage B -> global natural ky (after stage A with twiddles); the
// z order of the columns is given by KZMAP (transposed after an INIT z pass)
template <typename C, bool KZT, typename T>
__device__ __forceinline__ void pc_y_fwdB_global(const cpx<T> *P, cpx<T> *__restrict__ Sg)
{
    constexpr int KC = C::KC, KP = C::KP, R1 = C::RY1, R2 = C::RY2;
    for (int t = threadIdx.x; t < KC * R1; t += C::NT) {
        const int col = t % KC, k1 = t / KC, pc = C::zpos(col);
        const int kz = KZT ? C::zmap(col) : col;
        cpx<T> v[R2];
#pragma unroll
        for (int u = 0; u < R2; u++) v[u] = P[(R2 * k1 + u) * KP + pc];
        Dft<R2, -1, T>::run(v);
#pragma unroll
        for (int k2 = 0; k2 < R2; k2++) Sg[(k1 + R1 * k2) * KC + kz] = v[k2];
    }
}

// forward stage A -> global natural ky (end of transposed -> natural)
template <typename C, typename T>
__device__ __forceinline__ void pc_y_fwdA_global(const cpx<T> *P, cpx<T> *__restrict__ Sg)
{
    constexpr int KC = C::KC, KP = C::KP, R1 = C::RY1, R2 = C::RY2;
    const int t = threadIdx.x;
    if (t < KC * R2) {
        const int col = t % KC, j2 = t / KC, pc = C::zpos(col);
        cpx<T> v[R1];
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) v[k1] = P[(j2 + R2 * k1) * KP + pc];
        Dft<R1, -1, T>::run(v);
#pragma unroll
        for (int j1 = 0; j1 < R1; j1++) Sg[(j2 + R2 * j1) * KC + col] = v[j1];
    }
}

// ------------------------------------------------------------------ z phases
// stage A in place over this warp's rows: S = +1 inverse (twiddle after, NT
// order) or S = -1 forward with twiddles (INIT, natural -> transposed), or
// S = -1 without twiddles (transposed -> natural, end of the forward).
template <typename C, int S, bool TW, typename T>
__device__ __forceinline__ void pc_z_A(cpx<T> *P, const cpx<T> *twa)
{
    constexpr int KP = C::KP, R1 = C::RZ1, R2 = C::RZ2;
    int r0, nr;
    warp_rows<C>(threadIdx.x >> 5, r0, nr);
    const int lane = threadIdx.x & 31;
    for (int t = lane; t < nr * R2; t += 32) {
        const int row = r0 + t / R2, j2 = t % R2;
        cpx<T> *Z = P + row * KP;
        cpx<T> v[R1];
#pragma unroll
        for (int a = 0; a < R1; a++) v[a] = Z[C::zpos(j2 + R2 * a)];
        Dft<R1, S, T>::run(v);
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) Z[C::zpos(j2 + R2 * k1)] = TW ? ctw<S>(v[k1], twa[C::ta(j2, k1)]) : v[k1];
    }
}

// stage B, forward, no twiddles (INIT: natural -> transposed)
template <typename C, typename T>
__device__ __forceinline__ void pc_z_fwdB(cpx<T> *P)
{
    constexpr int KP = C::KP, R1 = C::RZ1, R2 = C::RZ2;
    int r0, nr;
    warp_rows<C>(threadIdx.x >> 5, r0, nr);
    const int lane = threadIdx.x & 31;
    for (int t = lane; t < nr * R1; t += 32) {
        const int row = r0 + t / R1, k1 = t % R1;
        cpx<T> *Z = P + row * KP;
        cpx<T> v[R2];
#pragma unroll
        for (int u = 0; u < R2; u++) v[u] = Z[C::zpos(R2 * k1 + u)];
        Dft<R2, -1, T>::run(v);
#pragma unroll
        for (int u = 0; u < R2; u++) Z[C::zpos(R2 * k1 + u)] = v[u];
    }
}

// h values of this warp's stage-B tasks (rows in transposed y order); loaded
// before the first z phase so the DRAM latency overlaps its shared-memory work.
// 8-byte pair load / streaming store of the stored propagators
__device__ __forceinline__ cpx<float> ld_pair(const cpx<float> *p)
{
    const float2 v = __ldg(reinterpret_cast<const float2 *>(p));
    return {v.x, v.y};
}
__device__ __forceinline__ void st_pair(cpx<float> *p, float a, float b)
{
    __stcs(reinterpret_cast<float2 *>(p), make_float2(a, b));
}
__device__ __forceinline__ cpx<double> ld_pair(const cpx<double> *p)
{
    const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    return {v.x, v.y};
}
__device__ __forceinline__ void st_pair(cpx<double> *p, double a, double b)
{
    __stcs(reinterpret_cast<double2 *>(p), make_double2(a, b));
}

template <typename C, typename T>
struct PcH {
    static constexpr int R1 = C::RZ1, R2 = C::RZ2, NZ = R1 * R2;
    static constexpr int RND = (C::ROWS_PER_WARP * R1 + 31) / 32;
    T v[RND][R2][2];
    // rounds [s0, s1) of this lane's tasks; hp = this plane's (hA, hB) pairs,
    // chain c takes hB when hsel_c = 1
    __device__ __forceinline__ void load(const cpx<T> *__restrict__ hp, int hsel0, int hsel1, int s0, int s1)
    {
        int r0, nr;
        warp_rows<C>(threadIdx.x >> 5, r0, nr);
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int s = 0; s < RND; s++) {
            if (s < s0 || s >= s1) continue;
            const int t = lane + 32 * s;
            if (t < nr * R1) {
                const int y = C::ymap(r0 + t / R1), k1 = t % R1;
#pragma unroll
                for (int k2 = 0; k2 < R2; k2++) {
                    const cpx<T> h = ld_pair(hp + y * NZ + k1 + R1 * k2);
                    v[s][k2][0] = hsel0 ? h.y : h.x;
                    v[s][k2][1] = hsel1 ? h.y : h.x;
                }
            }
        }
    }
};

// inverse stage B -> real space (Re: chain 1, Im: chain 2) times h, store
// both propagators; STEP: forward stage B with twiddles; LAST: chain-1 sum.
template <typename C, int MODE, typename T>
__device__ __forceinline__ void pc_z_invB_h(cpx<T> *P, const cpx<T> *twb, const PcH<C, T> &hv,
                                            cpx<T> *__restrict__ qp, double &qsum)
{
    constexpr int KP = C::KP, R1 = C::RZ1, R2 = C::RZ2, NZ = R1 * R2;
    constexpr int RND = PcH<C, T>::RND;
    int r0, nr;
    warp_rows<C>(threadIdx.x >> 5, r0, nr);
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 0; s < RND; s++) {
        const int t = lane + 32 * s;
        if (t >= nr * R1) continue;
        const int row = r0 + t / R1, k1 = t % R1;
        const int y = C::ymap(row);
        cpx<T> *Z = P + row * KP;
        cpx<T> v[R2];
#pragma unroll
        for (int u = 0; u < R2; u++) v[u] = Z[C::zpos(R2 * k1 + u)];
        Dft<R2, 1, T>::run(v);
#pragma unroll
        for (int k2 = 0; k2 < R2; k2++) {
            const int z = k1 + R1 * k2;
            const T a = v[k2].x * hv.v[s][k2][0];
            const T b = v[k2].y * hv.v[s][k2][1];
            st_pair(qp + y * NZ + z, a, b);
            if (MODE == PLANE_LAST) qsum += (double)a;
            v[k2] = {a, b};
        }
        if (MODE == PLANE_STEP) {
            Dft<R2, -1, T>::run(v);
#pragma unroll
            for (int u = 0; u < R2; u++) Z[C::zpos(R2 * k1 + u)] = ctw<-1>(v[u], twb[C::tb(k1, u)]);
        }
    }
}

// twiddle tables: twy[NY], TA, TB (as in plane_kernel)
template <typename C, typename T>
struct PcTw {
    static constexpr int NY = C::RY1 * C::RY2, NZ = C::RZ1 * C::RZ2;
    static constexpr int TOT = NY + C::NTA + C::NTB;
    static constexpr int PER = (TOT + C::NT - 1) / C::NT;
    cpx<T> r[PER];
    static __device__ __forceinline__ int src(int t)
    {
        if (t < NY) return t;
        t -= NY;
        if (t < C::NTA) {
            const int j2 = t / C::TAP, k1 = t % C::TAP;
            return k1 < C::RZ1 ? (j2 * k1) % NZ : 0;
        }
        t -= C::NTA;
        const int k1 = t / C::TBP, u = t % C::TBP;
        return u < C::RZ2 ? (u * k1) % NZ : 0;
    }
    __device__ __forceinline__ void load(const cpx<T> *__restrict__ twy_g, const cpx<T> *__restrict__ twz_g)
    {
#pragma unroll
        for (int s = 0; s < PER; s++) {
            const int t = threadIdx.x + s * C::NT;
            if (t < NY)
                r[s] = twy_g[t];
            else if (t < TOT)
                r[s] = twz_g[src(t)];
        }
    }
    __device__ __forceinline__ void store(cpx<T> *tw)
    {
#pragma unroll
        for (int s = 0; s < PER; s++) {
            const int t = threadIdx.x + s * C::NT;
            if (t < TOT) tw[t] = r[s];
        }
    }
};

// body of one CTA: x-plane x of an mx-plane field (the ensemble's batched
// launches call it with their own plane numbering)
template <typename T, int NY, int NZ, int MODE>
__device__ __forceinline__ void plane_c_body(const PlaneArgs<T> &a, const int x, const int mx)
{
    using C = PlaneCCfg<T, NY, NZ>;
    constexpr int KP = C::KP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T> *P = reinterpret_cast<cpx<T> *>(smem_raw);
    cpx<T> *twy = P + NY * KP;
    cpx<T> *twa = twy + NY;
    cpx<T> *twb = twa + C::NTA;

    const long long M = (long long)mx * NY * NZ;
    const long long plane_off = (long long)x * NY * NZ;
    cpx<T> *Sg = a.spec + (long long)x * NY * NZ;

    PcTw<C, T> tws;
    tws.load(a.twy, a.twz);
    pdl_launch_dependents();
    pdl_wait();

    if (MODE == PLANE_INIT_W || MODE == PLANE_INIT_Q) {
        tws.store(twy);
        int r0, nr;
        warp_rows<C>(threadIdx.x >> 5, r0, nr);
        const int lane = threadIdx.x & 31;
        // rows in natural y order: Z = q + i q^
        for (int t = lane; t < nr * NZ; t += 32) {
            const int y = r0 + t / NZ, z = t % NZ;
            const long long i = plane_off + (long long)y * NZ + z;
            T v1, v2;
            if (MODE == PLANE_INIT_W) {
                // hA = exp(-(W- + w+)/N), hB = exp(-(-W- + w+)/N)  (src/diblock.cc:64-72)
                const double wm = a.w[i], wp = a.w[M + i];
                v1 = (T)exp(-(wm + wp) / a.Nd);
                v2 = (T)exp(-(-wm + wp) / a.Nd);
                reinterpret_cast<cpx<T> *>(a.qout)[i] = {v1, v2};
            } else if (a.src) {
                v1 = a.src[i];
                v2 = a.src[a.src_stride + i];
            } else {
                v1 = (T)a.src64[i];
                v2 = (T)a.src64[a.src_stride + i];
            }
            P[y * KP + C::zpos(z)] = {v1, v2};
        }
        __syncthreads();  // twiddle tables (and rows)
        pc_z_A<C, -1, true>(P, twa);
        __syncwarp();
        pc_z_fwdB<C>(P);
        __syncthreads();
        {
            cpx<T> v[C::RY1];
            pc_y_A<C>(P, v, twy, false);
        }
        __syncthreads();
        pc_y_fwdB_global<C, true>(P, Sg);
        return;
    }

    {
        cpx<T> v[C::RY1];
        pc_y_invA_load<C>(Sg, v);
        tws.store(twy);
        __syncthreads();
        pc_y_A<C>(P, v, twy, true);
    }
    __syncthreads();
    pc_y_B<C, 1, false>(P, twy);
    __syncthreads();
    // z section, warp-local (rows in transposed y order)
    // h of the first stage-B round goes out before the first z phase, the
    // rest after it (register budget)
    PcH<C, T> hv;
    const cpx<T> *hp = reinterpret_cast<const cpx<T> *>(a.h) + plane_off;
    hv.load(hp, a.hsel0, a.hsel1, 0, 1);
    pc_z_A<C, 1, true>(P, twa);
    hv.load(hp, a.hsel0, a.hsel1, 1, PcH<C, T>::RND);
    __syncwarp();
    cpx<T> *qp = reinterpret_cast<cpx<T> *>(a.qout) + plane_off;
    double qsum = 0.0;
    pc_z_invB_h<C, MODE>(P, twb, hv, qp, qsum);
    if (MODE == PLANE_LAST) {
        __shared__ double red[C::NT / 32];
        for (int o = 16; o > 0; o >>= 1) qsum += __shfl_xor_sync(0xffffffffu, qsum, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = qsum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int i = 0; i < C::NT / 32; i++) s += red[i];
            a.qpart[x] = s;
        }
        return;
    }
    __syncwarp();
    pc_z_A<C, -1, false>(P, twa);
    __syncthreads();
    pc_y_B<C, -1, true>(P, twy);
    __syncthreads();
    pc_y_fwdA_global<C>(P, Sg);
}

template <typename T, int NY, int NZ, int MODE>
__global__ void __launch_bounds__(PlaneCCfg<T, NY, NZ>::NT, 1) plane_c_kernel(PlaneArgs<T> a)
{
    plane_c_body<T, NY, NZ, MODE>(a, blockIdx.x, gridDim.x);
}

}  // namespace lfts
