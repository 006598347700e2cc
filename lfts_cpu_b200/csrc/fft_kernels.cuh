// Fused contour-step kernels for sm_100a.
//
// One contour step of the reference (step::fwd, src/step.cc:35-65) is
//     q_{i+1} = h .* IFFT3( g .* FFT3(q_i) )
// for two chains at once.  Here a 3-D transform is split into
//   * a yz-plane pass (one CTA per x-plane per chain): inverse y, inverse z
//     (complex-to-real), multiply by h, store q_{i+1}, forward z
//     (real-to-complex), forward y -- i.e. the end of step i and the start of
//     step i+1 fused, with the whole plane's half spectrum resident in shared
//     memory (my x (mz/2+1) complex values);
//   * an x-pencil pass (one CTA per tile of (ky,kz) columns per chain):
//     forward x, multiply by g(k), inverse x.
// Each 1-D transform of length n = R1*R2 runs as two in-register radix
// stages separated by one shared-memory exchange: stage "A" works on the
// strided sets {j2 + R2 t}, stage "B" on the contiguous blocks {R2 k1 + u}.
// Running A then B leaves the data "transposed" (index k1 + R1 k2 stored at
// R2 k1 + k2); running B then A takes it back to natural order.  Every stage
// therefore works in place, and the order in between is only ever seen by
// code that knows the mapping (ymap below).
//
// Two real rows of a plane are packed into one complex line (a + i b) for
// the z transforms; the half spectra are separated / recombined with the
// Hermitian symmetry X[n-k] = conj X[k].  As in FFTW's c2r, the imaginary
// parts of the k=0 and k=n/2 coefficients are ignored on the way back.
#pragma once
#include "dft.cuh"

namespace lfts {

// Programmatic dependent launch: the chain's kernels are launched with
// programmatic stream serialisation, so a kernel's CTAs may start while the
// previous kernel drains.  Each kernel loads its constant tables first, then
// waits for the previous grid's results (griddepcontrol.wait) before touching
// the spectrum, h, q or w, and lets its dependent launch as soon as all of its
// own CTAs are running.  Launched without the attribute, both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" :::); }
// pull one 128-byte line into L2 (a hint: L2 is the point of coherence, so a
// line fetched before its last writer finished is still read current)
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

enum PlaneMode : int {
    PLANE_INIT_W = 0,  // h = exp(-w/N) from the fields, store h, forward transform
    PLANE_INIT_Q = 1,  // forward transform of given real rows (q_in or W-)
    PLANE_STEP = 2,    // inverse, x h, store q, forward
    PLANE_LAST = 3,    // inverse, x h, store q, partial sum of chain 0 (for Q)
    PLANE_G = 4,       // inverse, x g (separable tables), forward; stores nothing
};
constexpr int kPlaneModes = 5;

template <typename T>
struct PlaneArgs {
    const double *w;      // INIT_W: W- (M) and w+ (M), FP64
    const T *src;         // INIT_Q: source rows, chain c at src + c*src_stride
    long long src_stride;
    const double *src64;  // INIT_Q from FP64 rows (used when src == nullptr)
    T *qout;              // stored propagators, chain c at qout + c*M
    const T *h;           // [hA | hB]
    cpx<T> *spec;         // half spectra, chain c at spec + c*mx*my*KZ
    const cpx<T> *twy, *twz;  // exp(-2 pi i t/n) tables
    double *qpart;        // LAST: per-plane sums of chain 0
    int hsel0, hsel1;     // h half used by chain 0 / chain 1 (0 = hA, 1 = hB)
    int cbase;            // chain index of blockIdx.y == 0 (one-chain launches)
    int nchains;
    double Nd;            // N as a double (h = exp(-w/N))
    const T *gx, *gy, *gz;  // PLANE_G: separable Boltzmann weight, 1/M folded into gz
    const T *pf;          // PLANE_G: (chain 1, chain 2) slot that the next x-pencil reads, pulled into L2
    int pf_ctas;          // PLANE_G with pf: CTAs past the planes that pull pf into L2 (0: each plane CTA its plane)
};

template <typename T, int NY, int NZ>
struct PlaneCfg {
    static constexpr int KZ = NZ / 2 + 1;
    static constexpr int RY1 = Plan<NY>::R1, RY2 = Plan<NY>::R2;
    static constexpr int RZ1 = Plan<NZ>::R1, RZ2 = Plan<NZ>::R2;
    static constexpr int PAIRS = NY / 2;
    // Inside a row pair the packed z line is stored with one pad slot after
    // every RZ2 slots (zpos), so the contiguous-block stages hit distinct
    // shared-memory banks; the row pitch KZP leaves room for that.
    // KZP = 4 (mod 8): the row pairs a warp works on start on different
    // bank halves (FP32) / are bank-neutral (FP64).
    static constexpr int ZSPAN = NZ + (NZ - 1) / RZ2;
    static constexpr int KZP0 = KZ > (ZSPAN + 1) / 2 ? KZ : (ZSPAN + 1) / 2;
    static constexpr int KZP = (KZP0 + 3) / 8 * 8 + 4;
    // The kz = 0 and kz = NZ/2 columns are real along y in real space, so they
    // travel through the y transforms packed as one complex column (column 0:
    // x = kz 0, y = kz NZ/2); the y phases work on KC = NZ/2 columns.
    static constexpr int KC = NZ / 2;
    // one thread per stage-A task of the y and z transforms (the larger of
    // the two), so those phases take a single round; multiples of 4 warps
    // keep the SM sub-partitions balanced
    static constexpr int W0 = KC * RY2 > PAIRS * RZ2 ? KC * RY2 : PAIRS * RZ2;
    static constexpr int W1 = (W0 + 127) / 128 * 128;
    static constexpr int NT = W1 > 1024 ? 1024 : W1;
    // z twiddles as two padded 2-D tables so lanes that differ in j2 (stage
    // A) or k1 (stage B) hit different banks: TA[j2][k1] = TB[k1][j2] = w^(j2 k1)
    static constexpr int TAP = RZ1 + 1, TBP = RZ2 + 1;
    static constexpr int NTA = RZ2 * TAP, NTB = RZ1 * TBP;
    static constexpr size_t SMEM = sizeof(cpx<T>) * (size_t)(NY * KZP + 2 * NY + NTA + NTB);
    static __device__ __forceinline__ int ta(int j2, int k1) { return j2 * TAP + k1; }
    static __device__ __forceinline__ int tb(int k1, int u) { return k1 * TBP + u; }
    // resident CTAs per SM the register budget is sized for (FP32 planes are
    // small enough for two)
    static constexpr int MINB = (sizeof(T) == 4 && 2 * SMEM < 200 * 1024 && NT <= 512) ? 2 : 1;
    static_assert(NZ % 2 == 0 && NY % 2 == 0, "plane kernels need even my and mz");
    static __device__ __forceinline__ int ymap(int p) { return p / RY2 + RY1 * (p % RY2); }
    static __device__ __forceinline__ int zpos(int s) { return s + s / RZ2; }
};

template <int TASKS, int NT>
struct Tpt {
    static constexpr int v = (TASKS + NT - 1) / NT;
};

// The z-line phases are warp-local: warp w owns row pairs
// [first(w), first(w) + count(w)) for all of them, so only __syncwarp
// separates those phases and warps run through them independently.
template <typename C>
struct WarpPairs {
    static constexpr int NW = C::NT / 32;
    static constexpr int MAXP = (C::PAIRS + NW - 1) / NW;
    static __device__ __forceinline__ int first(int w) { return (w * C::PAIRS) / NW; }
    static __device__ __forceinline__ int count(int w) { return ((w + 1) * C::PAIRS) / NW - first(w); }
    // rounds a lane needs for TPQ tasks per pair
    template <int TPQ>
    struct Rounds {
        static constexpr int v = (MAXP * TPQ + 31) / 32;
    };
};

// ---------------------------------------------------------------- y phases --
// inverse, natural -> transposed, stage A reading the global half spectrum.
// KC * RY2 <= NT, so every thread has at most one task; the loads are issued
// by y_invA_load (before the barrier that publishes the twiddle tables) and
// consumed by y_invA_finish.
template <typename C, typename T>
__device__ __forceinline__ void y_invA_load(const cpx<T> *__restrict__ Sg, cpx<T> (&v)[C::RY1])
{
    constexpr int KZ = C::KZ, KC = C::KC, R1 = C::RY1, R2 = C::RY2;
    static_assert(KC * R2 <= C::NT, "one stage-A task per thread");
    const int t = threadIdx.x;
    if (t < KC * R2) {
        const int col = t % KC, j2 = t / KC;
#pragma unroll
        for (int a = 0; a < R1; a++) {
            v[a] = Sg[(j2 + R2 * a) * KZ + col];
            if (col == 0) {  // Y0 + i Y_{NZ/2}
                const cpx<T> n2 = Sg[(j2 + R2 * a) * KZ + KC];
                v[a] = {v[a].x - n2.y, v[a].y + n2.x};
            }
        }
    }
}

template <typename C, typename T>
__device__ __forceinline__ void y_invA_finish(cpx<T> *P, cpx<T> (&v)[C::RY1], const cpx<T> *twy)
{
    constexpr int KC = C::KC, KZP = C::KZP, R1 = C::RY1, R2 = C::RY2, NY = R1 * R2;
    const int t = threadIdx.x;
    if (t < KC * R2) {
        const int col = t % KC, j2 = t / KC;
        Dft<R1, 1, T>::run(v);
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++)
            P[(j2 + R2 * k1) * KZP + col] = ctw<1>(v[k1], twy[(j2 * k1) % NY]);
    }
}

// stage B in place with sign S; TW: apply exp(S 2pi i j2 k1/n) after the DFT
template <typename C, int S, bool TW, typename T>
__device__ __forceinline__ void y_B(cpx<T> *P, const cpx<T> *twy)
{
    constexpr int KC = C::KC, KZP = C::KZP, R1 = C::RY1, R2 = C::RY2, NY = R1 * R2;
    for (int t = threadIdx.x; t < KC * R1; t += C::NT) {
        const int col = t % KC, k1 = t / KC;
        cpx<T> v[R2];
#pragma unroll
        for (int u = 0; u < R2; u++) v[u] = P[(R2 * k1 + u) * KZP + col];
        Dft<R2, S, T>::run(v);
#pragma unroll
        for (int u = 0; u < R2; u++)
            P[(R2 * k1 + u) * KZP + col] = TW ? ctw<S>(v[u], twy[(u * k1) % NY]) : v[u];
    }
}

// forward, stage A in smem with twiddles (natural -> transposed start)
template <typename C, typename T>
__device__ __forceinline__ void y_fwdA_tw(cpx<T> *P, const cpx<T> *twy)
{
    constexpr int KC = C::KC, KZP = C::KZP, R1 = C::RY1, R2 = C::RY2, NY = R1 * R2;
    for (int t = threadIdx.x; t < KC * R2; t += C::NT) {
        const int col = t % KC, j2 = t / KC;
        cpx<T> v[R1];
#pragma unroll
        for (int a = 0; a < R1; a++) v[a] = P[(j2 + R2 * a) * KZP + col];
        Dft<R1, -1, T>::run(v);
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) P[(j2 + R2 * k1) * KZP + col] = ctw<-1>(v[k1], twy[(j2 * k1) % NY]);
    }
}

// forward stage B -> global, natural order (end of natural -> natural forward)
// (packed column 0 goes to colbuf for y_unpack0)
template <typename C, typename T>
__device__ __forceinline__ void y_fwdB_global(const cpx<T> *P, cpx<T> *__restrict__ Sg, cpx<T> *colbuf)
{
    constexpr int KZ = C::KZ, KC = C::KC, KZP = C::KZP, R1 = C::RY1, R2 = C::RY2;
    for (int t = threadIdx.x; t < KC * R1; t += C::NT) {
        const int col = t % KC, k1 = t / KC;
        cpx<T> v[R2];
#pragma unroll
        for (int u = 0; u < R2; u++) v[u] = P[(R2 * k1 + u) * KZP + col];
        Dft<R2, -1, T>::run(v);
#pragma unroll
        for (int k2 = 0; k2 < R2; k2++) {
            if (col == 0)
                colbuf[k1 + R1 * k2] = v[k2];
            else
                Sg[(k1 + R1 * k2) * KZ + col] = v[k2];
        }
    }
}

// forward stage A -> global, natural order (end of transposed -> natural forward)
template <typename C, typename T>
__device__ __forceinline__ void y_fwdA_global(const cpx<T> *P, cpx<T> *__restrict__ Sg, cpx<T> *colbuf)
{
    constexpr int KZ = C::KZ, KC = C::KC, KZP = C::KZP, R1 = C::RY1, R2 = C::RY2;
    for (int t = threadIdx.x; t < KC * R2; t += C::NT) {
        const int col = t % KC, j2 = t / KC;
        cpx<T> v[R1];
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) v[k1] = P[(j2 + R2 * k1) * KZP + col];
        Dft<R1, -1, T>::run(v);
#pragma unroll
        for (int j1 = 0; j1 < R1; j1++) {
            if (col == 0)
                colbuf[j2 + R2 * j1] = v[j1];
            else
                Sg[(j2 + R2 * j1) * KZ + col] = v[j1];
        }
    }
}

// Separate the packed column Y = Y0 + i Y_{NZ/2} (natural ky order in colbuf)
// into the kz = 0 and kz = NZ/2 columns of the global half spectrum.
template <typename C, typename T>
__device__ __forceinline__ void y_unpack0(const cpx<T> *colbuf, cpx<T> *__restrict__ Sg)
{
    constexpr int KZ = C::KZ, KC = C::KC, NY = C::RY1 * C::RY2;
    for (int k = threadIdx.x; k < NY; k += C::NT) {
        const cpx<T> z = colbuf[k], c = colbuf[(NY - k) % NY];
        Sg[k * KZ] = {(T)0.5 * (z.x + c.x), (T)0.5 * (z.y - c.y)};
        Sg[k * KZ + KC] = {(T)0.5 * (z.y + c.y), (T)-0.5 * (z.x - c.x)};
    }
}

// ---------------------------------------------------------------- z phases --
// Row pair q occupies the 2*KZP slots starting at P + 2q*KZP ("region");
// the packed line's slot s lives at region[zpos(s)], the rows' k at row[k].

// Build Z = A + iB (Hermitian-extended) and run inverse stage A.  Permuting
// inside each pair region: the warp reads everything before __syncwarp, then
// writes.
template <typename C, typename T>
__device__ __forceinline__ void z_build_invA(cpx<T> *P, const cpx<T> *twa)
{
    using WP = WarpPairs<C>;
    constexpr int KZP = C::KZP, R1 = C::RZ1, R2 = C::RZ2, NZ = R1 * R2;
    constexpr int RND = WP::template Rounds<R2>::v;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q0 = WP::first(w), ntask = WP::count(w) * R2;
    cpx<T> hold[RND][R1];
#pragma unroll
    for (int s = 0; s < RND; s++) {
        const int t = lane + 32 * s;
        if (t < ntask) {
            const int q = q0 + t / R2, j2 = t % R2;
            const cpx<T> *A = P + 2 * q * KZP, *B = A + KZP;
#pragma unroll
            for (int a = 0; a < R1; a++) {
                const int k = j2 + R2 * a;
                cpx<T> z;
                if (k == 0) {
                    z = {A[0].x, B[0].x};
                } else if (2 * k == NZ) {
                    z = {A[0].y, B[0].y};  // packed kz = NZ/2 (real part only, as c2r)
                } else if (2 * k < NZ) {
                    const cpx<T> av = A[k], bv = B[k];
                    z = {av.x - bv.y, av.y + bv.x};
                } else {
                    const cpx<T> av = A[NZ - k], bv = B[NZ - k];
                    z = {av.x + bv.y, bv.x - av.y};
                }
                hold[s][a] = z;
            }
            Dft<R1, 1, T>::run(hold[s]);
#pragma unroll
            for (int k1 = 0; k1 < R1; k1++) hold[s][k1] = ctw<1>(hold[s][k1], twa[C::ta(j2, k1)]);
        }
    }
    __syncwarp();
#pragma unroll
    for (int s = 0; s < RND; s++) {
        const int t = lane + 32 * s;
        if (t < ntask) {
            const int q = q0 + t / R2, j2 = t % R2;
            cpx<T> *Z = P + 2 * q * KZP;
#pragma unroll
            for (int k1 = 0; k1 < R1; k1++) Z[C::zpos(j2 + R2 * k1)] = hold[s][k1];
        }
    }
}

// Inverse stage B -> real rows (transposed z order), times h, store q;
// STEP: then forward stage B with twiddles back into smem.
// LAST: accumulate chain-0 values into *qsum instead.
// All of a lane's h values are loaded before its first task (they do not
// depend on shared memory), and q goes out with evict-first stores: it is
// read again only by the concentration pass.
template <typename C, int MODE, typename T>
__device__ __forceinline__ void z_invB_h(cpx<T> *P, const cpx<T> *twb, const T *__restrict__ h,
                                         T *__restrict__ qrow, double &qsum)
{
    using WP = WarpPairs<C>;
    constexpr int KZP = C::KZP, R1 = C::RZ1, R2 = C::RZ2, NZ = R1 * R2;
    constexpr int RND = WP::template Rounds<R1>::v;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q0 = WP::first(w), ntask = WP::count(w) * R1;
    T hv[RND][R2][2];
#pragma unroll
    for (int s = 0; s < RND; s++) {
        const int t = lane + 32 * s;
        if (t < ntask) {
            const int q = q0 + t / R1, k1 = t % R1;
            const int ya = C::ymap(2 * q), yb = C::ymap(2 * q + 1);
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) {
                hv[s][k2][0] = __ldg(h + ya * NZ + k1 + R1 * k2);
                hv[s][k2][1] = __ldg(h + yb * NZ + k1 + R1 * k2);
            }
        }
    }
#pragma unroll
    for (int s = 0; s < RND; s++) {
        const int t = lane + 32 * s;
        if (t >= ntask) continue;
        const int q = q0 + t / R1, k1 = t % R1;
        cpx<T> *Z = P + 2 * q * KZP;
        const int ya = C::ymap(2 * q), yb = C::ymap(2 * q + 1);
        cpx<T> v[R2];
#pragma unroll
        for (int u = 0; u < R2; u++) v[u] = Z[C::zpos(R2 * k1 + u)];
        Dft<R2, 1, T>::run(v);
#pragma unroll
        for (int k2 = 0; k2 < R2; k2++) {
            const int z = k1 + R1 * k2;
            const T a = v[k2].x * hv[s][k2][0];
            const T b = v[k2].y * hv[s][k2][1];
            __stcs(qrow + ya * NZ + z, a);
            __stcs(qrow + yb * NZ + z, b);
            if (MODE == PLANE_LAST) qsum += (double)a + (double)b;
            v[k2] = {a, b};
        }
        if (MODE == PLANE_STEP) {
            Dft<R2, -1, T>::run(v);
#pragma unroll
            for (int u = 0; u < R2; u++) Z[C::zpos(R2 * k1 + u)] = ctw<-1>(v[u], twb[C::tb(k1, u)]);
        }
    }
}

// forward stage A, transposed -> natural, in place
template <typename C, typename T>
__device__ __forceinline__ void z_fwdA(cpx<T> *P)
{
    using WP = WarpPairs<C>;
    constexpr int KZP = C::KZP, R1 = C::RZ1, R2 = C::RZ2;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q0 = WP::first(w), ntask = WP::count(w) * R2;
    for (int t = lane; t < ntask; t += 32) {
        const int q = q0 + t / R2, j2 = t % R2;
        cpx<T> *Z = P + 2 * q * KZP;
        cpx<T> v[R1];
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) v[k1] = Z[C::zpos(j2 + R2 * k1)];
        Dft<R1, -1, T>::run(v);
#pragma unroll
        for (int j1 = 0; j1 < R1; j1++) Z[C::zpos(j2 + R2 * j1)] = v[j1];
    }
}

// forward stage A with twiddles, natural -> (start of) transposed, in place
template <typename C, typename T>
__device__ __forceinline__ void z_fwdA_tw(cpx<T> *P, const cpx<T> *twa)
{
    using WP = WarpPairs<C>;
    constexpr int KZP = C::KZP, R1 = C::RZ1, R2 = C::RZ2, NZ = R1 * R2;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q0 = WP::first(w), ntask = WP::count(w) * R2;
    for (int t = lane; t < ntask; t += 32) {
        const int q = q0 + t / R2, j2 = t % R2;
        cpx<T> *Z = P + 2 * q * KZP;
        cpx<T> v[R1];
#pragma unroll
        for (int a = 0; a < R1; a++) v[a] = Z[C::zpos(j2 + R2 * a)];
        Dft<R1, -1, T>::run(v);
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) Z[C::zpos(j2 + R2 * k1)] = ctw<-1>(v[k1], twa[C::ta(j2, k1)]);
    }
}

// forward stage B without twiddles, in place (ends natural -> transposed)
template <typename C, typename T>
__device__ __forceinline__ void z_fwdB(cpx<T> *P)
{
    using WP = WarpPairs<C>;
    constexpr int KZP = C::KZP, R1 = C::RZ1, R2 = C::RZ2;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q0 = WP::first(w), ntask = WP::count(w) * R1;
    for (int t = lane; t < ntask; t += 32) {
        const int q = q0 + t / R1, k1 = t % R1;
        cpx<T> *Z = P + 2 * q * KZP;
        cpx<T> v[R2];
#pragma unroll
        for (int u = 0; u < R2; u++) v[u] = Z[C::zpos(R2 * k1 + u)];
        Dft<R2, -1, T>::run(v);
#pragma unroll
        for (int u = 0; u < R2; u++) Z[C::zpos(R2 * k1 + u)] = v[u];
    }
}

// Separate the packed spectrum Z of rows (a, b) into the half spectra A, B.
// TRANSPOSED: Z[k] sits at R2*(k % R1) + k / R1, else at k.  Permuting.
template <typename C, bool TRANSPOSED, typename T>
__device__ __forceinline__ void z_unpack(cpx<T> *P)
{
    using WP = WarpPairs<C>;
    constexpr int KC = C::KC, KZP = C::KZP, R1 = C::RZ1, R2 = C::RZ2, NZ = R1 * R2;
    constexpr int TPT = WP::template Rounds<KC>::v;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q0 = WP::first(w), ntask = WP::count(w) * KC;
    cpx<T> ha[TPT], hb[TPT];
#pragma unroll
    for (int s = 0; s < TPT; s++) {
        const int t = lane + 32 * s;
        if (t < ntask) {
            const int q = q0 + t / KC, k = t % KC;
            const int nk = (k == 0) ? NZ / 2 : NZ - k;  // k = 0 pairs DC with Nyquist
            const cpx<T> *Z = P + 2 * q * KZP;
            const int pk = TRANSPOSED ? R2 * (k % R1) + k / R1 : k;
            const int pn = TRANSPOSED ? R2 * (nk % R1) + nk / R1 : nk;
            const cpx<T> z = Z[C::zpos(pk)], c = Z[C::zpos(pn)];
            if (k == 0) {
                // A[0], A[NZ/2], B[0], B[NZ/2] are real: A = Re Z, B = Im Z
                ha[s] = {z.x, c.x};
                hb[s] = {z.y, c.y};
            } else {
                // A = (z + conj c)/2, B = (z - conj c)/(2i)
                ha[s] = {(T)0.5 * (z.x + c.x), (T)0.5 * (z.y - c.y)};
                hb[s] = {(T)0.5 * (z.y + c.y), (T)-0.5 * (z.x - c.x)};
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int s = 0; s < TPT; s++) {
        const int t = lane + 32 * s;
        if (t < ntask) {
            const int q = q0 + t / KC, k = t % KC;
            P[2 * q * KZP + k] = ha[s];
            P[(2 * q + 1) * KZP + k] = hb[s];
        }
    }
}

template <typename C, typename T>
__device__ __forceinline__ void load_tw(cpx<T> *dst, const cpx<T> *__restrict__ src, int n)
{
    for (int t = threadIdx.x; t < n; t += C::NT) dst[t] = src[t];
}

// Both twiddle tables through registers: the global loads go out first (before
// the wait on the previous kernel), the shared stores later.
template <typename C, typename T>
struct TwStage {
    static constexpr int NY = C::RY1 * C::RY2, NZ = C::RZ1 * C::RZ2;
    static constexpr int TOT = NY + C::NTA + C::NTB;
    static constexpr int PER = (TOT + C::NT - 1) / C::NT;
    cpx<T> r[PER];
    // global index of table entry t (twy, then TA, then TB; pads read entry 0)
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
    // twy[NY] is followed by TA and TB in shared memory
    __device__ __forceinline__ void store(cpx<T> *twy)
    {
#pragma unroll
        for (int s = 0; s < PER; s++) {
            const int t = threadIdx.x + s * C::NT;
            if (t < TOT) twy[t] = r[s];
        }
    }
};

// Pull this warp's h rows (used by z_invB_h) towards L1 while the z section
// starts: one prefetch per 128-byte line.
template <typename C, typename T>
__device__ __forceinline__ void prefetch_h_rows(const T *__restrict__ h)
{
    using WP = WarpPairs<C>;
    constexpr int NZ = C::RZ1 * C::RZ2;
    constexpr int LINES_PER_ROW = (NZ * (int)sizeof(T) + 127) / 128;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q0 = WP::first(w), nrows = 2 * WP::count(w);
    for (int t = lane; t < nrows * LINES_PER_ROW; t += 32) {
        const int row = t / LINES_PER_ROW, line = t % LINES_PER_ROW;
        const int p = 2 * q0 + row;
        const char *addr = reinterpret_cast<const char *>(h + C::ymap(p) * NZ) + 128 * line;
        asm volatile("prefetch.global.L1 [%0];" ::"l"(addr));
    }
}

// ------------------------------------------------------------ plane kernel --
template <typename T, int NY, int NZ, int MODE>
__global__ void __launch_bounds__(PlaneCfg<T, NY, NZ>::NT, PlaneCfg<T, NY, NZ>::MINB) plane_kernel(PlaneArgs<T> a)
{
    using C = PlaneCfg<T, NY, NZ>;
    constexpr int KZ = C::KZ, KZP = C::KZP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T> *P = reinterpret_cast<cpx<T> *>(smem_raw);
    cpx<T> *twy = P + NY * KZP;
    cpx<T> *twa = twy + NY;            // TA: stage-A z twiddles
    cpx<T> *twb = twa + C::NTA;        // TB: stage-B z twiddles
    cpx<T> *colbuf = twb + C::NTB;

    const int x = blockIdx.x, c = blockIdx.y + a.cbase;
    const int mx = gridDim.x;
    const long long M = (long long)mx * NY * NZ;
    const long long plane_off = (long long)x * NY * NZ;
    cpx<T> *Sg = a.spec + ((long long)c * mx + x) * NY * KZ;

    TwStage<C, T> tws;
    tws.load(a.twy, a.twz);
    pdl_launch_dependents();
    pdl_wait();

    if (MODE == PLANE_INIT_W || MODE == PLANE_INIT_Q) {
        // real rows (natural y order), packed two per complex line; the whole
        // z section is warp-local (see WarpPairs)
        tws.store(twy);
        __syncthreads();  // twiddle tables
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int q0 = WarpPairs<C>::first(w), ntask = WarpPairs<C>::count(w) * NZ;
        for (int t = lane; t < ntask; t += 32) {
            const int q = q0 + t / NZ, z = t % NZ;
            const long long ia = plane_off + (2 * q) * NZ + z, ib = ia + NZ;
            T va, vb;
            if (MODE == PLANE_INIT_W) {
                // hA = exp(-(W- + w+)/N), hB = exp(-(-W- + w+)/N)  (src/diblock.cc:64-72)
                const double sgn = c == 0 ? 1.0 : -1.0;
                const double da = exp(-(sgn * a.w[ia] + a.w[M + ia]) / a.Nd);
                const double db = exp(-(sgn * a.w[ib] + a.w[M + ib]) / a.Nd);
                va = (T)da;
                vb = (T)db;
                a.qout[c * M + ia] = va;
                a.qout[c * M + ib] = vb;
            } else if (a.src) {
                va = a.src[c * a.src_stride + ia];
                vb = a.src[c * a.src_stride + ib];
            } else {
                va = (T)a.src64[c * a.src_stride + ia];
                vb = (T)a.src64[c * a.src_stride + ib];
            }
            P[2 * q * KZP + C::zpos(z)] = {va, vb};
        }
        __syncwarp();
        z_fwdA_tw<C>(P, twa);
        __syncwarp();
        z_fwdB<C>(P);
        __syncwarp();
        z_unpack<C, true>(P);
        __syncthreads();
        y_fwdA_tw<C>(P, twy);
        __syncthreads();
        y_fwdB_global<C>(P, Sg, colbuf);
        __syncthreads();
        y_unpack0<C>(colbuf, Sg);
        return;
    }

    // inverse y (natural -> transposed rows), then packed z lines
    {
        cpx<T> v[C::RY1];
        y_invA_load<C>(Sg, v);
        tws.store(twy);
        __syncthreads();
        y_invA_finish<C>(P, v, twy);
    }
    __syncthreads();
    y_B<C, 1, false>(P, twy);
    __syncthreads();
    const T *h = a.h + (long long)(c == 0 ? a.hsel0 : a.hsel1) * M + plane_off;
    z_build_invA<C>(P, twa);
    __syncwarp();
    T *qrow = a.qout + c * M + plane_off;
    double qsum = 0.0;
    z_invB_h<C, MODE>(P, twb, h, qrow, qsum);
    if (MODE == PLANE_LAST) {
        if (c == 0) {
            // deterministic block reduction of the plane sum
            __shared__ double red[C::NT / 32];
            for (int o = 16; o > 0; o >>= 1) qsum += __shfl_xor_sync(0xffffffffu, qsum, o);
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = qsum;
            __syncthreads();
            if (threadIdx.x == 0) {
                double s = 0.0;
                for (int i = 0; i < C::NT / 32; i++) s += red[i];
                a.qpart[x] = s;
            }
        }
        return;
    }
    __syncwarp();
    z_fwdA<C>(P);
    __syncwarp();
    z_unpack<C, false>(P);
    __syncthreads();
    y_B<C, -1, true>(P, twy);
    __syncthreads();
    y_fwdA_global<C>(P, Sg, colbuf);
    __syncthreads();
    y_unpack0<C>(colbuf, Sg);
}

// ----------------------------------------------------------- pencil kernel --
enum PencilMode : int {
    PENCIL_CONV = 0,    // forward x, times g, inverse x (in place in the spectrum)
    PENCIL_POWER = 1,   // forward x, S += |X|^2 (structure function sample)
    // the h-in-pencil chain (FP32 packed field): see enqueue_chain_launches
    PENCIL_H = 2,       // forward x, times h, store q, inverse x
    PENCIL_H_LAST = 3,  // forward x, times h, store q
    PENCIL_INIT_W = 4,  // h = exp(-w/N) from the fields, store it, inverse x
    // the same with the concentration sums accumulated in the chain (second
    // half of the chain: the new slot's partner slot is already stored)
    PENCIL_HA = 5,       // forward x, times h, add the two phi products, inverse x (q not stored)
    PENCIL_HA_LAST = 6,  // forward x, times h, store q_N (for Q), add the two phi products
};
constexpr int kPencilModes = 7;

template <typename T>
struct PencilArgs {
    cpx<T> *spec;             // chain c at spec + c*mx*ncol
    const cpx<T> *twx;        // exp(-2 pi i t/mx)
    const T *gx, *gy, *gz;    // separable Boltzmann weight, 1/M folded into gz
    double *S;                // POWER: accumulator (mx*ncol)
    int ncol;                 // my*KZ
    int KZ;
    int cbase;                // chain index of blockIdx.y == 0
    // PENCIL_H, PENCIL_H_LAST, PENCIL_INIT_W (packed field: (chain 1, chain 2) pairs)
    const double *w;          // INIT_W: W- (M) and w+ (M), FP64
    const T *h;               // (hA, hB) pairs
    T *qout;                  // stored propagators (pairs), or h for INIT_W
    int hsel0, hsel1;         // h half used by chain 1 / chain 2 (0 = hA, 1 = hB)
    long long M;
    double Nd;                // N as a double (h = exp(-w/N))
    // PENCIL_HA, PENCIL_HA_LAST: the new slot i+1 = (q_{i+1}, q^_{N-i}) and its
    // partner slot N-i = (q_{N-i}, q^_{i+1}) give q_{i+1} q^_{i+1} and
    // q_{N-i} q^_{N-i}, added into acc = (sum over A monomers, sum over B)
    const T *partner;         // partner slot pairs (null: the slot pairs with itself, odd N)
    T *acc;                   // (A, B) sums per mesh point
    int acc_init;             // first accumulating step: acc starts at zero
    int a_is_A, b_is_A;       // monomer i+1 / N-i is an A monomer (index <= NA)
};

template <typename T, int NX, int CW>
struct PencilCfg {
    static constexpr int R1 = Plan<NX>::R1, R2 = Plan<NX>::R2;
    static constexpr int W0 = CW * (R1 > R2 ? R1 : R2);
    static constexpr int NT = W0 >= 512 ? 256 : (W0 <= 128 ? 128 : 256);
    static constexpr size_t SMEM = sizeof(cpx<T>) * (size_t)(NX * CW + NX) + sizeof(T) * NX;
    // FP32 tiles 8 columns wide are 64-byte rows, two to a 128-byte bank
    // window: stage B's half-warps read rows R2 apart (same window half), so
    // the low bit of the row index flips on alternate stage-B groups.  Stage
    // A's row pairs {2m, 2m+1} stay together.
    static constexpr bool SWZ = sizeof(T) == 4 && CW == 8 && R2 % 2 == 0;
    static __device__ __forceinline__ int row(int r) { return SWZ ? (r ^ ((r / R2) & 1)) : r; }
};

// body of one CTA: column tile `tile` of chain `chain` (the ensemble's
// batched launches call it with their own tile numbering)
template <typename T, int NX, int CW, int MODE>
__device__ __forceinline__ void pencil_body(const PencilArgs<T> &a, const int tile, const int chain)
{
    using C = PencilCfg<T, NX, CW>;
    constexpr int R1 = C::R1, R2 = C::R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T> *Tl = reinterpret_cast<cpx<T> *>(smem_raw);
    cpx<T> *twx = Tl + NX * CW;
    T *gxs = reinterpret_cast<T *>(twx + NX);

    const int col0 = tile * CW, c = chain + a.cbase;
    const int ncol = a.ncol;
    cpx<T> *Sg = a.spec + (long long)c * NX * ncol;
    for (int t = threadIdx.x; t < NX; t += C::NT) {
        twx[t] = a.twx[t];
        if (MODE == PENCIL_CONV) gxs[t] = a.gx[t];  // POWER mode has no g table
    }
    pdl_launch_dependents();
    pdl_wait();

    // X1: forward stage A from global (strided rows), twiddles, to smem.  At
    // most one task per thread (CW * R2 <= NT); its loads go out before the
    // barrier that publishes the tables.
    static_assert(CW * R2 <= C::NT, "one stage-A task per thread");
    if (MODE != PENCIL_INIT_W) {
        const int t = threadIdx.x;
        const int cl = t % CW, j2 = t / CW, col = col0 + cl;
        const bool act = t < CW * R2 && col < ncol;
        cpx<T> v[R1];
        if (act) {
#pragma unroll
            for (int s = 0; s < R1; s++) v[s] = Sg[(long long)(j2 + R2 * s) * ncol + col];
        }
        __syncthreads();
        if (act) {
            Dft<R1, -1, T>::run(v);
#pragma unroll
            for (int k1 = 0; k1 < R1; k1++) Tl[C::row(j2 + R2 * k1) * CW + cl] = ctw<-1>(v[k1], twx[(j2 * k1) % NX]);
        }
    }
    __syncthreads();

    // X2: forward stage B -> X[k1 + R1 k2]; then g and inverse stage B, or |X|^2.
    // The h modes see the forward transform of their input at real-space x =
    // k1 + R1 k2 (the chain that uses them is written out at
    // enqueue_chain_launches); INIT_W starts from h at those points.
    for (int t = threadIdx.x; t < CW * R1; t += C::NT) {
        const int cl = t % CW, k1 = t / CW, col = col0 + cl;
        if (col >= ncol) continue;
        cpx<T> v[R2];
        // PENCIL_HA*: the partner slot (HBM) and the running sums (L2) of this
        // task's points go out before its shared-memory reads and transform, so
        // their latency overlaps that work instead of each point's update
        constexpr bool kAcc = MODE == PENCIL_HA || MODE == PENCIL_HA_LAST;
        float2 pv[kAcc ? R2 : 1], av[kAcc ? R2 : 1];
        if constexpr (kAcc) {
            const float2 *__restrict__ pp = reinterpret_cast<const float2 *>(a.partner);
            const float2 *__restrict__ ap = reinterpret_cast<const float2 *>(a.acc);
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) {
                const long long o = (long long)(k1 + R1 * k2) * ncol + col;
                pv[k2] = pp ? __ldcs(pp + o) : make_float2(0.f, 0.f);
                av[k2] = a.acc_init ? make_float2(0.f, 0.f) : ap[o];
            }
        }
        if constexpr (MODE == PENCIL_INIT_W) {
            // hA = exp(-(W- + w+)/N), hB = exp(-(-W- + w+)/N)  (src/diblock.cc:64-72),
            // single-precision exponential as the FP32 plane kernels' INIT_W
            static_assert(sizeof(T) == sizeof(float), "FP32 packed field only");
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) {
                const long long o = (long long)(k1 + R1 * k2) * ncol + col;
                const double wm = a.w[o], wp = a.w[a.M + o];
                const float v1 = expf((float)(-(wm + wp) / a.Nd));
                const float v2 = expf((float)(-(-wm + wp) / a.Nd));
                reinterpret_cast<cpx<float> *>(a.qout)[o] = {v1, v2};
                v[k2] = {v1, v2};
            }
        } else {
#pragma unroll
            for (int u = 0; u < R2; u++) v[u] = Tl[C::row(R2 * k1 + u) * CW + cl];
            Dft<R2, -1, T>::run(v);
        }
        if constexpr (MODE == PENCIL_H || MODE == PENCIL_H_LAST) {
            static_assert(sizeof(T) == sizeof(float), "FP32 packed field only");
            const int hs0 = a.hsel0, hs1 = a.hsel1;
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) {
                const long long o = (long long)(k1 + R1 * k2) * ncol + col;
                const float2 h = __ldg(reinterpret_cast<const float2 *>(a.h) + o);
                const float va = v[k2].x * (hs0 ? h.y : h.x);
                const float vb = v[k2].y * (hs1 ? h.y : h.x);
                __stcs(reinterpret_cast<float2 *>(a.qout) + o, make_float2(va, vb));
                v[k2] = {va, vb};
            }
        }
        if constexpr (MODE == PENCIL_HA || MODE == PENCIL_HA_LAST) {
            static_assert(sizeof(T) == sizeof(float), "FP32 packed field only");
            const int hs0 = a.hsel0, hs1 = a.hsel1;
            float2 *accp = reinterpret_cast<float2 *>(a.acc);
            const bool has_partner = a.partner != nullptr;
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) {
                const long long o = (long long)(k1 + R1 * k2) * ncol + col;
                const float2 h = __ldg(reinterpret_cast<const float2 *>(a.h) + o);
                const float va = v[k2].x * (hs0 ? h.y : h.x);
                const float vb = v[k2].y * (hs1 ? h.y : h.x);
                if (MODE == PENCIL_HA_LAST) __stcs(reinterpret_cast<float2 *>(a.qout) + o, make_float2(va, vb));
                v[k2] = {va, vb};
                // q_{i+1} q^_{i+1} = va * partner.y and q_{N-i} q^_{N-i} = partner.x * vb;
                // with no partner (the middle slot of an odd chain) the slot
                // is (q_m, q^_m) and gives the one product va * vb
                float pa, pb = 0.f;
                if (has_partner) {
                    pa = va * pv[k2].y;
                    pb = pv[k2].x * vb;
                } else {
                    pa = va * vb;
                }
                float2 s = av[k2];
                if (a.a_is_A)
                    s.x += pa;
                else
                    s.y += pa;
                if (a.b_is_A)
                    s.x += pb;
                else
                    s.y += pb;
                accp[o] = s;
            }
        }
        if constexpr (MODE == PENCIL_H || MODE == PENCIL_INIT_W || MODE == PENCIL_HA) {
            Dft<R2, 1, T>::run(v);
#pragma unroll
            for (int u = 0; u < R2; u++) Tl[C::row(R2 * k1 + u) * CW + cl] = ctw<1>(v[u], twx[(u * k1) % NX]);
        }
        if (MODE == PENCIL_CONV) {
            const T gyz = a.gy[col / a.KZ] * a.gz[col % a.KZ];
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) v[k2] = cscale(v[k2], gxs[k1 + R1 * k2] * gyz);
            Dft<R2, 1, T>::run(v);
#pragma unroll
            for (int u = 0; u < R2; u++) Tl[C::row(R2 * k1 + u) * CW + cl] = ctw<1>(v[u], twx[(u * k1) % NX]);
        } else if (MODE == PENCIL_POWER) {
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) {
                const long long o = (long long)(k1 + R1 * k2) * ncol + col;
                a.S[o] += (double)v[k2].x * (double)v[k2].x + (double)v[k2].y * (double)v[k2].y;
            }
        }
    }
    if (MODE == PENCIL_POWER || MODE == PENCIL_H_LAST || MODE == PENCIL_HA_LAST) return;
    __syncthreads();

    // X3: inverse stage A (strided) -> natural order, to global
    for (int t = threadIdx.x; t < CW * R2; t += C::NT) {
        const int cl = t % CW, j2 = t / CW, col = col0 + cl;
        if (col >= ncol) continue;
        cpx<T> v[R1];
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) v[k1] = Tl[C::row(j2 + R2 * k1) * CW + cl];
        Dft<R1, 1, T>::run(v);
#pragma unroll
        for (int j1 = 0; j1 < R1; j1++) Sg[(long long)(j2 + R2 * j1) * ncol + col] = v[j1];
    }
}

template <typename T, int NX, int CW, int MODE>
__global__ void __launch_bounds__(PencilCfg<T, NX, CW>::NT) pencil_kernel(PencilArgs<T> a)
{
    pencil_body<T, NX, CW, MODE>(a, blockIdx.x, blockIdx.y);
}

}  // namespace lfts
