// Complex arithmetic and in-register small DFTs for the sm_100a FFT kernels.
//
// Convention (the one FFTW documents and the reference relies on at
// src/step.cc:41,50): forward X[k] = sum_j x[j] exp(-2 pi i jk/n), backward
// with +i, both unnormalised.  S = -1 selects forward, S = +1 backward.
//
// Radices 2, 3, 4, 5 are written out; 6, 8, 10, 12, 16, 32 are two-level
// Cooley-Tukey compositions of those with compile-time twiddles.  All
// constants are exact values of cos/sin at multiples of 0.75 degrees
// (the finest angle any supported radix needs), given to 20 digits.
#pragma once
#include <cuda_runtime.h>

namespace lfts {

template <typename T>
struct alignas(2 * sizeof(T)) cpx {
    T x, y;
};

template <typename T>
__device__ __forceinline__ cpx<T> cadd(cpx<T> a, cpx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T>
__device__ __forceinline__ cpx<T> csub(cpx<T> a, cpx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T>
__device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b)
{
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <typename T>
__device__ __forceinline__ cpx<T> cmulc(cpx<T> a, cpx<T> b)
{
    return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename T>
__device__ __forceinline__ cpx<T> cscale(cpx<T> a, T s) { return {a.x * s, a.y * s}; }
// a * s + c for a real scalar s
template <typename T>
__device__ __forceinline__ cpx<T> cfma(cpx<T> a, T s, cpx<T> c) { return {a.x * s + c.x, a.y * s + c.y}; }

// FP32 complex add/sub/scale/fma go through Blackwell's packed f32x2 pipe:
// one instruction per complex value instead of two (rounding is the same as
// the scalar operations'; fma is fused as the scalar path's contraction is).
__device__ __forceinline__ unsigned long long pk2(cpx<float> a)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1,%2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ cpx<float> upk2(unsigned long long r)
{
    cpx<float> a;
    asm("mov.b64 {%0,%1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
template <>
__device__ __forceinline__ cpx<float> cadd<float>(cpx<float> a, cpx<float> b)
{
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
    return upk2(r);
}
template <>
__device__ __forceinline__ cpx<float> csub<float>(cpx<float> a, cpx<float> b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
    return upk2(r);
}
template <>
__device__ __forceinline__ cpx<float> cscale<float>(cpx<float> a, float s)
{
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2({s, s})));
    return upk2(r);
}
template <>
__device__ __forceinline__ cpx<float> cfma<float>(cpx<float> a, float s, cpx<float> c)
{
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk2(a)), "l"(pk2({s, s})), "l"(pk2(c)));
    return upk2(r);
}

// a * (S i)
template <int S, typename T>
__device__ __forceinline__ cpx<T> cmul_i(cpx<T> a)
{
    return S > 0 ? cpx<T>{-a.y, a.x} : cpx<T>{a.y, -a.x};
}
// a times the table twiddle tw = exp(-2 pi i t/n) (forward) or its conjugate (backward)
template <int S, typename T>
__device__ __forceinline__ cpx<T> ctw(cpx<T> a, cpx<T> tw)
{
    return S < 0 ? cmul(a, tw) : cmulc(a, tw);
}

// cos and sin of 2 pi e / R for R dividing 480 (0.75-degree units).
__host__ __device__ constexpr double root_cos_sin(int e, int R, bool want_sin)
{
    int t = ((e % R + R) % R) * (480 / R);
    int q = t / 120, rem = t % 120;
    double c = 1.0, s = 0.0;
    switch (rem) {
        case 0: c = 1.0; s = 0.0; break;
        case 15: c = 0.98078528040323044913; s = 0.19509032201612826785; break;   // 11.25
        case 24: c = 0.95105651629515357212; s = 0.30901699437494742410; break;   // 18
        case 30: c = 0.92387953251128675613; s = 0.38268343236508977173; break;   // 22.5
        case 40: c = 0.86602540378443864676; s = 0.5; break;                      // 30
        case 45: c = 0.83146961230254523708; s = 0.55557023301960222474; break;   // 33.75
        case 48: c = 0.80901699437494742410; s = 0.58778525229247312917; break;   // 36
        case 60: c = 0.70710678118654752440; s = 0.70710678118654752440; break;   // 45
        case 72: c = 0.58778525229247312917; s = 0.80901699437494742410; break;   // 54
        case 75: c = 0.55557023301960222474; s = 0.83146961230254523708; break;   // 56.25
        case 80: c = 0.5; s = 0.86602540378443864676; break;                      // 60
        case 90: c = 0.38268343236508977173; s = 0.92387953251128675613; break;   // 67.5
        case 96: c = 0.30901699437494742410; s = 0.95105651629515357212; break;   // 72
        case 105: c = 0.19509032201612826785; s = 0.98078528040323044913; break;  // 78.75
        default: c = 0.0; s = 0.0; break;  // unreachable for supported radices
    }
    double cq = q == 0 ? c : q == 1 ? -s : q == 2 ? -c : s;
    double sq = q == 0 ? s : q == 1 ? c : q == 2 ? -s : -c;
    return want_sin ? sq : cq;
}

// a * exp(S 2 pi i e / R), e and R compile-time after unrolling
template <int S, int R, typename T>
__device__ __forceinline__ cpx<T> croot(cpx<T> a, int e)
{
    const int t = ((e % R) + R) % R;
    if (t == 0) return a;
    if (4 * t == R) return cmul_i<S>(a);
    if (2 * t == R) return {-a.x, -a.y};
    if (4 * t == 3 * R) return cmul_i<-S>(a);
    const T c = (T)root_cos_sin(t, R, false);
    const T s = (T)(S * root_cos_sin(t, R, true));
    return {a.x * c - a.y * s, a.x * s + a.y * c};
}

template <int R>
struct Split;  // R = A * B used by the composite DFT
template <> struct Split<6> { static constexpr int A = 3, B = 2; };
template <> struct Split<8> { static constexpr int A = 4, B = 2; };
template <> struct Split<10> { static constexpr int A = 5, B = 2; };
template <> struct Split<12> { static constexpr int A = 4, B = 3; };
template <> struct Split<16> { static constexpr int A = 4, B = 4; };
template <> struct Split<32> { static constexpr int A = 8, B = 4; };

template <int R, int S, typename T>
struct Dft {
    // X[ka + A kb] = sum_jb w_B^{jb kb} w_R^{jb ka} sum_ja x[jb + B ja] w_A^{ja ka}
    static __device__ __forceinline__ void run(cpx<T> *v)
    {
        constexpr int A = Split<R>::A, B = Split<R>::B;
        cpx<T> y[R];
#pragma unroll
        for (int jb = 0; jb < B; jb++) {
            cpx<T> t[A];
#pragma unroll
            for (int ja = 0; ja < A; ja++) t[ja] = v[jb + B * ja];
            Dft<A, S, T>::run(t);
#pragma unroll
            for (int ka = 0; ka < A; ka++) y[jb * A + ka] = croot<S, R>(t[ka], jb * ka);
        }
#pragma unroll
        for (int ka = 0; ka < A; ka++) {
            cpx<T> u[B];
#pragma unroll
            for (int jb = 0; jb < B; jb++) u[jb] = y[jb * A + ka];
            Dft<B, S, T>::run(u);
#pragma unroll
            for (int kb = 0; kb < B; kb++) v[ka + A * kb] = u[kb];
        }
    }
};

template <int S, typename T>
struct Dft<1, S, T> {
    static __device__ __forceinline__ void run(cpx<T> *) {}
};

template <int S, typename T>
struct Dft<2, S, T> {
    static __device__ __forceinline__ void run(cpx<T> *v)
    {
        cpx<T> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <int S, typename T>
struct Dft<3, S, T> {
    static __device__ __forceinline__ void run(cpx<T> *v)
    {
        const T h = (T)0.86602540378443864676;  // sin(2 pi / 3)
        cpx<T> s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        cpx<T> m = cfma(s, (T)-0.5, v[0]);
        cpx<T> r = cmul_i<S>(cscale(d, h));
        v[0] = cadd(v[0], s);
        v[1] = cadd(m, r);
        v[2] = csub(m, r);
    }
};

template <int S, typename T>
struct Dft<4, S, T> {
    static __device__ __forceinline__ void run(cpx<T> *v)
    {
        cpx<T> a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        cpx<T> b0 = cadd(v[1], v[3]), b1 = cmul_i<S>(csub(v[1], v[3]));
        v[0] = cadd(a0, b0);
        v[2] = csub(a0, b0);
        v[1] = cadd(a1, b1);
        v[3] = csub(a1, b1);
    }
};

template <int S, typename T>
struct Dft<5, S, T> {
    static __device__ __forceinline__ void run(cpx<T> *v)
    {
        const T c1 = (T)0.30901699437494742410;   // cos(2 pi/5)
        const T c2 = (T)-0.80901699437494742410;  // cos(4 pi/5)
        const T s1 = (T)0.95105651629515357212;   // sin(2 pi/5)
        const T s2 = (T)0.58778525229247312917;   // sin(4 pi/5)
        cpx<T> b1 = cadd(v[1], v[4]), b2 = cadd(v[2], v[3]);
        cpx<T> d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
        cpx<T> x0 = v[0];
        cpx<T> p1 = cfma(b2, c2, cfma(b1, c1, x0));
        cpx<T> p2 = cfma(b2, c1, cfma(b1, c2, x0));
        cpx<T> q1 = cmul_i<S>(cfma(d2, s2, cscale(d1, s1)));
        cpx<T> q2 = cmul_i<S>(cfma(d2, -s1, cscale(d1, s2)));
        v[0] = cadd(x0, cadd(b1, b2));
        v[1] = cadd(p1, q1);
        v[4] = csub(p1, q1);
        v[2] = cadd(p2, q2);
        v[3] = csub(p2, q2);
    }
};

// Two-stage plan of a supported line length n = R1 * R2.
template <int N>
struct Plan;
template <> struct Plan<8> { static constexpr int R1 = 4, R2 = 2; };
template <> struct Plan<12> { static constexpr int R1 = 4, R2 = 3; };
template <> struct Plan<16> { static constexpr int R1 = 4, R2 = 4; };
template <> struct Plan<20> { static constexpr int R1 = 5, R2 = 4; };
template <> struct Plan<24> { static constexpr int R1 = 8, R2 = 3; };
template <> struct Plan<32> { static constexpr int R1 = 8, R2 = 4; };
template <> struct Plan<40> { static constexpr int R1 = 8, R2 = 5; };
template <> struct Plan<48> { static constexpr int R1 = 8, R2 = 6; };
template <> struct Plan<64> { static constexpr int R1 = 8, R2 = 8; };
template <> struct Plan<80> { static constexpr int R1 = 16, R2 = 5; };
template <> struct Plan<96> { static constexpr int R1 = 12, R2 = 8; };
template <> struct Plan<128> { static constexpr int R1 = 16, R2 = 8; };

}  // namespace lfts
