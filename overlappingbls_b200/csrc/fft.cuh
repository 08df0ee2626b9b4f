// fft.cuh -- complex arithmetic helpers and the in-register DFT codelets (radix 2, 3,
// 4, 5 and the composites 6, 8, 9, 10, 12, 16) used by the Stockham passes of fft2.cuh.
//
// Convention (FFTW's, which the reference relies on, SBL/code/002_fft.f90:97-113):
//   forward  X[k] = sum_j x[j] exp(-2 pi i j k / N)
//   backward x[j] = sum_k X[k] exp(+2 pi i j k / N)   (unnormalised)
//
// Codelet constants (w_R^k for R <= 12) are evaluated at compile time by this file's
// own constexpr sin/cos (octant reduction + Taylor series).
#pragma once
#include <cuda_runtime.h>
#include <type_traits>
#include <utility>

#include "check.cuh"

namespace obl {

// Kernel launchers cache one-time set-up (function attributes, occupancy-derived grid
// caps).  Both belong to a device context, so the caches are kept per device; past
// kMaxDevices the set-up is redone on every launch.
constexpr int kMaxDevices = 64;
inline int device_slot()
{
    int d = 0;
    cudaGetDevice(&d);
    return (d >= 0 && d < kMaxDevices) ? d : -1;
}

// ----------------------------------------------------------------------------- complex
template <typename T> struct cplx_t;
template <> struct cplx_t<float> { using type = float2; };
template <> struct cplx_t<double> { using type = double2; };
template <typename T> using C2 = typename cplx_t<T>::type;

template <typename T> __device__ __forceinline__ C2<T> mk(T x, T y) { C2<T> r; r.x = x; r.y = y; return r; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b)
{
    C r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b)
{
    C r;
    r.x = a.x * b.x + a.y * b.y;
    r.y = a.y * b.x - a.x * b.y;
    return r;
}
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
// multiply by -i (fwd) or +i (!fwd)
template <bool FWD, typename C> __device__ __forceinline__ C mul_mi(C a)
{
    C r;
    if (FWD) { r.x = a.y; r.y = -a.x; }
    else     { r.x = -a.y; r.y = a.x; }
    return r;
}
template <typename C, typename S> __device__ __forceinline__ C cscale(C a, S s) { a.x *= s; a.y *= s; return a; }

// ----------------------------------------------------------------------------- constexpr trig
namespace ct {
constexpr double HALF_PI = 1.57079632679489661923132169163975144;
__host__ __device__ constexpr double taylor_sin(double x)
{
    double term = x, sum = x, x2 = x * x;
    for (int n = 1; n < 14; ++n) {
        term *= -x2 / ((2.0 * n) * (2.0 * n + 1.0));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double taylor_cos(double x)
{
    double term = 1.0, sum = 1.0, x2 = x * x;
    for (int n = 1; n < 14; ++n) {
        term *= -x2 / ((2.0 * n - 1.0) * (2.0 * n));
        sum += term;
    }
    return sum;
}
// cos and sin of 2*pi*k/R computed from the exact rational k/R
__host__ __device__ constexpr double cos2pi(long k, long R)
{
    k %= R;
    if (k < 0) k += R;
    long q = (4 * k) / R;        // quadrant
    long r4 = 4 * k - q * R;     // theta = q*pi/2 + (pi/2)*r4/R
    double c = 0, s = 0;
    if (2 * r4 <= R) {
        double psi = HALF_PI * (double)r4 / (double)R;
        c = taylor_cos(psi);
        s = taylor_sin(psi);
    } else {
        double psi = HALF_PI * (double)(R - r4) / (double)R;
        c = taylor_sin(psi);
        s = taylor_cos(psi);
    }
    switch (q) {
    case 0: return c;
    case 1: return -s;
    case 2: return -c;
    default: return s;
    }
}
} // namespace ct

// w_R^K for direction FWD: exp(-+ 2 pi i K / R), applied as a compile-time constant.
template <int R, int K, bool FWD, typename C> __device__ __forceinline__ C twc(C a)
{
    constexpr int k = ((K % R) + R) % R;
    if constexpr (k == 0) {
        return a;
    } else if constexpr (4 * k == R) {          // -i (fwd) / +i
        return mul_mi<FWD>(a);
    } else if constexpr (2 * k == R) {          // -1
        C r; r.x = -a.x; r.y = -a.y; return r;
    } else if constexpr (4 * k == 3 * R) {      // +i (fwd) / -i
        return mul_mi<!FWD>(a);
    } else {
        using T = decltype(a.x);
        constexpr double cr = ct::cos2pi(k, R);
        constexpr double si = ct::cos2pi(4 * k - R, 4 * R);   // sin(2 pi k/R) = cos(2 pi k/R - pi/2)
        const T c = (T)cr;
        const T s = FWD ? (T)(-si) : (T)si;
        C r;
        r.x = a.x * c - a.y * s;
        r.y = a.x * s + a.y * c;
        return r;
    }
}

// ----------------------------------------------------------------------------- compile-time loops
template <int I, int E> struct For {
    template <class F> __device__ __forceinline__ static void run(F &&f)
    {
        if constexpr (I < E) {
            f(std::integral_constant<int, I>{});
            For<I + 1, E>::run(f);
        }
    }
};

// ----------------------------------------------------------------------------- codelets
template <int R, bool FWD> struct Dft;

template <bool FWD> struct Dft<1, FWD> {
    template <typename C> __device__ __forceinline__ static void run(C *) {}
};

template <bool FWD> struct Dft<2, FWD> {
    template <typename C> __device__ __forceinline__ static void run(C *x)
    {
        C a = x[0], b = x[1];
        x[0] = cadd(a, b);
        x[1] = csub(a, b);
    }
};

template <bool FWD> struct Dft<3, FWD> {
    template <typename C> __device__ __forceinline__ static void run(C *x)
    {
        using T = decltype(x[0].x);
        const T h = (T)0.5;
        const T s3 = (T)ct::cos2pi(4 * 1 - 3, 12);   // sin(2 pi/3) = sqrt(3)/2
        C t1 = cadd(x[1], x[2]);
        C t2 = csub(x[0], cscale(t1, h));
        C d = csub(x[1], x[2]);
        C t3 = mul_mi<FWD>(cscale(d, s3));           // -i*sin(2pi/3)*(x1-x2) (fwd)
        x[0] = cadd(x[0], t1);
        x[1] = cadd(t2, t3);
        x[2] = csub(t2, t3);
    }
};

template <bool FWD> struct Dft<4, FWD> {
    template <typename C> __device__ __forceinline__ static void run(C *x)
    {
        C t0 = cadd(x[0], x[2]), t1 = csub(x[0], x[2]);
        C t2 = cadd(x[1], x[3]), t3 = mul_mi<FWD>(csub(x[1], x[3]));
        x[0] = cadd(t0, t2);
        x[2] = csub(t0, t2);
        x[1] = cadd(t1, t3);
        x[3] = csub(t1, t3);
    }
};

// 5-point DFT from its two conjugate-symmetric pairs (x1, x4) and (x2, x3):
//   X_k = x0 + c_k (x1 + x4) + c_2k (x2 + x3) -+ i [s_k (x1 - x4) + s_2k (x2 - x3)],
// with c_k = cos(2 pi k/5), s_k = sin(2 pi k/5); the sign is - for forward.
template <bool FWD> struct Dft<5, FWD> {
    template <typename C> __device__ __forceinline__ static void run(C *x)
    {
        using T = decltype(x[0].x);
        const T c1 = (T)ct::cos2pi(1, 5), c2 = (T)ct::cos2pi(2, 5);
        const T s1 = (T)ct::cos2pi(4 * 1 - 5, 20), s2 = (T)ct::cos2pi(4 * 2 - 5, 20);
        const C t1 = cadd(x[1], x[4]), t2 = cadd(x[2], x[3]);
        const C t3 = csub(x[1], x[4]), t4 = csub(x[2], x[3]);
        C a1, a2, b1, b2;
        a1.x = x[0].x + c1 * t1.x + c2 * t2.x;
        a1.y = x[0].y + c1 * t1.y + c2 * t2.y;
        a2.x = x[0].x + c2 * t1.x + c1 * t2.x;
        a2.y = x[0].y + c2 * t1.y + c1 * t2.y;
        b1.x = s1 * t3.x + s2 * t4.x;
        b1.y = s1 * t3.y + s2 * t4.y;
        b2.x = s2 * t3.x - s1 * t4.x;
        b2.y = s2 * t3.y - s1 * t4.y;
        const C m1 = mul_mi<FWD>(b1), m2 = mul_mi<FWD>(b2);
        x[0] = cadd(x[0], cadd(t1, t2));
        x[1] = cadd(a1, m1);
        x[4] = csub(a1, m1);
        x[2] = cadd(a2, m2);
        x[3] = csub(a2, m2);
    }
};

// Composite codelet R = A*B (four-step, all indices compile time):
//   X[q + B p] = sum_l w_A^{lp} w_R^{lq} sum_m x[l + A m] w_B^{mq}
template <int A, int B, bool FWD> struct DftComp {
    template <typename C> __device__ __forceinline__ static void run(C *x)
    {
        constexpr int R = A * B;
        C y[R]; // y[l*B + q]
        For<0, A>::run([&](auto lc) {
            constexpr int l = decltype(lc)::value;
            C t[B];
            For<0, B>::run([&](auto mc) { constexpr int m = decltype(mc)::value; t[m] = x[l + A * m]; });
            Dft<B, FWD>::run(t);
            For<0, B>::run([&](auto qc) {
                constexpr int q = decltype(qc)::value;
                y[l * B + q] = twc<R, l * q, FWD>(t[q]);
            });
        });
        For<0, B>::run([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            C t[A];
            For<0, A>::run([&](auto lc) { constexpr int l = decltype(lc)::value; t[l] = y[l * B + q]; });
            Dft<A, FWD>::run(t);
            For<0, A>::run([&](auto pc) { constexpr int p = decltype(pc)::value; x[q + B * p] = t[p]; });
        });
    }
};

template <bool FWD> struct Dft<6, FWD> : DftComp<2, 3, FWD> {};
template <bool FWD> struct Dft<8, FWD> : DftComp<2, 4, FWD> {};
template <bool FWD> struct Dft<9, FWD> : DftComp<3, 3, FWD> {};
template <bool FWD> struct Dft<12, FWD> : DftComp<4, 3, FWD> {};
template <bool FWD> struct Dft<16, FWD> : DftComp<4, 4, FWD> {};
template <bool FWD> struct Dft<10, FWD> : DftComp<2, 5, FWD> {};

} // namespace obl
