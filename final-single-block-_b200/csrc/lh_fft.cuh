// Register-resident FFT building blocks with compile-time sizes.
//
// DFT<R, SGN, NT>::run transforms R complex values held in registers
// (natural order in and out) by mixed-radix Cooley-Tukey splits R = P*Q,
// P in {4, 3, 2}; all indices are compile-time constants and the internal
// twiddles are immediates (RootSel).  The outer twiddles of the two-pass
// long transform start from one entry per lane of the table
// tw[m] = exp(+2 pi i m / NT) in global memory (the rotation-recurrence
// table for z, direct cos/sin for x).
//
// A length-N transform of a batch is done in two passes, N = N1 * N2:
//   pass 1: per (vector, n2): DFT_N1 over x[n2 + N2 n1], twiddle W_N^(n2 k1)
//   pass 2: per (vector, k1): DFT_N2 over n2  ->  X[k1 + N1 k2]
// with one shared-memory exchange in between.
#pragma once

#include "lh_core.cuh"

namespace lh {

// Compile-time roots of unity exp(+2 pi i m / R): the angle is reduced to
// [0, pi/4] by the symmetries of sin and cos and evaluated by Taylor series
// (14 terms, far below one ulp on that interval).
struct CW {
    double c, s;
};
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double taylor_sin(double x)
{
    double t = x, s = x;
    for (int n = 1; n < 14; n++) {
        t *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
        s += t;
    }
    return s;
}
constexpr double taylor_cos(double x)
{
    double t = 1.0, s = 1.0;
    for (int n = 1; n < 14; n++) {
        t *= -x * x / ((2.0 * n - 1.0) * (2.0 * n));
        s += t;
    }
    return s;
}
constexpr CW unit_root(int m, int R)
{
    long a = 8L * (((m % R) + R) % R), d = R;  // angle = (pi/4) a/d, a/d in [0, 8)
    double sc = 1.0, ss = 1.0;
    bool swap = false;
    if (a > 4 * d) {  // theta > pi: cos(2pi - theta), -sin(2pi - theta)
        a = 8 * d - a;
        ss = -1.0;
    }
    if (a > 2 * d) {  // theta > pi/2: -cos(pi - theta), sin(pi - theta)
        a = 4 * d - a;
        sc = -1.0;
    }
    if (a > d) {  // theta > pi/4: sin and cos of pi/2 - theta
        a = 2 * d - a;
        swap = true;
    }
    const double x = kPi / 4.0 * (double)a / (double)d;
    double c = taylor_cos(x), s = taylor_sin(x);
    if (swap) {
        const double tmp = c;
        c = s;
        s = tmp;
    }
    return CW{sc * c, ss * s};
}

// Root m (0 <= m < R, a constant after unrolling) as an immediate.
template <int R, int K = 0>
struct RootSel {
    static __device__ __forceinline__ double2 get(int m)
    {
        if (m == K) {
            constexpr CW w = unit_root(K, R);
            return make_double2(w.c, w.s);
        }
        return RootSel<R, K + 1>::get(m);
    }
};
template <int R>
struct RootSel<R, R> {
    static __device__ __forceinline__ double2 get(int) { return make_double2(1.0, 0.0); }
};

// c times the root exp(SGN 2 pi i m / R); quarter turns are exact swaps,
// eighth turns use the factored (x -+ y) sqrt(1/2) form.
template <int SGN, int R>
__device__ __forceinline__ double2 twiddle_const(int m, double2 c)
{
    const int mm = m % R;
    if (mm == 0) return c;
    if (2 * mm == R) return make_double2(-c.x, -c.y);
    if (4 * mm == R) return SGN > 0 ? make_double2(-c.y, c.x) : make_double2(c.y, -c.x);
    if (4 * mm == 3 * R) return SGN > 0 ? make_double2(c.y, -c.x) : make_double2(-c.y, c.x);
    if ((8 * mm) % R == 0) {
        constexpr double h = 0.70710678118654752440084436210484904;
        const double2 w = RootSel<R>::get(mm);  // (+-h, +-h)
        const double wc = w.x > 0.0 ? 1.0 : -1.0, ws = SGN * (w.y > 0.0 ? 1.0 : -1.0);
        // (wc + i ws) h (x + i y) = h (wc x - ws y) + i h (wc y + ws x)
        return make_double2(h * (wc * c.x - ws * c.y), h * (wc * c.y + ws * c.x));
    }
    return twiddle<SGN>(RootSel<R>::get(mm), c);
}

template <int R>
struct Split {
    static constexpr int P = (R % 4 == 0) ? 4 : ((R % 3 == 0) ? 3 : 2);
    static constexpr int Q = R / P;
};

template <int R, int SGN, int NT>
struct DFT {
    static __device__ __forceinline__ void run(double2 *a, const double2 *tw)
    {
        constexpr int P = Split<R>::P, Q = Split<R>::Q;
        double2 b[Q][P];
#pragma unroll
        for (int q = 0; q < Q; q++) {
#pragma unroll
            for (int p = 0; p < P; p++) b[q][p] = a[q + Q * p];
            DFT<P, SGN, NT>::run(b[q], tw);
            if (q > 0) {
#pragma unroll
                for (int k1 = 1; k1 < P; k1++) b[q][k1] = twiddle_const<SGN, R>(q * k1, b[q][k1]);
            }
        }
#pragma unroll
        for (int k1 = 0; k1 < P; k1++) {
            double2 c[Q];
#pragma unroll
            for (int q = 0; q < Q; q++) c[q] = b[q][k1];
            DFT<Q, SGN, NT>::run(c, tw);
#pragma unroll
            for (int k2 = 0; k2 < Q; k2++) a[k1 + P * k2] = c[k2];
        }
    }
};

template <int SGN, int NT>
struct DFT<1, SGN, NT> {
    static __device__ __forceinline__ void run(double2 *, const double2 *) {}
};

template <int SGN, int NT>
struct DFT<2, SGN, NT> {
    static __device__ __forceinline__ void run(double2 *a, const double2 *)
    {
        const double2 t = a[0];
        a[0] = cadd(t, a[1]);
        a[1] = csub(t, a[1]);
    }
};

template <int SGN, int NT>
struct DFT<3, SGN, NT> {
    static __device__ __forceinline__ void run(double2 *a, const double2 *) { dft3<SGN>(a[0], a[1], a[2]); }
};

template <int SGN, int NT>
struct DFT<4, SGN, NT> {
    static __device__ __forceinline__ void run(double2 *a, const double2 *) { dft4<SGN>(a[0], a[1], a[2], a[3]); }
};

// Two-pass split N = N1 * N2 of a length-N transform: the pair with the
// smallest max(N1, N2) (threads per vector are max(N1, N2), so a lopsided
// split idles most of them in one pass), N1 in {16, 12, 9, 8, 6, 4, 3, 2},
// N2 <= 24 and 3-smooth; ties keep the larger N1.
constexpr bool smooth23(int n)
{
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    return n == 1;
}
constexpr int plan2_n1(int N)
{
    const int cand[8] = {16, 12, 9, 8, 6, 4, 3, 2};
    int best = 1, score = N;
    for (int k = 0; k < 8; k++) {
        const int c = cand[k];
        if (N % c != 0 || N / c > 24 || !smooth23(N / c)) continue;
        const int sc = c > N / c ? c : N / c;
        if (sc < score) {
            score = sc;
            best = c;
        }
    }
    return best;
}
template <int N>
struct Plan2 {
    static constexpr int N1 = plan2_n1(N);
    static constexpr int N2 = N / N1;
};

// q = e / d and e % d for 0 <= e < 2^16 and a runtime divisor 1 <= d < 2^16,
// by one multiply-high with m = ceil(2^32 / d): e*m/2^32 = e/d + e*delta/(d*2^32)
// with 0 <= delta < d, and e*delta < 2^32 keeps the excess below 1/d.
struct FastDiv {
    unsigned d, m;
    __device__ explicit FastDiv(int dd) : d((unsigned)dd), m(dd > 1 ? (unsigned)(0xFFFFFFFFull / (unsigned)dd + 1) : 0u) {}
    __device__ __forceinline__ int div(int e) const { return d > 1 ? (int)__umulhi((unsigned)e, m) : e; }
    __device__ __forceinline__ int mod(int e, int q) const { return e - q * (int)d; }
};

// Sizes with a compiled fast path (Ngal = 3N/2 of the usual channel grids).
#define LH_FAST_SIZES(X) X(12) X(24) X(48) X(96) X(144) X(192) X(288) X(384)

}  // namespace lh
