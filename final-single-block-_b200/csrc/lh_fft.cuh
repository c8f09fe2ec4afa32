// Register-resident FFT building blocks with compile-time sizes.
//
// DFT<R, SGN, NT>::run transforms R complex values held in registers
// (natural order in and out) by mixed-radix Cooley-Tukey splits R = P*Q,
// P in {4, 3, 2}; all indices are compile-time constants.  Twiddles are read
// from a table tw[m] = exp(+2 pi i m / NT) held in shared memory (R divides
// NT), so the constants come from the same table the long transform uses
// (the rotation-recurrence table for z, direct cos/sin for x).
//
// A length-N transform of a batch is done in two passes, N = N1 * N2:
//   pass 1: per (vector, n2): DFT_N1 over x[n2 + N2 n1], twiddle W_N^(n2 k1)
//   pass 2: per (vector, k1): DFT_N2 over n2  ->  X[k1 + N1 k2]
// with one shared-memory exchange in between.
#pragma once

#include "lh_core.cuh"

namespace lh {

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
                for (int k1 = 1; k1 < P; k1++) b[q][k1] = twiddle<SGN>(tw[(q * k1 * (NT / R)) % NT], b[q][k1]);
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

// Two-pass split of a length-N transform.
template <int N>
struct Plan2 {
    static constexpr int N1 = (N % 16 == 0 && N / 16 <= 24) ? 16
                              : (N % 8 == 0 && N / 8 <= 24) ? 8
                              : (N % 4 == 0 && N / 4 <= 24) ? 4
                              : (N % 2 == 0) ? 2 : 1;
    static constexpr int N2 = N / N1;
};

// Sizes with a compiled fast path (Ngal = 3N/2 of the usual channel grids).
#define LH_FAST_SIZES(X) X(12) X(24) X(48) X(96) X(144) X(192) X(288) X(384)

__device__ __forceinline__ void load_table(double2 *dst, const double2 *__restrict__ src, int n)
{
    for (int t = threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
}

}  // namespace lh
