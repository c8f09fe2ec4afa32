// Device-side data model and FFT building blocks of the B200 time-step engine.
//
// State layout in HBM (per channel instance): every spectral field is
// plane-major, element (j, column) at j*ncols + column, complex FP64 as
// double2.  column = kr*(Nx/2+1) + i with kr the spectral z row (0..Nz-1,
// kz >= 0 first, then kz < 0) and i the x mode (0..Nx/2) -- the reference's
// np=1 column order (start.f90:964-981) -- so one y-plane is contiguous and
// x is fastest inside it.  Plane kernels read whole planes; column kernels
// (one thread per column) read row j of all columns with unit stride.  The
// reference's MPI plane<->column transposes (FOU3D.f90:718-2001) therefore
// have no counterpart at run time; the only transposes are the host-layout
// conversions at upload/download.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lh {

constexpr int kMaxRad = 12;
constexpr int kNumProducts = 6;
// Chunk rounds of the plane pipeline in flight at once, on as many streams,
// each with its own share of the staging.
#ifndef LH_ROUND_STREAMS
#define LH_ROUND_STREAMS 2
#endif
constexpr int kRoundStreams = LH_ROUND_STREAMS;
// Planes per work item of the multi-plane x stage (odd, so that its v-row
// pairs, which start at the group's first plane, cover the group exactly);
// groups start at absolute planes 1 + kXGroup g.
constexpr int kXGroup = 5;

// Radix-3 constant exactly as the reference's FFTPACK carries it
// (cft_buff.f:333, rft_buff.f:364): 15 significant digits.
constexpr double kTaur = -0.5;
constexpr double kTaui = 0.866025403784439;

// Scalars kept on the device so a step can be captured in a CUDA graph.
enum Scalar {
    SC_T = 0,      // simulation time
    SC_DT = 1,     // current dt
    SC_MPGX = 2,   // mean pressure gradient (changes with flag_ctpress = 0)
    SC_U1MAX = 3,  // bit pattern of max|u1| for the CFL rule
    SC_U3MAX = 4,  // bit pattern of max|u3|
    SC_QX = 5,     // flow rate of the (0,0) mode after the last step
    SC_QXT = 6,    // target flow rate (flag_ctpress = 0)
    SC_ITER = 7,   // completed RK3 steps
    SC_DTC = 8,    // convective dt of the last CFL evaluation
    SC_DGX = 9,    // last pressure-gradient correction
    SC_COUNT = 16
};

// Error word bits
enum DevError { ERR_NONFINITE = 1 };

struct Inst {
    // sizes
    int Nx, Nz, Mx, Mz, nxh, nc, nyu, nyv;
    int dt_mode, flag_ctpress;
    int nradz, nradx;
    int radz[kMaxRad], radx[kMaxRad];
    // parameters
    double Re, alp, bet, CFL, dtv, dt_fixed;
    double gw1, gw2, gwbc, gwi1, gwi2, ddthetavi;
    // grid and operators (device pointers)
    const double *yu, *yv, *dthdyu, *dthdyv;  // yu[0..nyu+1], yv[0..nyv+1]
    const double *dyu2i, *dyv2i;              // [3*j + r]
    const double *kx, *kz, *k2x, *k2z;        // kx[i], kz[kr]
    const double *DG1;                        // [j], j = 1..nyu
    const double *DG2, *DG3;                  // [(j-1)*nc + col]
    const double2 *twz, *twx;                 // exp(+2 pi i t / M)
    // state
    double2 *U1, *U2, *U3, *P;                // U1/U3 rows 0..nyu+1, U2 0..nyv+1, P 1..nyu
    double2 *NU1, *NU2, *NU3;                 // Nu of the last substep, rows 1..
    double2 *NXZ1, *NXZ2, *NXZ3;              // x/z part of Nu, rows 1..nyu
    double2 *UVF, *WVF, *VVC;                 // y-flux spectra, rows 0..nyu(+1)
    double *FACU, *FACV;                      // scaled upper diagonals
    double2 *PSI;                             // pressure correction, rows 1..nyu
    double2 *Y1, *Y2, *Y3;                    // forward-eliminated rows of a split column pass
    double2 *CARRY;                           // sweep state between its chunks [3][6][nc]
    double *U11, *F11;                        // (0,0)-mode flow-rate solve, rows 0..nyu+1
    double2 *S;                               // plane-pipeline staging
    double *sc;                               // Scalar slots
    int *err;
    int chunk;                                // staging capacity in planes
};

// One unit of work for a batched launch.
struct Work {
    int inst;   // instance index
    int j;      // plane (plane kernels) or column block (column kernel)
    int slot;   // staging slot of the plane
    int blk;    // sub-block
    int aux;    // x stage: Sin slot of row j-1
};

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// Twiddle product w*c (SGN=+1, backward) or conj(w)*c (SGN=-1, forward) in
// the operation order of passb*/passf* (cft_buff.f:313-324, 759-770).
template <int SGN>
__device__ __forceinline__ double2 twiddle(double2 w, double2 c)
{
    if (SGN > 0) return make_double2(w.x * c.x - w.y * c.y, w.x * c.y + w.y * c.x);
    return make_double2(w.x * c.x + w.y * c.y, w.x * c.y - w.y * c.x);
}

// Radix butterflies with the reference's operation order.
template <int SGN>
__device__ __forceinline__ void dft3(double2 &a0, double2 &a1, double2 &a2)
{
    // passb3/passf3 (cft_buff.f:354-372)
    double2 t1 = cadd(a1, a2), t2 = csub(a1, a2);
    double2 y0 = cadd(a0, t1);
    double2 m = make_double2(a0.x + kTaur * t1.x, a0.y + kTaur * t1.y);
    const double ti = SGN > 0 ? kTaui : -kTaui;
    double2 c3 = make_double2(ti * t2.x, ti * t2.y);
    a0 = y0;
    a1 = make_double2(m.x - c3.y, m.y + c3.x);
    a2 = make_double2(m.x + c3.y, m.y - c3.x);
}

template <int SGN>
__device__ __forceinline__ void dft4(double2 &a0, double2 &a1, double2 &a2, double2 &a3)
{
    // passb4/passf4 (cft_buff.f:411-452)
    double2 c4 = SGN > 0 ? make_double2(a3.y - a1.y, a1.x - a3.x) : make_double2(a1.y - a3.y, a3.x - a1.x);
    double2 c2 = cadd(a0, a2), c3 = cadd(a1, a3), c1 = csub(a0, a2);
    a0 = cadd(c2, c3);
    a2 = csub(c2, c3);
    a1 = cadd(c1, c4);
    a3 = csub(c1, c4);
}

// One self-sorting (Stockham, decimation in frequency) pass over a batch of
// nv vectors of length N stored [n][v] in shared memory.  Same index map as
// the reference passes: input cc(i, j, k) = x[i + m (j + p k)], output
// c1(i, k, j') = y[i + m (k + l1 j')], twiddle W_N^(i j' l1) applied after
// the butterfly (cft_buff.f:247-274).
template <int SGN>
__device__ __forceinline__ void stockham_pass(const double2 *__restrict__ in, double2 *__restrict__ out, int N,
                                              int p, int l1, int nv, const double2 *__restrict__ tw, int tid,
                                              int nthr)
{
    const int m = N / (p * l1);
    const int total = (N / p) * nv;
    for (int w = tid; w < total; w += nthr) {
        const int v = w % nv;
        const int bi = w / nv;
        const int i = bi % m;
        const int k = bi / m;
        const int ib = i + m * p * k;
        const int ob = i + m * k;
        if (p == 4) {
            double2 a0 = in[(ib) * nv + v], a1 = in[(ib + m) * nv + v], a2 = in[(ib + 2 * m) * nv + v],
                    a3 = in[(ib + 3 * m) * nv + v];
            dft4<SGN>(a0, a1, a2, a3);
            if (i > 0) {
                a1 = twiddle<SGN>(__ldg(&tw[i * l1]), a1);
                a2 = twiddle<SGN>(__ldg(&tw[2 * i * l1]), a2);
                a3 = twiddle<SGN>(__ldg(&tw[3 * i * l1]), a3);
            }
            out[(ob)*nv + v] = a0;
            out[(ob + m * l1) * nv + v] = a1;
            out[(ob + 2 * m * l1) * nv + v] = a2;
            out[(ob + 3 * m * l1) * nv + v] = a3;
        } else if (p == 3) {
            double2 a0 = in[(ib)*nv + v], a1 = in[(ib + m) * nv + v], a2 = in[(ib + 2 * m) * nv + v];
            dft3<SGN>(a0, a1, a2);
            if (i > 0) {
                a1 = twiddle<SGN>(__ldg(&tw[i * l1]), a1);
                a2 = twiddle<SGN>(__ldg(&tw[2 * i * l1]), a2);
            }
            out[(ob)*nv + v] = a0;
            out[(ob + m * l1) * nv + v] = a1;
            out[(ob + 2 * m * l1) * nv + v] = a2;
        } else {
            double2 a0 = in[(ib)*nv + v], a1 = in[(ib + m) * nv + v];
            double2 y0 = cadd(a0, a1), y1 = csub(a0, a1);
            if (i > 0) y1 = twiddle<SGN>(__ldg(&tw[i * l1]), y1);
            out[(ob)*nv + v] = y0;
            out[(ob + m * l1) * nv + v] = y1;
        }
    }
}

// Full transform of a batch: ping-pong between a and b; returns the buffer
// holding the result.  All threads of the block must call it.
template <int SGN>
__device__ double2 *fft_batch(double2 *a, double2 *b, int N, const int *rad, int nrad, int nv,
                              const double2 *__restrict__ tw)
{
    const int tid = threadIdx.x, nthr = blockDim.x;
    int l1 = 1;
    double2 *src = a, *dst = b;
    for (int s = 0; s < nrad; s++) {
        const int p = rad[s];
        stockham_pass<SGN>(src, dst, N, p, l1, nv, tw, tid, nthr);
        __syncthreads();
        l1 *= p;
        double2 *t = src;
        src = dst;
        dst = t;
    }
    return src;
}

}  // namespace lh
