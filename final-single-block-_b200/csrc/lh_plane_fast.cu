// Compile-time-sized plane pipeline (the fast path of lh_plane.cu).
//
// Every transform is a two-pass register FFT (lh_fft.cuh) whose index
// arithmetic folds to constants; one template per stage, instantiated for
// the Ngal sizes of the usual grids.  One CTA per work item; each lane reads
// its one outer-twiddle base from the table in global memory, so shared
// memory holds only the transform data.
//
// Staging (per instance, inside I.S; the kRoundStreams chunk rounds in
// flight use disjoint shares):
//   Sin  [cap+2*kRoundStreams][3][Mz][nxh]  z-inverse of u1, u3 and u2 on the y rows of
//        a round's planes plus one halo row each side; x stays spectral.
//   Sprod[cap][6][Mz][nxh]    the six products after the forward x
//        transform, one slot per plane of a round.
// The y interpolations of the reference (interp_u/interp_v, FOU3D.f90:
// 373-418) are linear and commute with the z transform, so they are applied
// to the z-transformed rows in the x stage: the z inverse runs on three
// fields per plane instead of six.
#include <cstdlib>

#include "lh_fft.cuh"

// Launch bounds (max threads, min resident CTAs per SM) each kernel's
// register allocation is sized for.
#ifndef LH_FFT_MINB
#define LH_FFT_MINB 2
#endif
#ifndef LH_ZINV_T
#define LH_ZINV_T 256
#endif
#ifndef LH_ZINV_B
#define LH_ZINV_B 3
#endif
#ifndef LH_XPROD_T
#define LH_XPROD_T 256
#endif
#ifndef LH_XPROD_B
#define LH_XPROD_B 3
#endif
#ifndef LH_XMULTI_T
#define LH_XMULTI_T 192
#endif
#ifndef LH_XMULTI_B
#define LH_XMULTI_B 2
#endif
#ifndef LH_ZFWD_T
#define LH_ZFWD_T 256
#endif
#ifndef LH_ZFWD_B
#define LH_ZFWD_B 3
#endif
// The block-synchronous kernels at the large lengths hold longer register
// FFTs (18 and 24 threads per vector at Ngal 288 and 384): at three CTAs per
// SM (80 registers) they spilled 0.1-0.8 KB per thread.  From LH_LARGE_N on,
// the bound is LH_LARGE_B CTAs per SM (128 registers, no spills).  Measured
// on B200 (ms per RK3 step): 256^2 x 257 12.32 -> 10.15; 192^2 x 257 5.04 ->
// 4.88, x 153 3.11 -> 3.01, x 97 2.00 -> 1.93 (with one z row per x CTA; with
// three it lost 1 %); at Ngal 192 two CTAs lost in the step graph.
#ifndef LH_LARGE_N
#define LH_LARGE_N 288
#endif
#ifndef LH_LARGE_B
#define LH_LARGE_B 2
#endif
#define LH_MINB(N, B) ((N) >= LH_LARGE_N ? LH_LARGE_B : (B))
// iterations of the warp-local x stage's gather loop unrolled (its loads of
// later modes are then issued before the shared-memory stores of earlier ones)
#ifndef LH_XGATHER_UNROLL
#define LH_XGATHER_UNROLL 1
#endif
#include "lh_kernels.cuh"

namespace lh {

// Outer twiddles W^(r k1), k1 = 1.., of a two-pass transform by the
// recurrence W^(r k1) = W^(r (k1-1)) W^r from one table entry, which keeps the
// per-point table reads out of the shared-memory pipe (the kernels' busiest
// unit); the recurrence's rounding stays within a few ulp for k1 <= 24.
struct TwStep {
    double2 w1, wk;
    __device__ explicit TwStep(double2 base) : w1(base), wk(make_double2(1.0, 0.0)) {}
    __device__ __forceinline__ double2 next()
    {
        wk = make_double2(wk.x * w1.x - wk.y * w1.y, wk.x * w1.y + wk.y * w1.x);
        return wk;
    }
};

__device__ __forceinline__ double2 *sin_field(const Inst &I, int p, int f)
{
    return I.S + ((size_t)p * 3 + f) * I.Mz * I.nxh;
}
__device__ __forceinline__ double2 *sprod_slot(const Inst &I, int s)
{
    return I.S + ((size_t)(I.chunk + 2 * kRoundStreams) * 3 + (size_t)s * kNumProducts) * I.Mz * I.nxh;
}

// ---------------------------------------------------------------------------
// z inverse of one (y row jp, field f in {u1, u3, u2}, block of cb x modes):
// the pruned cft of four_to_phys_u (FOU3D.f90:653-679), -> Sin[slot][f]
template <int NZ>
__global__ void __launch_bounds__(LH_ZINV_T, LH_MINB(NZ, LH_ZINV_B)) k_zinv_f(const Inst *__restrict__ insts, const Work *__restrict__ work,
                                                         int count, int cb)
{
    constexpr int N1 = Plan2<NZ>::N1, N2 = Plan2<NZ>::N2;
    constexpr int Nz = 2 * NZ / 3;
    extern __shared__ double2 sm[];
    double2 *T = sm;
    if ((int)blockIdx.x >= count) return;
    const double2 *tw = insts[work[blockIdx.x].inst].twz;  // depends on Mz only
    const int t = threadIdx.x, v = t % cb, r = t / cb;
    const double2 twr = __ldg(tw + r);  // outer-twiddle base W^r, issued before the data loads
    {
        const Work w = work[blockIdx.x];
        const Inst &I = insts[w.inst];
        const int nxh = I.nxh, nc = I.nc;
        const int nblk = (nxh + cb - 1) / cb;
        const int f = w.blk / nblk, i = (w.blk % nblk) * cb + v;
        const double2 *src = (f == 0 ? I.U1 : (f == 1 ? I.U3 : I.U2)) + (size_t)w.j * nc;
        const bool ok = i < nxh;
        if (r < N2) {
            double2 a[N1];
#pragma unroll
            for (int n1 = 0; n1 < N1; n1++) {
                const int n = r + N2 * n1;
                int kr = -1;
                if (n < Nz / 2) kr = n;
                else if (n >= NZ - Nz / 2) kr = n - (NZ - Nz);
                a[n1] = (kr >= 0 && ok) ? src[kr * nxh + i] : make_double2(0.0, 0.0);
            }
            DFT<N1, +1, NZ>::run(a, tw);
            TwStep ts(twr);
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++) {
                double2 z = a[k1];
                if (k1 > 0) z = twiddle<+1>(ts.next(), z);
                T[(k1 * N2 + r) * cb + v] = z;
            }
        }
        __syncthreads();
        if (r < N1) {
            double2 b[N2];
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) b[n2] = T[(r * N2 + n2) * cb + v];
            DFT<N2, +1, NZ>::run(b, tw);
            if (ok) {
                double2 *dst = sin_field(I, w.slot, f) + i;
#pragma unroll
                for (int k2 = 0; k2 < N2; k2++) dst[(size_t)(r + N1 * k2) * nxh] = b[k2];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The same z inverse with the threads of a vector in one warp (vector-major:
// thread t works on x mode t / VT, VT = max(N1, N2) in {8, 16}), so the
// exchange between the two passes is warp-local: a __syncwarp instead of
// block barriers, and the warps of a CTA never wait on one another.  The
// N1 x N2 exchange matrix of a vector is stored with a padded row (N2 + 1)
// so the column-wise reads of the second pass are free of bank conflicts.
// Same arithmetic as k_zinv_f, element for element.
template <int NZ>
__global__ void __launch_bounds__(LH_ZINV_T, LH_ZINV_B) k_zinv_w(const Inst *__restrict__ insts, const Work *__restrict__ work,
                                                         int count, int cb)
{
    constexpr int N1 = Plan2<NZ>::N1, N2 = Plan2<NZ>::N2;
    constexpr int VT = N1 > N2 ? N1 : N2;
    // sizes whose vectors do not fit a warp are never launched (zinv_warp_size)
    if constexpr (32 % VT != 0) return;
    constexpr int LD = N2 + 1;
    constexpr int Nz = 2 * NZ / 3;
    extern __shared__ double2 sm[];
    if ((int)blockIdx.x >= count) return;
    const double2 *tw = insts[work[blockIdx.x].inst].twz;
    const int t = threadIdx.x, v = t / VT, r = t % VT;
    const double2 twr = __ldg(tw + (r < N2 ? r : 0));
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    const int nxh = I.nxh, nc = I.nc;
    const int nblk = (nxh + cb - 1) / cb;
    const int f = w.blk / nblk, i = (w.blk % nblk) * cb + v;
    const bool ok = v < cb && i < nxh;
    double2 *T = sm + (size_t)(v < cb ? v : 0) * N1 * LD;
    const double2 *src = (f == 0 ? I.U1 : (f == 1 ? I.U3 : I.U2)) + (size_t)w.j * nc;
    if (v < cb && r < N2) {
        double2 a[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) {
            const int n = r + N2 * n1;
            int kr = -1;
            if (n < Nz / 2) kr = n;
            else if (n >= NZ - Nz / 2) kr = n - (NZ - Nz);
            a[n1] = (kr >= 0 && ok) ? src[kr * nxh + i] : make_double2(0.0, 0.0);
        }
        DFT<N1, +1, NZ>::run(a, tw);
        TwStep ts(twr);
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) {
            double2 z = a[k1];
            if (k1 > 0) z = twiddle<+1>(ts.next(), z);
            T[k1 * LD + r] = z;
        }
    }
    __syncwarp();
    if (ok && r < N1) {
        double2 b[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; n2++) b[n2] = T[r * LD + n2];
        DFT<N2, +1, NZ>::run(b, tw);
        double2 *dst = sin_field(I, w.slot, f) + i;
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) dst[(size_t)(r + N1 * k2) * nxh] = b[k2];
    }
}

// ---------------------------------------------------------------------------
// x transforms and products of one (plane j, block of rb z rows).  Rows are
// gathered from Sin with the y interpolations (interp_v FOU3D.f90:407,
// interp_u :387): fields 0 u1(j), 1 u2 at centre j, 2 u3(j), 3 u1 at face j,
// 4 u2(j), 5 u3 at face j; then inverse real x FFT (two real rows per
// complex FFT), products, forward real x FFT (ops_in_planes2,
// FOU3D.f90:1514-1652) -> Sprod[slot]
template <int NX>
__global__ void __launch_bounds__(LH_XPROD_T, LH_MINB(NX, LH_XPROD_B)) k_xprod_f(const Inst *__restrict__ insts, const Work *__restrict__ work,
                                                          int count, int rb, int want_max)
{
    constexpr int N1 = Plan2<NX>::N1, N2 = Plan2<NX>::N2;
    extern __shared__ double2 sm[];
    __shared__ double red[2][16];
    double2 *buf = sm;
    if ((int)blockIdx.x >= count) return;
    const double2 *tw = insts[work[blockIdx.x].inst].twx;  // depends on Mx only
    // buf[x][v] with an odd row stride ld (double2): the column-wise gather
    // and pass-2 accesses then spread over all bank groups
    const int t = threadIdx.x, nv = 3 * rb, ld = nv | 1, v = t % nv, r = t / nv;
    const double2 twr = __ldg(tw + r);  // outer-twiddle base W^r, issued before the data loads
    constexpr int nxh = NX / 3 + 1;  // Nx/2 + 1 with Mx = 3 Nx / 2
    const FastDiv by_rb(rb), by_nv(nv);
    {
        const Work w = work[blockIdx.x];
        const Inst &I = insts[w.inst];
        const int Mz = I.Mz, j = w.j;
        const int q0 = w.blk * rb;
        const size_t fs = (size_t)Mz * nxh;
        const double2 *u1j = sin_field(I, w.aux + 1, 0), *u3j = u1j + fs, *vj = u3j + fs;
        const double2 *vjm = sin_field(I, w.aux, 2);
        const double2 *u1p = sin_field(I, w.aux + 2, 0), *u3p = u1p + fs;
        const double dnv = 1.0 / (I.yv[j] - I.yv[j - 1]), dnu = 1.0 / (I.yu[j + 1] - I.yu[j]);
        const double w0v = (I.yu[j] - I.yv[j - 1]) * dnv, w1v = (I.yv[j] - I.yu[j]) * dnv;
        const double w0u = (I.yv[j] - I.yu[j]) * dnu, w1u = (I.yu[j + 1] - I.yv[j]) * dnu;
        double2 *S = sprod_slot(I, w.slot);
        // (0) coalesced gather of the rows (k fastest) straight into the packed
        // complex vectors of the inverse transform, z[n][v] (v = pair*rb + row):
        // z = A + iB for the two real rows A, B of a pair, Hermitian-extended,
        // Im of mode 0 dropped (rft_buff.f:78-81), zero between the retained
        // modes
        for (int e = t; e < 3 * rb * nxh; e += blockDim.x) {
            const int fr = e / nxh, k = e - fr * nxh, p2 = by_rb.div(fr), r2 = by_rb.mod(fr, p2);
            const int q = q0 + r2;
            double2 A = make_double2(0.0, 0.0), B = A;
            if (q < Mz) {
                const size_t o = (size_t)q * nxh + k;
                if (p2 == 0) {  // (u1, u3) at the centre
                    A = u1j[o];
                    B = u3j[o];
                } else if (p2 == 1) {  // (u2 at the centre, u2 at the face)
                    const double2 x0 = vj[o], x1 = vjm[o];
                    A = make_double2(w0v * x0.x + w1v * x1.x, w0v * x0.y + w1v * x1.y);
                    B = x0;
                } else {  // (u1, u3) at the face
                    const double2 a0 = u1p[o], a1 = u1j[o], b0 = u3p[o], b1 = u3j[o];
                    A = make_double2(w0u * a0.x + w1u * a1.x, w0u * a0.y + w1u * a1.y);
                    B = make_double2(w0u * b0.x + w1u * b1.x, w0u * b0.y + w1u * b1.y);
                }
            }
            const int vv = p2 * rb + r2;
            if (k == 0) {
                buf[vv] = make_double2(A.x, B.x);
            } else {
                buf[k * ld + vv] = make_double2(A.x - B.y, A.y + B.x);
                buf[(NX - k) * ld + vv] = make_double2(A.x + B.y, B.x - A.y);
            }
        }
        for (int e = t; e < (NX - 2 * nxh + 1) * nv; e += blockDim.x) {
            const int x = by_nv.div(e);
            buf[(nxh + x) * ld + by_nv.mod(e, x)] = make_double2(0.0, 0.0);
        }
        __syncthreads();
        // (1) inverse pass 1: lane r < N2 holds n = r + N2*n1
        {
            double2 a[N1];
            if (r < N2) {
#pragma unroll
                for (int n1 = 0; n1 < N1; n1++) a[n1] = buf[(r + N2 * n1) * ld + v];
            }
            __syncthreads();
            if (r < N2) {
                DFT<N1, +1, NX>::run(a, tw);
                TwStep ts(twr);
#pragma unroll
                for (int k1 = 0; k1 < N1; k1++) {
                    double2 z = a[k1];
                    if (k1 > 0) z = twiddle<+1>(ts.next(), z);
                    buf[(k1 * N2 + r) * ld + v] = z;
                }
            }
        }
        __syncthreads();
        // (2) inverse pass 2 -> physical values buf[x][v]
        {
            double2 b[N2];
            if (r < N1) {
#pragma unroll
                for (int n2 = 0; n2 < N2; n2++) b[n2] = buf[(r * N2 + n2) * ld + v];
                DFT<N2, +1, NX>::run(b, tw);
            }
            __syncthreads();
            if (r < N1) {
#pragma unroll
                for (int k2 = 0; k2 < N2; k2++) buf[(r + N1 * k2) * ld + v] = b[k2];
            }
        }
        __syncthreads();
        // (3) products; CFL maxima over planes 1..nyu-1 (dtc_calc's dummies see
        // actual planes 0..nyu-1, FOU3D.f90:622-626)
        const bool track = want_max && I.dt_mode == 0 && j <= I.nyu - 1;
        double m1 = 0.0, m3 = 0.0;
        for (int e = t; e < NX * rb; e += blockDim.x) {
            const int x = by_rb.div(e), r2 = by_rb.mod(e, x);
            double2 *p = buf + x * ld;
            const double2 p0 = p[r2], p1 = p[rb + r2], p2 = p[2 * rb + r2];
            const double u1 = p0.x, u3 = p0.y, u2c = p1.x, u2 = p1.y, u1f = p2.x, u3f = p2.y;
            if (track && q0 + r2 < Mz) {
                m1 = fmax(m1, fabs(u1));
                m3 = fmax(m3, fabs(u3));
            }
            p[r2] = make_double2(u1 * u1, u1 * u3);
            p[rb + r2] = make_double2(u2c * u2c, u3 * u3);
            p[2 * rb + r2] = make_double2(u1f * u2, u3f * u2);
        }
        if (track) {
            for (int o = 16; o > 0; o >>= 1) {
                m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
                m3 = fmax(m3, __shfl_xor_sync(0xffffffffu, m3, o));
            }
            if ((t & 31) == 0) {
                red[0][t >> 5] = m1;
                red[1][t >> 5] = m3;
            }
        }
        __syncthreads();
        if (track && t == 0) {
            double a1 = 0.0, a3 = 0.0;
            for (int k = 0; k < (int)(blockDim.x + 31) / 32; k++) {
                a1 = fmax(a1, red[0][k]);
                a3 = fmax(a3, red[1][k]);
            }
            atomicMax(reinterpret_cast<unsigned long long *>(&I.sc[SC_U1MAX]), (unsigned long long)__double_as_longlong(a1));
            atomicMax(reinterpret_cast<unsigned long long *>(&I.sc[SC_U3MAX]), (unsigned long long)__double_as_longlong(a3));
        }
        // (4) forward pass 1
        {
            double2 a[N1];
            if (r < N2) {
#pragma unroll
                for (int n1 = 0; n1 < N1; n1++) a[n1] = buf[(r + N2 * n1) * ld + v];
                DFT<N1, -1, NX>::run(a, tw);
            }
            __syncthreads();
            if (r < N2) {
                TwStep ts(twr);
#pragma unroll
                for (int k1 = 0; k1 < N1; k1++) {
                    double2 z = a[k1];
                    if (k1 > 0) z = twiddle<-1>(ts.next(), z);
                    buf[(k1 * N2 + r) * ld + v] = z;
                }
            }
        }
        __syncthreads();
        // (5) forward pass 2 -> X[k][v]
        {
            double2 b[N2];
            if (r < N1) {
#pragma unroll
                for (int n2 = 0; n2 < N2; n2++) b[n2] = buf[(r * N2 + n2) * ld + v];
                DFT<N2, -1, NX>::run(b, tw);
            }
            __syncthreads();
            if (r < N1) {
#pragma unroll
                for (int k2 = 0; k2 < N2; k2++) buf[(r + N1 * k2) * ld + v] = b[k2];
            }
        }
        __syncthreads();
        // (6) split the packed real transforms, scale 1/Mx, keep modes i <= Nx/2
        const double dn1 = 1.0 / NX;
        for (int e = t; e < nxh * nv; e += blockDim.x) {
            const int k = by_nv.div(e), vv = by_nv.mod(e, k);
            const int p2 = by_rb.div(vv), r2 = by_rb.mod(vv, p2), qq = q0 + r2;
            if (qq >= Mz) continue;
            const double2 zk = buf[k * ld + vv];
            const double2 zm = buf[(k == 0 ? 0 : NX - k) * ld + vv];
            double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
            double2 B = make_double2(0.5 * (zk.y + zm.y), 0.5 * (zm.x - zk.x));
            if (k == 0) {
                A.y = 0.0;
                B.y = 0.0;
            }
            S[((size_t)(2 * p2) * Mz + qq) * nxh + k] = make_double2(dn1 * A.x, dn1 * A.y);
            S[((size_t)(2 * p2 + 1) * Mz + qq) * nxh + k] = make_double2(dn1 * B.x, dn1 * B.y);
        }
    }
}

// ---------------------------------------------------------------------------
// The same x stage with the threads of a vector in one warp.  Vector v of a
// CTA is (z row v / 3, pair v % 3); its VT = max(N1, N2) threads are
// consecutive, so the gather, both transforms and the split of a vector
// are warp-local (__syncwarp), and only the products, which combine the
// three pairs of a row, synchronise -- the 96 threads of a row group (2
// rows at VT = 16, 4 at VT = 8) on a named barrier of their own, so the
// groups of a CTA never wait on one another.  Each vector owns one region
// of max(NX, N1 (N2 + 1)) complex: natural order for the gather, the
// products and the first pass's reads, an N1 x (N2 + 1) padded matrix for
// the exchange between the passes (conflict-free column reads).  The CFL
// maxima are reduced per warp.  Same arithmetic as k_xprod_f, element for
// element.
//
// DIRECT = 1: the first pass reads its N1 elements of the packed vector
// straight from the staging rows in global memory (each mode's two rows are
// read by the two lanes holding z[k] and z[NX - k]), so the gather's shared
// memory round trip and its __syncwarp disappear.
template <int NX, int DIRECT>
__global__ void __launch_bounds__(LH_XPROD_T, LH_XPROD_B) k_xprod_w(const Inst *__restrict__ insts, const Work *__restrict__ work,
                                                          int count, int rb, int want_max)
{
    constexpr int N1 = Plan2<NX>::N1, N2 = Plan2<NX>::N2;
    constexpr int VT = N1 > N2 ? N1 : N2;
    if constexpr (32 % VT != 0) return;  // never launched (xprod_warp_size)
    constexpr int LD = N2 + 1;
    constexpr int REG = (NX > N1 * LD ? NX : N1 * LD);
    constexpr int RG = 32 / VT;  // rows per 96-thread group
    constexpr int nxh = NX / 3 + 1;
    extern __shared__ double2 sm[];
    if ((int)blockIdx.x >= count) return;
    const double2 *tw = insts[work[blockIdx.x].inst].twx;
    const int t = threadIdx.x, v = t / VT, r = t % VT;
    const int row = v / 3, pair = v % 3, grp = row / RG;
    const double2 twr = __ldg(tw + (r < N2 ? r : 0));
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    const int Mz = I.Mz, j = w.j;
    const int q = w.blk * rb + row;  // this vector's z row
    const bool live = row < rb;      // threads past the CTA's rows only join the barriers
    const bool rowok = live && q < Mz;
    double2 *z = sm + (size_t)(live ? v : 0) * REG;
    const size_t fs = (size_t)Mz * nxh;
    // (0) this vector's two real rows with the y interpolations (interp_v
    // FOU3D.f90:407, interp_u :387) as the packed Hermitian-extended complex
    // vector z = A + iB: z[0] = (A0.x, B0.x), z[k] = A_k + iB_k and
    // z[NX - k] = conj(A_k) + i conj(B_k) for 0 < k <= Nx/2, zero between
    const double2 *u1j = sin_field(I, w.aux + 1, 0), *u3j = u1j + fs, *vj = u3j + fs;
    const double2 *vjm = sin_field(I, w.aux, 2);
    const double2 *u1p = sin_field(I, w.aux + 2, 0), *u3p = u1p + fs;
    const double dnv = 1.0 / (I.yv[j] - I.yv[j - 1]), dnu = 1.0 / (I.yu[j + 1] - I.yu[j]);
    const double w0v = (I.yu[j] - I.yv[j - 1]) * dnv, w1v = (I.yv[j] - I.yu[j]) * dnv;
    const double w0u = (I.yv[j] - I.yu[j]) * dnu, w1u = (I.yu[j + 1] - I.yv[j]) * dnu;
    auto rows_at = [&](int k, double2 &A, double2 &B) {
        const size_t o = (size_t)q * nxh + k;
        if (pair == 0) {
            A = u1j[o];
            B = u3j[o];
        } else if (pair == 1) {
            const double2 x0 = vj[o], x1 = vjm[o];
            A = make_double2(w0v * x0.x + w1v * x1.x, w0v * x0.y + w1v * x1.y);
            B = x0;
        } else {
            const double2 a0 = u1p[o], a1 = u1j[o], b0 = u3p[o], b1 = u3j[o];
            A = make_double2(w0u * a0.x + w1u * a1.x, w0u * a0.y + w1u * a1.y);
            B = make_double2(w0u * b0.x + w1u * b1.x, w0u * b0.y + w1u * b1.y);
        }
    };
    if (!DIRECT && live) {
        constexpr int kGatherUnroll = LH_XGATHER_UNROLL;
#pragma unroll kGatherUnroll
        for (int k = r; k < nxh; k += VT) {
            double2 A = make_double2(0.0, 0.0), B = A;
            if (rowok) rows_at(k, A, B);
            if (k == 0) {
                z[0] = make_double2(A.x, B.x);
            } else {
                z[k] = make_double2(A.x - B.y, A.y + B.x);
                z[NX - k] = make_double2(A.x + B.y, B.x - A.y);
            }
        }
        for (int x = nxh + r; x <= NX - nxh; x += VT) z[x] = make_double2(0.0, 0.0);
    }
    if (!DIRECT) __syncwarp();
    // (1) inverse pass 1: lane r < N2 holds n = r + N2 n1; out to the padded matrix
    {
        double2 a[N1];
        if (live && r < N2) {
            if (DIRECT) {
#pragma unroll
                for (int n1 = 0; n1 < N1; n1++) {
                    const int n = r + N2 * n1;
                    double2 A = make_double2(0.0, 0.0), B = A, y = A;
                    if (rowok && n < nxh) {
                        rows_at(n, A, B);
                        y = n == 0 ? make_double2(A.x, B.x) : make_double2(A.x - B.y, A.y + B.x);
                    } else if (rowok && n > NX - nxh) {
                        rows_at(NX - n, A, B);
                        y = make_double2(A.x + B.y, B.x - A.y);
                    }
                    a[n1] = y;
                }
            } else {
#pragma unroll
                for (int n1 = 0; n1 < N1; n1++) a[n1] = z[r + N2 * n1];
            }
        }
        if (!DIRECT) __syncwarp();
        if (live && r < N2) {
            DFT<N1, +1, NX>::run(a, tw);
            TwStep ts(twr);
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++) {
                double2 y = a[k1];
                if (k1 > 0) y = twiddle<+1>(ts.next(), y);
                z[k1 * LD + r] = y;
            }
        }
    }
    __syncwarp();
    // (2) inverse pass 2 -> physical values z[x], natural order
    {
        double2 b[N2];
        if (live && r < N1) {
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) b[n2] = z[r * LD + n2];
            DFT<N2, +1, NX>::run(b, tw);
        }
        __syncwarp();
        if (live && r < N1) {
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) z[r + N1 * k2] = b[k2];
        }
    }
    // (3) products of each row group's rows (the three pairs of a row sit in
    // up to two warps of the group); CFL maxima over planes 1..nyu-1
    asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(96) : "memory");
    const bool track = want_max && I.dt_mode == 0 && j <= I.nyu - 1;
    double m1 = 0.0, m3 = 0.0;
    {
        const int gt = t - grp * 96;  // thread within the group
        const int row0 = grp * RG;
        for (int e = gt; e < RG * NX; e += 96) {
            const int rr = row0 + e / NX, x = e % NX;
            if (rr >= rb) continue;
            double2 *p0 = sm + (size_t)(3 * rr) * REG + x, *p1 = p0 + REG, *p2 = p1 + REG;
            const double2 a0 = *p0, a1 = *p1, a2 = *p2;
            const double u1 = a0.x, u3 = a0.y, u2c = a1.x, u2 = a1.y, u1f = a2.x, u3f = a2.y;
            if (track && w.blk * rb + rr < Mz) {
                m1 = fmax(m1, fabs(u1));
                m3 = fmax(m3, fabs(u3));
            }
            *p0 = make_double2(u1 * u1, u1 * u3);
            *p1 = make_double2(u2c * u2c, u3 * u3);
            *p2 = make_double2(u1f * u2, u3f * u2);
        }
    }
    if (track) {
        for (int o = 16; o > 0; o >>= 1) {
            m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
            m3 = fmax(m3, __shfl_xor_sync(0xffffffffu, m3, o));
        }
        if ((t & 31) == 0) {
            atomicMax(reinterpret_cast<unsigned long long *>(&I.sc[SC_U1MAX]), (unsigned long long)__double_as_longlong(m1));
            atomicMax(reinterpret_cast<unsigned long long *>(&I.sc[SC_U3MAX]), (unsigned long long)__double_as_longlong(m3));
        }
    }
    asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(96) : "memory");
    // (4) forward pass 1
    {
        double2 a[N1];
        if (live && r < N2) {
#pragma unroll
            for (int n1 = 0; n1 < N1; n1++) a[n1] = z[r + N2 * n1];
            DFT<N1, -1, NX>::run(a, tw);
        }
        __syncwarp();
        if (live && r < N2) {
            TwStep ts(twr);
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++) {
                double2 y = a[k1];
                if (k1 > 0) y = twiddle<-1>(ts.next(), y);
                z[k1 * LD + r] = y;
            }
        }
    }
    __syncwarp();
    // (5) forward pass 2 -> X[k], natural order
    {
        double2 b[N2];
        if (live && r < N1) {
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) b[n2] = z[r * LD + n2];
            DFT<N2, -1, NX>::run(b, tw);
        }
        __syncwarp();
        if (live && r < N1) {
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) z[r + N1 * k2] = b[k2];
        }
    }
    __syncwarp();
    // (6) split the packed real transforms, scale 1/Mx, keep modes i <= Nx/2
    if (rowok) {
        double2 *S = sprod_slot(I, w.slot);
        const double dn1 = 1.0 / NX;
        for (int k = r; k < nxh; k += VT) {
            const double2 zk = z[k];
            const double2 zm = z[k == 0 ? 0 : NX - k];
            double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
            double2 B = make_double2(0.5 * (zk.y + zm.y), 0.5 * (zm.x - zk.x));
            if (k == 0) {
                A.y = 0.0;
                B.y = 0.0;
            }
            S[((size_t)(2 * pair) * Mz + q) * nxh + k] = make_double2(dn1 * A.x, dn1 * A.y);
            S[((size_t)(2 * pair + 1) * Mz + q) * nxh + k] = make_double2(dn1 * B.x, dn1 * B.y);
        }
    }
}

// Two-pass transform of one packed vector of length NX held by the VT lanes
// of a warp in its shared-memory region z (natural order in and out; the
// N1 x (N2 + 1) padded matrix in between).  SGN = +1 inverse, -1 forward.
// Every lane of the warp calls it (act = false only joins the __syncwarp).
template <int NX, int SGN>
__device__ __forceinline__ void xvec_fft(double2 *z, const double2 *tw, double2 twr, int r, bool act)
{
    constexpr int N1 = Plan2<NX>::N1, N2 = Plan2<NX>::N2;
    constexpr int LD = N2 + 1;
    __syncwarp();
    {
        double2 a[N1];
        if (act && r < N2) {
#pragma unroll
            for (int n1 = 0; n1 < N1; n1++) a[n1] = z[r + N2 * n1];
        }
        __syncwarp();
        if (act && r < N2) {
            DFT<N1, SGN, NX>::run(a, tw);
            TwStep ts(twr);
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++) {
                double2 y = a[k1];
                if (k1 > 0) y = twiddle<SGN>(ts.next(), y);
                z[k1 * LD + r] = y;
            }
        }
    }
    __syncwarp();
    {
        double2 b[N2];
        if (act && r < N1) {
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) b[n2] = z[r * LD + n2];
            DFT<N2, SGN, NX>::run(b, tw);
        }
        __syncwarp();
        if (act && r < N1) {
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) z[r + N1 * k2] = b[k2];
        }
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// The x stage over a group of consecutive planes (the default where a
// vector fits a warp).  The y interpolations are linear and commute with
// the x transform too, so this stage transforms each y row's fields once --
// (u1, u3) of a u plane as one packed vector, two adjacent v rows as
// another -- and interpolates the physical rows of neighbouring planes: u2
// at the u plane (interp_v, FOU3D.f90:407), u1 and u3 at the v plane
// (interp_u, :387), with the weights of k_xprod_w.  Per plane that is 1.5
// inverse transforms instead of 3, and 3 staging rows read instead of 8.
//
// A work item is a group of np <= kXGroup planes j .. j+np-1 and a block of
// rb z rows; the plan starts groups at absolute planes 1 + kXGroup g, and v
// rows are paired from the group's first plane, V_m = (v(j-1+2m), v(j+2m)),
// so every row is transformed with the same partner -- and every plane's
// products come out of the same operations -- whatever the plan's rounds,
// staging budget or batch, as long as a round holds at least kXGroup planes
// (below that the groups are cut at the round boundaries).  A row's physical
// values depend on the partner packed with it at the rounding level.
//
// Each z row runs sub-rounds of three vectors on its three vector slots
// (VT lanes each, one warp-local transform per vector): sub-round 0
// transforms A_0 = (u1, u3)(j), A_1 and V_0, after which plane j's products
// are formed and transformed forward; sub-round k >= 1 transforms A_2k,
// A_2k+1 and V_k, after which planes j+2k-1 and j+2k follow.  Regions per z
// row: three for the A vectors (index mod 3), two for the V vectors (mod 2)
// and two for the second and third product pairs; the first pair (u1 u1,
// u1 u3) overwrites A_p in place.  Row groups of 96 threads synchronise on a
// named barrier of their own before each sub-round and around each plane's
// products.  Same transforms, products, split and CFL maxima as k_xprod_w.
template <int NX>
__global__ void __launch_bounds__(LH_XMULTI_T, LH_XMULTI_B) k_xprod_m(const Inst *__restrict__ insts,
                                                                      const Work *__restrict__ work, int count,
                                                                      int rb, int want_max)
{
    constexpr int N1 = Plan2<NX>::N1, N2 = Plan2<NX>::N2;
    constexpr int VT = N1 > N2 ? N1 : N2;
    if constexpr (32 % VT != 0) return;  // never launched (xprod_warp_size)
    constexpr int LD = N2 + 1;
    constexpr int REG = (NX > N1 * LD ? NX : N1 * LD);
    constexpr int RG = 32 / VT;  // rows per 96-thread group
    constexpr int nxh = NX / 3 + 1;
    constexpr int kRegions = 7;
    extern __shared__ double2 sm[];
    if ((int)blockIdx.x >= count) return;
    const double2 *tw = insts[work[blockIdx.x].inst].twx;
    const int t = threadIdx.x, v = t / VT, r = t % VT;
    const int row = v / 3, slot = v % 3, grp = row / RG;
    const double2 twr = __ldg(tw + (r < N2 ? r : 0));
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    const int Mz = I.Mz, j = w.j, np = w.blk >> 16;
    const int q = (w.blk & 0xffff) * rb + row;  // this thread's z row
    const bool live = row < rb;                  // threads past the CTA's rows only join the barriers
    const bool rowok = live && q < Mz;
    double2 *const R = sm + (size_t)(live ? row : 0) * kRegions * REG;
    const size_t fs = (size_t)Mz * nxh, orow = (size_t)q * nxh;
    const bool track = want_max && I.dt_mode == 0;
    double m1 = 0.0, m3 = 0.0;
    // sub-round k: the inverse transforms of A_2k, A_2k+1 and V_k
    auto subround = [&](const int k) {
        // the regions this sub-round fills were last read by other slots
        if (k > 0) asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(96) : "memory");
        double2 *z;
        const double2 *sa = nullptr, *sb = nullptr;
        bool act = live;
        if (slot < 2) {
            const int tt = 2 * k + slot;  // A_tt: (u1, u3) of plane j + tt
            z = R + (tt % 3) * REG;
            act = act && tt <= np;
            sa = sin_field(I, w.aux + 1 + tt, 0);
            sb = sa + fs;
        } else {
            // V_k: v rows j-1+2k and j+2k; the second is past the group only
            // when np is even, i.e. in the last group below the top wall,
            // where it is the ghost row above v(nyu): zero
            z = R + (3 + (k & 1)) * REG;
            sa = sin_field(I, w.aux + 2 * k, 2);
            sb = 2 * k < np ? sin_field(I, w.aux + 2 * k + 1, 2) : nullptr;
        }
        if (act) {
            for (int m = r; m < nxh; m += VT) {
                double2 A = make_double2(0.0, 0.0), B = A;
                if (rowok) {
                    A = sa[orow + m];
                    if (sb) B = sb[orow + m];
                }
                if (m == 0) {
                    z[0] = make_double2(A.x, B.x);
                } else {
                    z[m] = make_double2(A.x - B.y, A.y + B.x);
                    z[NX - m] = make_double2(A.x + B.y, B.x - A.y);
                }
            }
            for (int x = nxh + r; x <= NX - nxh; x += VT) z[x] = make_double2(0.0, 0.0);
        }
        xvec_fft<NX, +1>(z, tw, twr, r, act);
    };
    // plane j + p: products, forward transforms and split
    auto plane = [&](const int p) {
        const int jp = j + p;
        const double dnv = 1.0 / (I.yv[jp] - I.yv[jp - 1]), dnu = 1.0 / (I.yu[jp + 1] - I.yu[jp]);
        const double w0v = (I.yu[jp] - I.yv[jp - 1]) * dnv, w1v = (I.yv[jp] - I.yu[jp]) * dnv;
        const double w0u = (I.yv[jp] - I.yu[jp]) * dnu, w1u = (I.yu[jp + 1] - I.yv[jp]) * dnu;
        const bool trk = track && jp <= I.nyu - 1;
        asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(96) : "memory");
        {
            const int gt = t - grp * 96, row0 = grp * RG;
            const int ra = p % 3, rn = (p + 1) % 3, rvm = 3 + ((p >> 1) & 1), rvv = 3 + (((p + 1) >> 1) & 1);
            for (int e = gt; e < RG * NX; e += 96) {
                const int rr = row0 + e / NX, x = e % NX;
                if (rr >= rb) continue;
                double2 *Rr = sm + (size_t)rr * kRegions * REG;
                const double2 a0 = Rr[ra * REG + x], a1 = Rr[rn * REG + x];
                const double2 c0 = Rr[rvm * REG + x], c1 = Rr[rvv * REG + x];
                const double u1 = a0.x, u3 = a0.y;
                const double vm = (p & 1) ? c0.y : c0.x;        // v(jp - 1)
                const double u2 = ((p + 1) & 1) ? c1.y : c1.x;  // v(jp)
                const double u2c = w0v * u2 + w1v * vm;
                const double u1f = w0u * a1.x + w1u * u1, u3f = w0u * a1.y + w1u * u3;
                if (trk && (w.blk & 0xffff) * rb + rr < Mz) {
                    m1 = fmax(m1, fabs(u1));
                    m3 = fmax(m3, fabs(u3));
                }
                Rr[ra * REG + x] = make_double2(u1 * u1, u1 * u3);
                Rr[5 * REG + x] = make_double2(u2c * u2c, u3 * u3);
                Rr[6 * REG + x] = make_double2(u1f * u2, u3f * u2);
            }
        }
        asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(96) : "memory");
        double2 *zf = R + (slot == 0 ? p % 3 : 4 + slot) * REG;
        xvec_fft<NX, -1>(zf, tw, twr, r, live);
        // split the packed real transforms, scale 1/Mx, keep modes i <= Nx/2
        if (rowok) {
            double2 *S = sprod_slot(I, w.slot + p);
            const double dn1 = 1.0 / NX;
            for (int m = r; m < nxh; m += VT) {
                const double2 zk = zf[m];
                const double2 zm = zf[m == 0 ? 0 : NX - m];
                double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
                double2 B = make_double2(0.5 * (zk.y + zm.y), 0.5 * (zm.x - zk.x));
                if (m == 0) {
                    A.y = 0.0;
                    B.y = 0.0;
                }
                S[((size_t)(2 * slot) * Mz + q) * nxh + m] = make_double2(dn1 * A.x, dn1 * A.y);
                S[((size_t)(2 * slot + 1) * Mz + q) * nxh + m] = make_double2(dn1 * B.x, dn1 * B.y);
            }
        }
    };
    // straight-line code for the group size: as a runtime loop over the
    // sub-rounds the compiler keeps values live across iterations and spills
    // (168 registers and 1.3 KB of spills at Mx = 192, against 124 and none)
    static_assert(kXGroup == 5, "the sequence below covers groups of five planes");
    subround(0);
    plane(0);
    if (np > 1) {
        subround(1);
        plane(1);
        if (np > 2) plane(2);
    }
    if (np > 3) {
        subround(2);
        plane(3);
        if (np > 4) plane(4);
    }
    if (track) {
        for (int o = 16; o > 0; o >>= 1) {
            m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
            m3 = fmax(m3, __shfl_xor_sync(0xffffffffu, m3, o));
        }
        if ((t & 31) == 0) {
            atomicMax(reinterpret_cast<unsigned long long *>(&I.sc[SC_U1MAX]), (unsigned long long)__double_as_longlong(m1));
            atomicMax(reinterpret_cast<unsigned long long *>(&I.sc[SC_U3MAX]), (unsigned long long)__double_as_longlong(m3));
        }
    }
}

// ---------------------------------------------------------------------------
// z forward, masks and derivatives of one (plane, block of cb x modes, half):
// phys_to_four_du's cft (FOU3D.f90:1654-1672), der_x/der_z (:420-523) and
// planes_to_modes_UVP/NUVP.  The six products split into two independent
// halves: {uu, uw, ww} -> Nu1 and Nu3 x/z parts; {vv, uv, wv} -> vv_c, uv_f,
// wv_f and the Nu2 x/z part.
template <int NZ>
__global__ void __launch_bounds__(LH_ZFWD_T, LH_MINB(NZ, LH_ZFWD_B)) k_zfwd_f(const Inst *__restrict__ insts, const Work *__restrict__ work,
                                                         int count, int cb)
{
    constexpr int N1 = Plan2<NZ>::N1, N2 = Plan2<NZ>::N2;
    constexpr int Nz = 2 * NZ / 3;
    extern __shared__ double2 sm[];
    double2 *T = sm;
    if ((int)blockIdx.x >= count) return;
    const double2 *tw = insts[work[blockIdx.x].inst].twz;  // depends on Mz only
    // T[z][v] with an odd row stride ld (double2), as in the x stage
    const int t = threadIdx.x, nv = 3 * cb, ld = nv | 1, v = t % nv, r = t / nv;
    const double2 twr = __ldg(tw + r);  // outer-twiddle base W^r, issued before the data loads
    const int f = v / cb, c = v % cb;
    const FastDiv by_cb(cb);
    {
        const Work w = work[blockIdx.x];
        const Inst &I = insts[w.inst];
        const int nxh = I.nxh, nc = I.nc, j = w.j;
        const int h = w.blk & 1;
        const int i0 = (w.blk >> 1) * cb, i = i0 + c;
        const int g = h == 0 ? (f == 2 ? 3 : f) : (f == 0 ? 2 : f + 3);  // product of this vector
        const double2 *S = sprod_slot(I, w.slot);
        const bool ok = i < nxh;
        if (r < N2) {
            double2 a[N1];
#pragma unroll
            for (int n1 = 0; n1 < N1; n1++)
                a[n1] = ok ? S[((size_t)g * NZ + r + N2 * n1) * nxh + i] : make_double2(0.0, 0.0);
            DFT<N1, -1, NZ>::run(a, tw);
            TwStep ts(twr);
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++) {
                double2 z = a[k1];
                if (k1 > 0) z = twiddle<-1>(ts.next(), z);
                T[(k1 * N2 + r) * ld + v] = z;
            }
        }
        __syncthreads();
        {
            double2 b[N2];
            if (r < N1) {
#pragma unroll
                for (int n2 = 0; n2 < N2; n2++) b[n2] = T[(r * N2 + n2) * ld + v];
                DFT<N2, -1, NZ>::run(b, tw);
            }
            __syncthreads();
            if (r < N1) {
                const double dn1 = 1.0 / NZ;
#pragma unroll
                for (int k2 = 0; k2 < N2; k2++) T[(r + N1 * k2) * ld + v] = make_double2(dn1 * b[k2].x, dn1 * b[k2].y);
            }
        }
        __syncthreads();
        for (int e = t; e < Nz * cb; e += blockDim.x) {
            const int kr = by_cb.div(e), cc = by_cb.mod(e, kr), ii = i0 + cc;
            if (ii >= nxh) continue;
            const int zp = kr < Nz / 2 ? kr : kr + NZ - Nz;
            const double2 *row = T + zp * ld + cc;
            const double2 p0 = row[0], p1 = row[cb], p2 = row[2 * cb];
            const size_t on = (size_t)(j - 1) * nc + kr * nxh + ii;
            const bool keep = kr != Nz / 2;  // der_x/der_z zero the kz = -Nz/2 row (FOU3D.f90:444-447)
            const double kx = I.kx[ii], kz = I.kz[kr];
            if (h == 0) {  // p0 uu, p1 uw, p2 ww
                double2 n1 = make_double2(0.0, 0.0), n3 = n1;
                if (keep) {
                    n1 = make_double2(-(kx * p0.y) + -(kz * p1.y), kx * p0.x + kz * p1.x);
                    n3 = make_double2(-(kx * p1.y) + -(kz * p2.y), kx * p1.x + kz * p2.x);
                }
                I.NXZ1[on] = n1;
                I.NXZ3[on] = n3;
            } else {  // p0 vv, p1 uv, p2 wv
                const size_t o = (size_t)j * nc + kr * nxh + ii;
                I.VVC[o] = p0;
                I.UVF[o] = p1;
                I.WVF[o] = p2;
                double2 n2 = make_double2(0.0, 0.0);
                if (keep) n2 = make_double2(-(kx * p1.y) + -(kz * p2.y), kx * p1.x + kz * p2.x);
                I.NXZ2[on] = n2;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The same z forward with the threads of a vector in one warp.  Vector v is
// (product f = v / cb, x mode c = v % cb), so the two vectors of a warp are
// neighbouring x modes of one product and its loads of a z row share their
// sectors.  Both transform passes are warp-local (__syncwarp); one block
// barrier precedes the masks and derivatives, which combine the three
// products of an x mode.  Each vector owns one region of max(NZ, N1 (N2+1))
// complex (the padded exchange matrix, then the scaled spectrum in natural
// order).  Same arithmetic as k_zfwd_f, element for element.
template <int NZ>
__global__ void __launch_bounds__(LH_ZFWD_T, LH_ZFWD_B) k_zfwd_w(const Inst *__restrict__ insts, const Work *__restrict__ work,
                                                         int count, int cb)
{
    constexpr int N1 = Plan2<NZ>::N1, N2 = Plan2<NZ>::N2;
    constexpr int VT = N1 > N2 ? N1 : N2;
    if constexpr (32 % VT != 0) return;  // never launched (zfwd_warp_size)
    constexpr int LD = N2 + 1;
    // region stride rounded up to odd (in double2): the masks step reads the
    // same z row of neighbouring modes' regions, which then fall in
    // different banks
    constexpr int REG = (NZ > N1 * LD ? NZ : N1 * LD) | 1;
    constexpr int Nz = 2 * NZ / 3;
    extern __shared__ double2 sm[];
    if ((int)blockIdx.x >= count) return;
    const double2 *tw = insts[work[blockIdx.x].inst].twz;
    const int t = threadIdx.x, v = t / VT, r = t % VT;
    const int f = v / cb, c = v % cb;
    const bool live = f < 3;
    const double2 twr = __ldg(tw + (r < N2 ? r : 0));
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    const int nxh = I.nxh, nc = I.nc, j = w.j;
    const int h = w.blk & 1;
    const int i0 = (w.blk >> 1) * cb, i = i0 + c;
    const int g = h == 0 ? (f == 2 ? 3 : f) : (f == 0 ? 2 : f + 3);  // product of this vector
    const double2 *S = sprod_slot(I, w.slot);
    const bool ok = live && i < nxh;
    double2 *z = sm + (size_t)(live ? v : 0) * REG;
    {
        double2 a[N1];
        if (live && r < N2) {
#pragma unroll
            for (int n1 = 0; n1 < N1; n1++)
                a[n1] = ok ? S[((size_t)g * NZ + r + N2 * n1) * nxh + i] : make_double2(0.0, 0.0);
            DFT<N1, -1, NZ>::run(a, tw);
            TwStep ts(twr);
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++) {
                double2 y = a[k1];
                if (k1 > 0) y = twiddle<-1>(ts.next(), y);
                z[k1 * LD + r] = y;
            }
        }
    }
    __syncwarp();
    {
        double2 b[N2];
        if (live && r < N1) {
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) b[n2] = z[r * LD + n2];
            DFT<N2, -1, NZ>::run(b, tw);
        }
        __syncwarp();
        if (live && r < N1) {
            const double dn1 = 1.0 / NZ;
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) z[r + N1 * k2] = make_double2(dn1 * b[k2].x, dn1 * b[k2].y);
        }
    }
    __syncthreads();
    const FastDiv by_cb(cb);
    for (int e = t; e < Nz * cb; e += blockDim.x) {
        const int kr = by_cb.div(e), cc = by_cb.mod(e, kr), ii = i0 + cc;
        if (ii >= nxh) continue;
        const int zp = kr < Nz / 2 ? kr : kr + NZ - Nz;
        const double2 p0 = sm[(size_t)cc * REG + zp], p1 = sm[(size_t)(cb + cc) * REG + zp],
                      p2 = sm[(size_t)(2 * cb + cc) * REG + zp];
        const size_t on = (size_t)(j - 1) * nc + kr * nxh + ii;
        const bool keep = kr != Nz / 2;  // der_x/der_z zero the kz = -Nz/2 row (FOU3D.f90:444-447)
        const double kx = I.kx[ii], kz = I.kz[kr];
        if (h == 0) {  // p0 uu, p1 uw, p2 ww
            double2 n1 = make_double2(0.0, 0.0), n3 = n1;
            if (keep) {
                n1 = make_double2(-(kx * p0.y) + -(kz * p1.y), kx * p0.x + kz * p1.x);
                n3 = make_double2(-(kx * p1.y) + -(kz * p2.y), kx * p1.x + kz * p2.x);
            }
            I.NXZ1[on] = n1;
            I.NXZ3[on] = n3;
        } else {  // p0 vv, p1 uv, p2 wv
            const size_t o = (size_t)j * nc + kr * nxh + ii;
            I.VVC[o] = p0;
            I.UVF[o] = p1;
            I.WVF[o] = p2;
            double2 n2 = make_double2(0.0, 0.0);
            if (keep) n2 = make_double2(-(kx * p1.y) + -(kz * p2.y), kx * p1.x + kz * p2.x);
            I.NXZ2[on] = n2;
        }
    }
}

// ---------------------------------------------------------------------------
// host dispatch
int fast_max_threads(int stage) { return stage == 0 ? LH_ZINV_T : (stage == 1 ? LH_XPROD_T : LH_ZFWD_T); }
int xprod_max_threads(int n) { return xprod_multi(n) ? LH_XMULTI_T : LH_XPROD_T; }

bool fast_size(int n)
{
    switch (n) {
#define LH_CASE(N) case N:
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
        return true;
    default:
        return false;
    }
}

// Threads one vector of length n uses: max(N1, N2) of its two-pass split.
int fast_vector_threads(int n)
{
    switch (n) {
#define LH_CASE(N) \
    case N:        \
        return Plan2<N>::N1 > Plan2<N>::N2 ? Plan2<N>::N1 : Plan2<N>::N2;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    default:
        return 0;
    }
}

int fast_threads(int n, int vectors)
{
    int n1 = 1, n2 = 1;
    switch (n) {
#define LH_CASE(N)              \
    case N:                     \
        n1 = Plan2<N>::N1;      \
        n2 = Plan2<N>::N2;      \
        break;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    default:
        return 0;
    }
    int t = vectors * (n1 > n2 ? n1 : n2);
    return ((t + 31) / 32) * 32;
}

// z-inverse sizes whose vectors fit a warp (max(N1, N2) divides 32), and
// whether the warp-local variant is selected (LH_ZINV_WARP=1).
bool zinv_warp_size(int n)
{
    switch (n) {
#define LH_CASE(N) \
    case N:        \
        return 32 % (Plan2<N>::N1 > Plan2<N>::N2 ? Plan2<N>::N1 : Plan2<N>::N2) == 0;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    default:
        return false;
    }
}

bool zinv_warp(int n)
{
    const char *ev = getenv("LH_ZINV_WARP");
    return ev && ev[0] == '1' && zinv_warp_size(n);
}

// x stage: sizes whose vectors fit a warp, and the variant selection.
// Where a vector fits a warp the warp-local k_xprod_w is the default
// (measured on B200 at 128x128x153: x products 0.256 -> 0.236 ms per
// substep, step 1.283 -> 1.218 ms); LH_XPROD_WARP selects the others for
// measurement: 0 the block-synchronous k_xprod_f, 2 k_xprod_w's direct-read
// form, 3 the multi-plane k_xprod_m.
bool xprod_warp_size(int n) { return zinv_warp_size(n); }
static int xprod_mode(int n)
{
    if (!xprod_warp_size(n)) return 0;
    const char *ev = getenv("LH_XPROD_WARP");
    if (!ev || !*ev || ev[0] == '1') return 1;
    return ev[0] == '3' ? 3 : (ev[0] == '2' ? 2 : 0);
}
bool xprod_warp(int n) { return xprod_mode(n) != 0; }
bool xprod_multi(int n) { return xprod_mode(n) == 3; }

// Threads and shared memory of an x-stage CTA of rb z rows: the warp variants
// run 96-thread row groups (32 / VT rows each), one region per vector
// (k_xprod_w) or seven per z row (k_xprod_m).
int xprod_threads(int n, int rb)
{
    if (!xprod_warp(n)) return fast_threads(n, 3 * rb);
    const int vt = fast_vector_threads(n), rg = 32 / vt;
    return 96 * ((rb + rg - 1) / rg);
}

size_t xprod_smem(int n, int rb)
{
    const int mode = xprod_mode(n);
    if (mode == 0) return (size_t)n * ((3 * rb) | 1) * sizeof(double2);
    const int per_row = mode == 3 ? 7 : 3;
    switch (n) {
#define LH_CASE(N)                                                                                  \
    case N: {                                                                                       \
        const int reg = N > Plan2<N>::N1 * (Plan2<N>::N2 + 1) ? N : Plan2<N>::N1 * (Plan2<N>::N2 + 1); \
        const int rg = 32 / fast_vector_threads(N);                                                 \
        return (size_t)per_row * rg * ((rb + rg - 1) / rg) * reg * sizeof(double2);               \
    }
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    default:
        return 0;
    }
}

// z forward: sizes whose vectors fit a warp, the LH_ZFWD_WARP=1 selection,
// threads and shared memory of a CTA of cb x modes (3 cb vectors)
bool zfwd_warp(int n)
{
    const char *ev = getenv("LH_ZFWD_WARP");
    return ev && ev[0] == '1' && zinv_warp_size(n);
}

int zfwd_threads(int n, int cb)
{
    if (!zfwd_warp(n)) return fast_threads(n, 3 * cb);
    return ((3 * cb * fast_vector_threads(n) + 31) / 32) * 32;
}

size_t zfwd_smem(int n, int cb)
{
    if (!zfwd_warp(n)) return (size_t)n * ((3 * cb) | 1) * sizeof(double2);
    switch (n) {
#define LH_CASE(N)                                                                                  \
    case N: {                                                                                       \
        const int reg = (N > Plan2<N>::N1 * (Plan2<N>::N2 + 1) ? N : Plan2<N>::N1 * (Plan2<N>::N2 + 1)) | 1; \
        return (size_t)3 * cb * reg * sizeof(double2);                                            \
    }
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    default:
        return 0;
    }
}

// Shared memory of a z-inverse CTA of cb vectors.
size_t zinv_smem(int n, int cb)
{
    if (!zinv_warp(n)) return (size_t)n * cb * sizeof(double2);
    switch (n) {
#define LH_CASE(N) \
    case N:        \
        return (size_t)cb * Plan2<N>::N1 * (Plan2<N>::N2 + 1) * sizeof(double2);
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    default:
        return 0;
    }
}

cudaError_t fast_set_attributes(int Mz, int Mx, size_t smz, size_t smx, size_t smf)
{
    cudaError_t e = cudaSuccess;
    switch (Mz) {
#define LH_CASE(N)                                        \
    case N:                                               \
        e = raise_smem_limit((const void *)k_zinv_f<N>, smz); \
        if (e == cudaSuccess) e = raise_smem_limit((const void *)k_zinv_w<N>, smz); \
        if (e == cudaSuccess) e = raise_smem_limit((const void *)k_zfwd_f<N>, smf); \
        if (e == cudaSuccess) e = raise_smem_limit((const void *)k_zfwd_w<N>, smf); \
        break;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    default:
        return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    switch (Mx) {
#define LH_CASE(N)                                         \
    case N:                                                \
        e = raise_smem_limit((const void *)k_xprod_f<N>, smx); \
        if (e == cudaSuccess) e = raise_smem_limit((const void *)k_xprod_w<N, 0>, smx); \
        if (e == cudaSuccess) e = raise_smem_limit((const void *)k_xprod_w<N, 1>, smx); \
        if (e == cudaSuccess) e = raise_smem_limit((const void *)k_xprod_m<N>, smx); \
        break;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    default:
        return cudaErrorInvalidValue;
    }
    return e;
}

void fast_launch_zinv(int Mz, unsigned grid, int threads, size_t smem, cudaStream_t st, const Inst *insts,
                      const Work *work, int count, int cb)
{
    switch (Mz) {
#define LH_CASE(N)                                                                   \
    case N:                                                                          \
        if (zinv_warp(N)) k_zinv_w<N><<<grid, threads, smem, st>>>(insts, work, count, cb); \
        else k_zinv_f<N><<<grid, threads, smem, st>>>(insts, work, count, cb);       \
        break;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    }
}

void fast_launch_xprod(int Mx, unsigned grid, int threads, size_t smem, cudaStream_t st, const Inst *insts,
                       const Work *work, int count, int rb, int want_max)
{
    switch (Mx) {
#define LH_CASE(N)                                                                   \
    case N:                                                                          \
        switch (xprod_mode(N)) {                                                     \
        case 3: k_xprod_m<N><<<grid, threads, smem, st>>>(insts, work, count, rb, want_max); break; \
        case 2: k_xprod_w<N, 1><<<grid, threads, smem, st>>>(insts, work, count, rb, want_max); break; \
        case 1: k_xprod_w<N, 0><<<grid, threads, smem, st>>>(insts, work, count, rb, want_max); break; \
        default: k_xprod_f<N><<<grid, threads, smem, st>>>(insts, work, count, rb, want_max); \
        }                                                                            \
        break;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    }
}

void fast_launch_zfwd(int Mz, unsigned grid, int threads, size_t smem, cudaStream_t st, const Inst *insts,
                      const Work *work, int count, int cb)
{
    switch (Mz) {
#define LH_CASE(N)                                                                   \
    case N:                                                                          \
        if (zfwd_warp(N)) k_zfwd_w<N><<<grid, threads, smem, st>>>(insts, work, count, cb); \
        else k_zfwd_f<N><<<grid, threads, smem, st>>>(insts, work, count, cb);       \
        break;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    }
}

}  // namespace lh
