// Compile-time-sized plane pipeline (the fast path of lh_plane.cu).
//
// Same three stages and the same staging layout as the generic kernels,
// but every transform is a two-pass register FFT (lh_fft.cuh) whose index
// arithmetic folds to constants: z inverse / x products / z forward are one
// template each, instantiated for the Ngal sizes of the usual grids.
// Twiddles are copied once per CTA into shared memory.
#include "lh_fft.cuh"

// resident CTAs per SM the register allocation is sized for
#ifndef LH_FFT_MINB
#define LH_FFT_MINB 2
#endif
#include "lh_kernels.cuh"

namespace lh {

// ---------------------------------------------------------------------------
// z inverse of one (plane, field, block of cb x modes)
template <int NZ>
__global__ void __launch_bounds__(512, LH_FFT_MINB) k_zinv_f(const Inst *__restrict__ insts, const Work *__restrict__ work, int cb)
{
    constexpr int N1 = Plan2<NZ>::N1, N2 = Plan2<NZ>::N2;
    constexpr int Nz = 2 * NZ / 3;
    extern __shared__ double2 sm[];
    double2 *tw = sm, *T = sm + NZ;
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    load_table(tw, I.twz, NZ);
    const int nxh = I.nxh, nc = I.nc, j = w.j;
    const int nblk = (nxh + cb - 1) / cb;
    const int f = w.blk / nblk, i0 = (w.blk % nblk) * cb;
    const double2 *src0, *src1 = nullptr;
    double w0 = 0.0, w1 = 0.0, den = 1.0;
    if (f == 0) src0 = I.U1 + (size_t)j * nc;
    else if (f == 2) src0 = I.U3 + (size_t)j * nc;
    else if (f == 4) src0 = I.U2 + (size_t)j * nc;
    else if (f == 1) {  // u2 at centre j (interp_v, FOU3D.f90:407)
        src0 = I.U2 + (size_t)j * nc;
        src1 = I.U2 + (size_t)(j - 1) * nc;
        w0 = I.yu[j] - I.yv[j - 1];
        w1 = I.yv[j] - I.yu[j];
        den = I.yv[j] - I.yv[j - 1];
    } else {  // u1/u3 at face j (interp_u, FOU3D.f90:387)
        const double2 *base = f == 3 ? I.U1 : I.U3;
        src0 = base + (size_t)(j + 1) * nc;
        src1 = base + (size_t)j * nc;
        w0 = I.yv[j] - I.yu[j];
        w1 = I.yu[j + 1] - I.yv[j];
        den = I.yu[j + 1] - I.yu[j];
    }
    __syncthreads();
    const int t = threadIdx.x, v = t % cb, r = t / cb, i = i0 + v;
    const bool ok = i < nxh;
    if (r < N2) {
        double2 a[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) {
            const int n = r + N2 * n1;
            int kr = -1;
            if (n < Nz / 2) kr = n;
            else if (n >= NZ - Nz / 2) kr = n - (NZ - Nz);
            double2 val = make_double2(0.0, 0.0);
            if (kr >= 0 && ok) {
                const int col = kr * nxh + i;
                if (src1 == nullptr) {
                    val = src0[col];
                } else {
                    const double2 x0 = src0[col], x1 = src1[col];
                    val.x = (w0 * x0.x + w1 * x1.x) / den;
                    val.y = (w0 * x0.y + w1 * x1.y) / den;
                }
            }
            a[n1] = val;
        }
        DFT<N1, +1, NZ>::run(a, tw);
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) {
            double2 z = a[k1];
            if (k1 > 0 && r > 0) z = twiddle<+1>(tw[r * k1], z);
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
            double2 *dst = I.S + ((size_t)(w.slot * kNumProducts + f) * NZ) * nxh + i;
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) dst[(size_t)(r + N1 * k2) * nxh] = b[k2];
        }
    }
}

// ---------------------------------------------------------------------------
// x transforms and products of one (plane, block of rb z rows)
template <int NX>
__global__ void __launch_bounds__(512, LH_FFT_MINB) k_xprod_f(const Inst *__restrict__ insts, const Work *__restrict__ work, int rb,
                                                 int want_max)
{
    constexpr int N1 = Plan2<NX>::N1, N2 = Plan2<NX>::N2;
    extern __shared__ double2 sm[];
    __shared__ double red[2][16];
    double2 *tw = sm, *buf = sm + NX;
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    load_table(tw, I.twx, NX);
    const int Mz = I.Mz, nxh = I.nxh;
    const int q0 = w.blk * rb;
    const int nv = 3 * rb;
    double2 *S = I.S + (size_t)w.slot * kNumProducts * Mz * nxh;
    __syncthreads();
    const int t = threadIdx.x, v = t % nv, r = t / nv;
    const int pr = v / rb, rr = v % rb, q = q0 + rr;
    (void)q;
    // (0) coalesced load of the 6 fields x rb rows x (Nx/2+1) modes: in[f][rr][k]
    double2 *in = buf;
    for (int e = t; e < kNumProducts * rb * nxh; e += blockDim.x) {
        const int k = e % nxh, fr = e / nxh, rr2 = fr % rb, f = fr / rb;
        in[e] = (q0 + rr2 < Mz) ? S[((size_t)f * Mz + q0 + rr2) * nxh + k] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    // (1) inverse pass 1 on the Hermitian extension of two half spectra
    {
        double2 a[N1];
        if (r < N2) {
            const int fa = pr == 0 ? 0 : (pr == 1 ? 1 : 3), fb = pr == 0 ? 2 : (pr == 1 ? 4 : 5);
            const double2 *A = in + (fa * rb + rr) * nxh, *B = in + (fb * rb + rr) * nxh;
#pragma unroll
            for (int n1 = 0; n1 < N1; n1++) {
                const int n = r + N2 * n1;
                double2 z = make_double2(0.0, 0.0);
                if (n == 0) {
                    z = make_double2(A[0].x, B[0].x);  // Im of mode 0 dropped (rft_buff.f:78-81)
                } else if (n < nxh) {
                    const double2 x = A[n], y = B[n];
                    z = make_double2(x.x - y.y, x.y + y.x);
                } else if (NX - n < nxh) {
                    const double2 x = A[NX - n], y = B[NX - n];
                    z = make_double2(x.x + y.y, y.x - x.y);
                }
                a[n1] = z;
            }
        }
        __syncthreads();
        if (r < N2) {
            DFT<N1, +1, NX>::run(a, tw);
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++) {
                double2 z = a[k1];
                if (k1 > 0 && r > 0) z = twiddle<+1>(tw[r * k1], z);
                buf[(k1 * N2 + r) * nv + v] = z;
            }
        }
    }
    __syncthreads();
    // (2) inverse pass 2 -> physical values buf[x][v]
    {
        double2 b[N2];
        if (r < N1) {
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) b[n2] = buf[(r * N2 + n2) * nv + v];
            DFT<N2, +1, NX>::run(b, tw);
        }
        __syncthreads();
        if (r < N1) {
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) buf[(r + N1 * k2) * nv + v] = b[k2];
        }
    }
    __syncthreads();
    // (3) products; CFL maxima over planes 1..nyu-1 (dtc_calc's dummies see
    // actual planes 0..nyu-1, FOU3D.f90:622-626)
    const bool track = want_max && I.dt_mode == 0 && w.j <= I.nyu - 1;
    double m1 = 0.0, m3 = 0.0;
    for (int e = t; e < NX * rb; e += blockDim.x) {
        const int x = e / rb, r2 = e % rb;
        double2 *p = buf + x * nv;
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
            for (int n1 = 0; n1 < N1; n1++) a[n1] = buf[(r + N2 * n1) * nv + v];
            DFT<N1, -1, NX>::run(a, tw);
        }
        __syncthreads();
        if (r < N2) {
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++) {
                double2 z = a[k1];
                if (k1 > 0 && r > 0) z = twiddle<-1>(tw[r * k1], z);
                buf[(k1 * N2 + r) * nv + v] = z;
            }
        }
    }
    __syncthreads();
    // (5) forward pass 2 -> X[k][v]
    {
        double2 b[N2];
        if (r < N1) {
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) b[n2] = buf[(r * N2 + n2) * nv + v];
            DFT<N2, -1, NX>::run(b, tw);
        }
        __syncthreads();
        if (r < N1) {
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) buf[(r + N1 * k2) * nv + v] = b[k2];
        }
    }
    __syncthreads();
    // (6) split the packed real transforms, scale 1/Mx, keep modes i <= Nx/2
    const double dn1 = 1.0 / NX;
    for (int e = t; e < nxh * nv; e += blockDim.x) {
        const int k = e / nv, vv = e % nv;
        const int p2 = vv / rb, r2 = vv % rb, qq = q0 + r2;
        if (qq >= Mz) continue;
        const double2 zk = buf[k * nv + vv];
        const double2 zm = buf[((NX - k) % NX) * nv + vv];
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

// ---------------------------------------------------------------------------
// z forward, masks and derivatives of one (plane, block of cb x modes)
template <int NZ>
__global__ void __launch_bounds__(512, LH_FFT_MINB) k_zfwd_f(const Inst *__restrict__ insts, const Work *__restrict__ work, int cb)
{
    constexpr int N1 = Plan2<NZ>::N1, N2 = Plan2<NZ>::N2;
    constexpr int Nz = 2 * NZ / 3;
    extern __shared__ double2 sm[];
    double2 *tw = sm, *T = sm + NZ;
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    load_table(tw, I.twz, NZ);
    const int nxh = I.nxh, nc = I.nc, j = w.j;
    const int i0 = w.blk * cb;
    const int nv = kNumProducts * cb;
    const double2 *S = I.S + (size_t)w.slot * kNumProducts * NZ * nxh;
    __syncthreads();
    const int t = threadIdx.x, v = t % nv, r = t / nv;
    const int f = v / cb, c = v % cb, i = i0 + c;
    const bool ok = i < nxh;
    if (r < N2) {
        double2 a[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++)
            a[n1] = ok ? S[((size_t)f * NZ + r + N2 * n1) * nxh + i] : make_double2(0.0, 0.0);
        DFT<N1, -1, NZ>::run(a, tw);
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) {
            double2 z = a[k1];
            if (k1 > 0 && r > 0) z = twiddle<-1>(tw[r * k1], z);
            T[(k1 * N2 + r) * nv + v] = z;
        }
    }
    __syncthreads();
    {
        double2 b[N2];
        if (r < N1) {
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) b[n2] = T[(r * N2 + n2) * nv + v];
            DFT<N2, -1, NZ>::run(b, tw);
        }
        __syncthreads();
        if (r < N1) {
            const double dn1 = 1.0 / NZ;
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) T[(r + N1 * k2) * nv + v] = make_double2(dn1 * b[k2].x, dn1 * b[k2].y);
        }
    }
    __syncthreads();
    for (int e = t; e < Nz * cb; e += blockDim.x) {
        const int cc = e % cb, kr = e / cb, ii = i0 + cc;
        if (ii >= nxh) continue;
        const int zp = kr < Nz / 2 ? kr : kr + NZ - Nz;
        const double2 *row = T + zp * nv + cc;
        double2 pr[kNumProducts];
#pragma unroll
        for (int g = 0; g < kNumProducts; g++) pr[g] = row[g * cb];
        const size_t o = (size_t)j * nc + kr * nxh + ii;
        I.VVC[o] = pr[2];
        I.UVF[o] = pr[4];
        I.WVF[o] = pr[5];
        double2 n1 = make_double2(0.0, 0.0), n2 = n1, n3 = n1;
        if (kr != Nz / 2) {  // der_x/der_z zero the kz = -Nz/2 row (FOU3D.f90:444-447)
            const double kx = I.kx[ii], kz = I.kz[kr];
            n1 = make_double2(-(kx * pr[0].y) + -(kz * pr[1].y), kx * pr[0].x + kz * pr[1].x);
            n3 = make_double2(-(kx * pr[1].y) + -(kz * pr[3].y), kx * pr[1].x + kz * pr[3].x);
            n2 = make_double2(-(kx * pr[4].y) + -(kz * pr[5].y), kx * pr[4].x + kz * pr[5].x);
        }
        const size_t on = (size_t)(j - 1) * nc + kr * nxh + ii;
        I.NXZ1[on] = n1;
        I.NXZ2[on] = n2;
        I.NXZ3[on] = n3;
    }
}

// ---------------------------------------------------------------------------
// host dispatch
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

cudaError_t fast_set_attributes(int Mz, int Mx, size_t smz, size_t smx, size_t smf)
{
    cudaError_t e = cudaSuccess;
    switch (Mz) {
#define LH_CASE(N)                                                   \
    case N:                                                          \
        e = cudaFuncSetAttribute(k_zinv_f<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz); \
        if (e == cudaSuccess)                                        \
            e = cudaFuncSetAttribute(k_zfwd_f<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf); \
        break;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    default:
        return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    switch (Mx) {
#define LH_CASE(N)                                                   \
    case N:                                                          \
        e = cudaFuncSetAttribute(k_xprod_f<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx); \
        break;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    default:
        return cudaErrorInvalidValue;
    }
    return e;
}

void fast_launch_zinv(int Mz, unsigned grid, int threads, size_t smem, cudaStream_t st, const Inst *insts,
                      const Work *work, int cb)
{
    switch (Mz) {
#define LH_CASE(N)                                                                   \
    case N:                                                                          \
        k_zinv_f<N><<<grid, threads, smem, st>>>(insts, work, cb);                   \
        break;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    }
}

void fast_launch_xprod(int Mx, unsigned grid, int threads, size_t smem, cudaStream_t st, const Inst *insts,
                       const Work *work, int rb, int want_max)
{
    switch (Mx) {
#define LH_CASE(N)                                                                   \
    case N:                                                                          \
        k_xprod_f<N><<<grid, threads, smem, st>>>(insts, work, rb, want_max);        \
        break;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    }
}

void fast_launch_zfwd(int Mz, unsigned grid, int threads, size_t smem, cudaStream_t st, const Inst *insts,
                      const Work *work, int cb)
{
    switch (Mz) {
#define LH_CASE(N)                                                                   \
    case N:                                                                          \
        k_zfwd_f<N><<<grid, threads, smem, st>>>(insts, work, cb);                   \
        break;
        LH_FAST_SIZES(LH_CASE)
#undef LH_CASE
    }
}

}  // namespace lh
