// Plane pipeline: the pseudo-spectral nonlinear term of one RK3 substep.
//
// Replaces interp_u/interp_v (FOU3D.f90:373-418), modes_to_planes_UVP x6
// (:126-131), ops_in_planes2 (:1514-1652) with four_to_phys_u (:653-679) and
// phys_to_four_du (:1654-1672) on FFTPACK cft/rft, der_x/der_z (:420-523)
// and planes_to_modes_UVP/NUVP x6 (:248-261).  Three kernels per chunk of
// y-planes, staging through a per-instance buffer S that stays resident in
// L2 when the chunk is sized for it:
//
//   k_zinv  : gather 6 velocity fields of a plane (3 at u centres, 3 at v
//             faces, interpolated in y on the fly), inverse complex FFT along
//             z on the Nx/2+1 retained x modes (the pruned cft of the
//             reference), -> S[slot][field][q][i]
//   k_xprod : per z row: inverse real FFT along x (two real rows packed in
//             one complex FFT), the six products uu uw vv ww (u planes) and
//             uv wv (v planes), forward real FFT, keep modes i <= Nx/2
//             -> S (in place)
//   k_zfwd  : forward complex FFT along z, the reference's masks, x/z
//             derivatives and the y-flux spectra -> NXZ1..3, UVF, WVF, VVC
//
// All arithmetic is FP64.  The z transforms use the reference's radix order
// and its rotation-recurrence twiddle table so they round like cft.
#include "lh_core.cuh"

namespace lh {

// ---------------------------------------------------------------------------
// z inverse: one CTA per (instance, plane, field, block of x modes)
// field: 0 u1(j)  1 u2 at centre j  2 u3(j)  3 u1 at face j  4 u2(j)  5 u3 at face j
__global__ void k_zinv(const Inst *__restrict__ insts, const Work *__restrict__ work, int bc)
{
    extern __shared__ double2 sm[];
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    const int Mz = I.Mz, Nz = I.Nz, nxh = I.nxh, nc = I.nc;
    const int j = w.j;
    const int nblk = (nxh + bc - 1) / bc;
    const int f = w.blk / nblk;
    const int i0 = (w.blk % nblk) * bc;
    double2 *a = sm, *b = sm + Mz * bc;

    // interpolation weights (interp_v FOU3D.f90:407, interp_u FOU3D.f90:387)
    const double2 *src0 = nullptr, *src1 = nullptr;
    double w0 = 0.0, w1 = 0.0, den = 1.0;
    switch (f) {
    case 0: src0 = I.U1 + (size_t)j * nc; break;
    case 2: src0 = I.U3 + (size_t)j * nc; break;
    case 4: src0 = I.U2 + (size_t)j * nc; break;
    case 1:  // u2 at centre j from faces j, j-1
        src0 = I.U2 + (size_t)j * nc;
        src1 = I.U2 + (size_t)(j - 1) * nc;
        w0 = I.yu[j] - I.yv[j - 1];
        w1 = I.yv[j] - I.yu[j];
        den = I.yv[j] - I.yv[j - 1];
        break;
    default: {  // u1/u3 at face j from centres j+1, j
        const double2 *base = f == 3 ? I.U1 : I.U3;
        src0 = base + (size_t)(j + 1) * nc;
        src1 = base + (size_t)j * nc;
        w0 = I.yv[j] - I.yu[j];
        w1 = I.yu[j + 1] - I.yv[j];
        den = I.yu[j + 1] - I.yu[j];
    }
    }
    const int tot = Mz * bc;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int v = t % bc, q = t / bc;
        const int i = i0 + v;
        int kr = -1;
        if (q < Nz / 2) kr = q;
        else if (q >= Mz - Nz / 2) kr = q - (Mz - Nz);
        double2 val = make_double2(0.0, 0.0);
        if (kr >= 0 && i < nxh) {
            const int col = kr * nxh + i;
            if (src1 == nullptr) {
                val = src0[col];
            } else {
                double2 x0 = src0[col], x1 = src1[col];
                val.x = (w0 * x0.x + w1 * x1.x) / den;
                val.y = (w0 * x0.y + w1 * x1.y) / den;
            }
        }
        a[q * bc + v] = val;
    }
    __syncthreads();
    double2 *r = fft_batch<+1>(a, b, Mz, I.radz, I.nradz, bc, I.twz);
    double2 *dst = I.S + ((size_t)(w.slot * kNumProducts + f) * Mz) * nxh;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int v = t % bc, q = t / bc;
        const int i = i0 + v;
        if (i < nxh) dst[(size_t)q * nxh + i] = r[q * bc + v];
    }
}

__device__ __forceinline__ void atomic_max_pos(double *slot, double v)
{
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long *>(slot), (unsigned long long)__double_as_longlong(v));
}

// ---------------------------------------------------------------------------
// x transforms and products: one CTA per (instance, plane, block of z rows)
// Packed pairs: 0 (u1, u3)  1 (u2c, u2)  2 (u1f, u3f)
// Products:     0 (uu, uw)  1 (vv, ww)  2 (uv, wv)
__global__ void k_xprod(const Inst *__restrict__ insts, const Work *__restrict__ work, int br, int want_max)
{
    extern __shared__ double2 sm[];
    __shared__ double red[2][32];
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    const int Mx = I.Mx, Mz = I.Mz, nxh = I.nxh;
    const int q0 = w.blk * br;
    const int nr = min(br, Mz - q0);
    const int nv = 3 * br;
    double2 *a = sm, *b = sm + Mx * nv;
    double2 *S = I.S + (size_t)w.slot * kNumProducts * Mz * nxh;
    const int fa[3] = {0, 1, 3}, fb[3] = {2, 4, 5};

    // Hermitian extension of two half spectra into one complex spectrum.
    const int tot = Mx * nv;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int v = t % nv, n = t / nv;
        const int pr = v / br, r = v % br;
        double2 z = make_double2(0.0, 0.0);
        if (r < nr) {
            const int q = q0 + r;
            const double2 *A = S + ((size_t)fa[pr] * Mz + q) * nxh;
            const double2 *B = S + ((size_t)fb[pr] * Mz + q) * nxh;
            if (n == 0) {
                z = make_double2(A[0].x, B[0].x);  // Im of mode 0 is dropped (rft_buff.f:78-81)
            } else if (n < nxh) {
                double2 x = A[n], y = B[n];
                z = make_double2(x.x - y.y, x.y + y.x);
            } else if (Mx - n < nxh) {
                double2 x = A[Mx - n], y = B[Mx - n];
                z = make_double2(x.x + y.y, y.x - x.y);
            }
        }
        a[n * nv + v] = z;
    }
    __syncthreads();
    double2 *x = fft_batch<+1>(a, b, Mx, I.radx, I.nradx, nv, I.twx);

    // products, optional CFL maxima (planes 1..nyu-1 only: dtc_calc's
    // explicit-shape dummies see actual planes 0..nyu-1, FOU3D.f90:622-626)
    double m1 = 0.0, m3 = 0.0;
    const bool track = want_max && I.dt_mode == 0 && w.j <= I.nyu - 1;
    const int half = Mx * br;
    for (int t = threadIdx.x; t < half; t += blockDim.x) {
        const int r = t % br, n = t / br;
        double2 p0 = x[n * nv + r], p1 = x[n * nv + br + r], p2 = x[n * nv + 2 * br + r];
        const double u1 = p0.x, u3 = p0.y, u2c = p1.x, u2 = p1.y, u1f = p2.x, u3f = p2.y;
        if (track && r < nr) {
            m1 = fmax(m1, fabs(u1));
            m3 = fmax(m3, fabs(u3));
        }
        x[n * nv + r] = make_double2(u1 * u1, u1 * u3);
        x[n * nv + br + r] = make_double2(u2c * u2c, u3 * u3);
        x[n * nv + 2 * br + r] = make_double2(u1f * u2, u3f * u2);
    }
    if (track) {
        for (int o = 16; o > 0; o >>= 1) {
            m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
            m3 = fmax(m3, __shfl_xor_sync(0xffffffffu, m3, o));
        }
        if ((threadIdx.x & 31) == 0) {
            red[0][threadIdx.x >> 5] = m1;
            red[1][threadIdx.x >> 5] = m3;
        }
    }
    __syncthreads();
    if (track && threadIdx.x == 0) {
        double a1 = 0.0, a3 = 0.0;
        for (int k = 0; k < (int)(blockDim.x + 31) / 32; k++) {
            a1 = fmax(a1, red[0][k]);
            a3 = fmax(a3, red[1][k]);
        }
        atomic_max_pos(&I.sc[SC_U1MAX], a1);
        atomic_max_pos(&I.sc[SC_U3MAX], a3);
    }
    double2 *y = fft_batch<-1>(x, x == a ? b : a, Mx, I.radx, I.nradx, nv, I.twx);

    // split the two real transforms, scale 1/Mx (rft_buff.f:64-74), keep i <= Nx/2
    const double dn1 = 1.0 / Mx;
    const int tot2 = nxh * nv;
    for (int t = threadIdx.x; t < tot2; t += blockDim.x) {
        const int v = t % nv, k = t / nv;
        const int pr = v / br, r = v % br;
        if (r >= nr) continue;
        const double2 zk = y[k * nv + v];
        const double2 zm = y[((Mx - k) % Mx) * nv + v];
        double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
        double2 B = make_double2(0.5 * (zk.y + zm.y), 0.5 * (zm.x - zk.x));
        if (k == 0) {
            A.y = 0.0;
            B.y = 0.0;
        }
        A.x *= dn1;
        A.y *= dn1;
        B.x *= dn1;
        B.y *= dn1;
        const int q = q0 + r;
        S[((size_t)(2 * pr) * Mz + q) * nxh + k] = A;
        S[((size_t)(2 * pr + 1) * Mz + q) * nxh + k] = B;
    }
}

// ---------------------------------------------------------------------------
// z forward, masks and derivatives: one CTA per (instance, plane, x-mode block)
__global__ void k_zfwd(const Inst *__restrict__ insts, const Work *__restrict__ work, int bc)
{
    extern __shared__ double2 sm[];
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    const int Mz = I.Mz, Nz = I.Nz, nxh = I.nxh, nc = I.nc;
    const int j = w.j;
    const int i0 = w.blk * bc;
    const int nv = kNumProducts * bc;
    double2 *a = sm, *b = sm + Mz * nv;
    const double2 *S = I.S + (size_t)w.slot * kNumProducts * Mz * nxh;
    const int tot = Mz * nv;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int v = t % nv, q = t / nv;
        const int f = v / bc, c = v % bc, i = i0 + c;
        a[q * nv + v] = i < nxh ? S[((size_t)f * Mz + q) * nxh + i] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    double2 *y = fft_batch<-1>(a, b, Mz, I.radz, I.nradz, nv, I.twz);
    const double dn1 = 1.0 / Mz;
    const int tot2 = Nz * bc;
    for (int t = threadIdx.x; t < tot2; t += blockDim.x) {
        const int c = t % bc, kr = t / bc, i = i0 + c;
        if (i >= nxh) continue;
        const int zp = kr < Nz / 2 ? kr : kr + Mz - Nz;
        double2 pr[kNumProducts];
#pragma unroll
        for (int f = 0; f < kNumProducts; f++) {
            double2 v = y[zp * nv + f * bc + c];
            pr[f] = make_double2(dn1 * v.x, dn1 * v.y);
        }
        const size_t o = (size_t)j * nc + kr * nxh + i;
        I.VVC[o] = pr[2];
        I.UVF[o] = pr[4];
        I.WVF[o] = pr[5];
        double2 n1 = make_double2(0.0, 0.0), n2 = n1, n3 = n1;
        if (kr != Nz / 2) {  // rows Nz/2+1..Mz-Nz/2+1 are zero in der_x/der_z (kz = -Nz/2)
            const double kx = I.kx[i], kz = I.kz[kr];
            // (i kx) a + (i kz) b with the textbook complex product
            n1 = make_double2(-(kx * pr[0].y) + -(kz * pr[1].y), kx * pr[0].x + kz * pr[1].x);
            n3 = make_double2(-(kx * pr[1].y) + -(kz * pr[3].y), kx * pr[1].x + kz * pr[3].x);
            n2 = make_double2(-(kx * pr[4].y) + -(kz * pr[5].y), kx * pr[4].x + kz * pr[5].x);
        }
        const size_t on = (size_t)(j - 1) * nc + kr * nxh + i;
        I.NXZ1[on] = n1;
        I.NXZ2[on] = n2;
        I.NXZ3[on] = n3;
    }
}

// ---------------------------------------------------------------------------
// Stand-alone plane transforms with the reference's full semantics, for the
// four_to_phys/phys_to_four entry points.  Planes are real (Mx+2) x Mz
// arrays, x fastest, (re, im) pairs for spectral columns.

// z transform of the columns i = 0..Nx/2 of a plane (cft with m = (Nx+2)/2).
// With zero_row (SGN = +1) row Mz/2+1 is zeroed first, as four_to_phys_u
// does (FOU3D.f90:668-670): each CTA reads its own columns of that row as
// zero (its transform then overwrites them), and the first CTA of the plane
// clears the slots beyond the transformed columns, which no CTA writes.
template <int SGN>
__device__ void plane_z(const Inst *__restrict__ insts, double *planes, int bc, int zero_row)
{
    extern __shared__ double2 sm[];
    const Inst &I = insts[0];
    const int Mz = I.Mz, nxh = I.nxh, ig = I.Mx + 2;
    const int nblk = (nxh + bc - 1) / bc;
    const int pl = blockIdx.x / nblk, i0 = (blockIdx.x % nblk) * bc;
    double2 *P = reinterpret_cast<double2 *>(planes + (size_t)pl * ig * Mz);
    const int ig2 = ig / 2;
    double2 *a = sm, *b = sm + Mz * bc;
    const int tot = Mz * bc;
    const int zq = (SGN > 0 && zero_row) ? Mz / 2 : -1;
    if (zq >= 0 && i0 == 0)
        for (int t = nxh + threadIdx.x; t < ig2; t += blockDim.x) P[(size_t)zq * ig2 + t] = make_double2(0.0, 0.0);
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int v = t % bc, q = t / bc, i = i0 + v;
        a[q * bc + v] = (i < nxh && q != zq) ? P[(size_t)q * ig2 + i] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    double2 *r = fft_batch<SGN>(a, b, Mz, I.radz, I.nradz, bc, I.twz);
    const double s = SGN > 0 ? 1.0 : 1.0 / Mz;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int v = t % bc, q = t / bc, i = i0 + v;
        double2 val = r[q * bc + v];
        if (SGN < 0) val = make_double2(s * val.x, s * val.y);
        if (i < nxh) P[(size_t)q * ig2 + i] = val;
    }
}

// zero row Mz/2+1 of every plane (after the forward transform, FOU3D.f90:1670)
__global__ void k_plane_zero_row(const Inst *__restrict__ insts, double *planes)
{
    const Inst &I = insts[0];
    const int ig = I.Mx + 2;
    double *P = planes + (size_t)blockIdx.x * ig * I.Mz + (size_t)(I.Mz / 2) * ig;
    for (int t = threadIdx.x; t < ig; t += blockDim.x) P[t] = 0.0;
}

// x transform of all rows of a plane, two rows per complex FFT.
// SGN=+1: rft inverse (Im of modes 0 and Mx/2 ignored; slots Mx+1, Mx+2 keep
// the input values as the reference's shift loop leaves them).
// SGN=-1: rft forward (all modes 0..Mx/2, scaled 1/Mx, Im(0)=Im(Mx/2)=0).
template <int SGN>
__device__ void plane_x(const Inst *__restrict__ insts, double *planes, int br)
{
    extern __shared__ double2 sm[];
    const Inst &I = insts[0];
    const int Mx = I.Mx, Mz = I.Mz, ig = Mx + 2, h = Mx / 2;
    const int pairs = (Mz + 1) / 2;
    const int nblk = (pairs + br - 1) / br;
    const int pl = blockIdx.x / nblk, p0 = (blockIdx.x % nblk) * br;
    double *P = planes + (size_t)pl * ig * Mz;
    double2 *a = sm, *b = sm + Mx * br;
    const int tot = Mx * br;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int v = t % br, n = t / br;
        const int qa = 2 * (p0 + v), qb = qa + 1;
        double2 z = make_double2(0.0, 0.0);
        if (p0 + v < pairs) {
            const double *A = P + (size_t)qa * ig;
            const double *B = qb < Mz ? P + (size_t)qb * ig : nullptr;
            if (SGN > 0) {
                double ar, ai, brr = 0.0, bi = 0.0;
                int k = n <= h ? n : Mx - n;
                ar = A[2 * k];
                ai = (k == 0 || k == h) ? 0.0 : A[2 * k + 1];
                if (B) {
                    brr = B[2 * k];
                    bi = (k == 0 || k == h) ? 0.0 : B[2 * k + 1];
                }
                if (n <= h) z = make_double2(ar - bi, ai + brr);
                else z = make_double2(ar + bi, brr - ai);
            } else {
                z = make_double2(A[n], B ? B[n] : 0.0);
            }
        }
        a[n * br + v] = z;
    }
    __syncthreads();
    double2 *y = fft_batch<SGN>(a, b, Mx, I.radx, I.nradx, br, I.twx);
    if (SGN > 0) {
        for (int t = threadIdx.x; t < tot; t += blockDim.x) {
            const int v = t % br, n = t / br;
            const int qa = 2 * (p0 + v), qb = qa + 1;
            if (p0 + v >= pairs) continue;
            double2 z = y[n * br + v];
            P[(size_t)qa * ig + n] = z.x;
            if (qb < Mz) P[(size_t)qb * ig + n] = z.y;
        }
    } else {
        const double dn1 = 1.0 / Mx;
        const int tot2 = (h + 1) * br;
        for (int t = threadIdx.x; t < tot2; t += blockDim.x) {
            const int v = t % br, k = t / br;
            const int qa = 2 * (p0 + v), qb = qa + 1;
            if (p0 + v >= pairs) continue;
            const double2 zk = y[k * br + v], zm = y[((Mx - k) % Mx) * br + v];
            double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
            double2 B = make_double2(0.5 * (zk.y + zm.y), 0.5 * (zm.x - zk.x));
            if (k == 0 || k == h) {
                A.y = 0.0;
                B.y = 0.0;
            }
            P[(size_t)qa * ig + 2 * k] = dn1 * A.x;
            P[(size_t)qa * ig + 2 * k + 1] = dn1 * A.y;
            if (qb < Mz) {
                P[(size_t)qb * ig + 2 * k] = dn1 * B.x;
                P[(size_t)qb * ig + 2 * k + 1] = dn1 * B.y;
            }
        }
    }
}

__global__ void k_plane_z_inv(const Inst *__restrict__ insts, double *planes, int bc, int zero_row)
{
    plane_z<+1>(insts, planes, bc, zero_row);
}
__global__ void k_plane_z_fwd(const Inst *__restrict__ insts, double *planes, int bc) { plane_z<-1>(insts, planes, bc, 0); }
__global__ void k_plane_x_inv(const Inst *__restrict__ insts, double *planes, int br) { plane_x<+1>(insts, planes, br); }
__global__ void k_plane_x_fwd(const Inst *__restrict__ insts, double *planes, int br) { plane_x<-1>(insts, planes, br); }

}  // namespace lh
