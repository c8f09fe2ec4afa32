// On-device diagnostics of flagged steps.
//
// Spectra: spectra() (spectra.f90:7-66), which the reference accumulates
// inside nonlinear() every nstat steps at kRK = 1 (FOU3D.f90:76-81, 137-141):
//
//   spU(j,col)  += Re(u1)^2 + Im(u1)^2      rows 0..nyu+1   (buildsp, ugrid)
//   spV(j,col)  += Re(u2)^2 + Im(u2)^2      rows 0..nyv+1   (vgrid)
//   spW(j,col)  += Re(u3)^2 + Im(u3)^2      rows 0..nyu+1
//   spUV(j,col) += Re(u1) Re(u2i) + Im(u1) Im(u2i), u2i = interp_v(u2)
//                                           rows 0..nyu+1   (buildspUV)
//   spP(j,col)  += Re(p)^2 + Im(p)^2        rows 1..nyu     (pgrid)
//
// The accumulators stay on the device in the plane-major layout of the
// state (row j, then column); one thread per (row, column) adds the current
// state's terms, in the reference's operation order with explicitly rounded
// multiplies and adds (no fused multiply-add), so the sums match the host
// restatement bit for bit on the same state.
#include <algorithm>

#include "lh_kernels.cuh"

namespace lh {

__device__ __forceinline__ double sq_add(double s, double2 a)
{
    return __dadd_rn(__dadd_rn(s, __dmul_rn(a.x, a.x)), __dmul_rn(a.y, a.y));
}

// interp_v (FOU3D.f90:394-418) of column col at u row j
__device__ __forceinline__ double2 u2_at_u(const Inst &I, size_t col, int j)
{
    const size_t nc = I.nc;
    auto inner = [&](int jj) {
        const double2 a = I.U2[(size_t)jj * nc + col], b = I.U2[(size_t)(jj - 1) * nc + col];
        const double w1 = I.yu[jj] - I.yv[jj - 1], w2 = I.yv[jj] - I.yu[jj], d = I.yv[jj] - I.yv[jj - 1];
        return make_double2(__ddiv_rn(__dadd_rn(__dmul_rn(w1, a.x), __dmul_rn(w2, b.x)), d),
                            __ddiv_rn(__dadd_rn(__dmul_rn(w1, a.y), __dmul_rn(w2, b.y)), d));
    };
    if (j >= 1 && j <= I.nyu) return inner(j);
    if (j == 0) {
        const double2 o1 = inner(1), v0 = I.U2[col];
        return make_double2(__dadd_rn(__dmul_rn(I.gwi1, __dsub_rn(v0.x, o1.x)), o1.x),
                            __dadd_rn(__dmul_rn(I.gwi1, __dsub_rn(v0.y, o1.y)), o1.y));
    }
    const double2 o1 = inner(I.nyu), vt = I.U2[(size_t)(I.nyv + 1) * nc + col];
    return make_double2(__dadd_rn(__dmul_rn(I.gwi2, __dsub_rn(vt.x, o1.x)), o1.x),
                        __dadd_rn(__dmul_rn(I.gwi2, __dsub_rn(vt.y, o1.y)), o1.y));
}

__global__ void k_spectra_accumulate(const Inst *__restrict__ insts, double *__restrict__ sp)
{
    const Inst &I = insts[0];
    const size_t nc = I.nc, nu = (size_t)(I.nyu + 2) * nc, nv = (size_t)(I.nyv + 2) * nc;
    double *spU = sp, *spV = spU + nu, *spW = spV + nv, *spUV = spW + nu, *spP = spUV + nu;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nu; e += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / nc);
        const size_t col = e - (size_t)j * nc;
        const double2 u1 = I.U1[e], u3 = I.U3[e];
        spU[e] = sq_add(spU[e], u1);
        spW[e] = sq_add(spW[e], u3);
        const double2 v = u2_at_u(I, col, j);
        spUV[e] = __dadd_rn(__dadd_rn(spUV[e], __dmul_rn(u1.x, v.x)), __dmul_rn(u1.y, v.y));
        if (e < nv) spV[e] = sq_add(spV[e], I.U2[e]);
        if (j >= 1 && j <= I.nyu) {
            const size_t o = e - nc;  // p row j is stored at index j-1
            spP[o] = sq_add(spP[o], I.P[o]);
        }
    }
}

// interp_u (FOU3D.f90:373-392) of column col at v row j
__device__ __forceinline__ double2 u3_at_v(const Inst &I, size_t col, int j)
{
    const size_t nc = I.nc;
    const double2 a = I.U3[(size_t)(j + 1) * nc + col], b = I.U3[(size_t)j * nc + col];
    const double w1 = I.yv[j] - I.yu[j], w2 = I.yu[j + 1] - I.yv[j], d = I.yu[j + 1] - I.yu[j];
    return make_double2(__ddiv_rn(__dadd_rn(__dmul_rn(w1, a.x), __dmul_rn(w2, b.x)), d),
                        __ddiv_rn(__dadd_rn(__dmul_rn(w1, a.y), __dmul_rn(w2, b.y)), d));
}

// Stats: stats() (stats.f90:1-97) at flagged output steps.  When nonlinear()
// calls it (FOU3D.f90:300-341) the plane arrays still hold the spectral
// coefficients that modes_to_planes_UVP placed (re, im interleaved along
// x, kz rows mapped into the dealiased plane, zeros elsewhere), so each
// plane sum runs over those coefficients: plane rows k = 1..Mz, then
// entries i = 1..Mx.  One thread per plane j = 0..nyu+1 adds, in that order,
// every entry's terms into the nine sums (zero entries add nothing):
//   Um U2m (u1)  Vm V2m (u2, planes > nyv+1 empty)  Wm W2m (u3)
//   UVm (u1 x u2 interpolated to u rows)  UWm (u1 x u3)
//   VWm (u2 x u3 interpolated to v rows)
__global__ void k_stats_accumulate(const Inst *__restrict__ insts, double *__restrict__ acc)
{
    const Inst &I = insts[0];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int nyu = I.nyu, nyv = I.nyv, npl = nyu + 2;
    if (j >= npl) return;
    const int Mz = I.Mz, Nz = I.Nz, nxh = I.nxh;
    const size_t nc = I.nc;
    const bool vrow = j <= nyv + 1;
    double s[9];
#pragma unroll
    for (int q = 0; q < 9; q++) s[q] = acc[q * npl + j];
    for (int k = 1; k <= Mz; k++) {
        int kr;
        if (k <= Nz / 2) kr = k - 1;
        else if (k >= Mz - Nz / 2 + 1) kr = k - 1 - (Mz - Nz);
        else continue;  // rows between the retained kz modes are zero
        for (int i = 0; i < nxh; i++) {
            const size_t col = (size_t)kr * nxh + i;
            const double2 a = I.U1[(size_t)j * nc + col], w = I.U3[(size_t)j * nc + col];
            const double2 v = vrow ? I.U2[(size_t)j * nc + col] : make_double2(0.0, 0.0);
            const double2 vi = u2_at_u(I, col, j);
            const double2 wi = vrow ? u3_at_v(I, col, j) : make_double2(0.0, 0.0);
            // the re entry, then the im entry
#pragma unroll
            for (int part = 0; part < 2; part++) {
                const double av = part ? a.y : a.x, vv = part ? v.y : v.x, wv = part ? w.y : w.x;
                const double viv = part ? vi.y : vi.x, wiv = part ? wi.y : wi.x;
                s[0] = __dadd_rn(s[0], av);
                s[1] = __dadd_rn(s[1], __dmul_rn(av, av));
                s[2] = __dadd_rn(s[2], vv);
                s[3] = __dadd_rn(s[3], __dmul_rn(vv, vv));
                s[4] = __dadd_rn(s[4], wv);
                s[5] = __dadd_rn(s[5], __dmul_rn(wv, wv));
                s[6] = __dadd_rn(s[6], __dmul_rn(av, viv));
                s[7] = __dadd_rn(s[7], __dmul_rn(av, wv));
                s[8] = __dadd_rn(s[8], __dmul_rn(vv, wiv));
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 9; q++) acc[q * npl + j] = s[q];
}

size_t stats_doubles(int nyu) { return 9 * (size_t)(nyu + 2); }

void launch_stats_accumulate(const Inst *d_inst, double *acc, int nyu, cudaStream_t st)
{
    k_stats_accumulate<<<(nyu + 2 + 63) / 64, 64, 0, st>>>(d_inst, acc);
}

size_t spectra_doubles(int nyu, int nyv, int nc)
{
    return (size_t)nc * (3 * (size_t)(nyu + 2) + (size_t)(nyv + 2) + (size_t)nyu);
}

void launch_spectra_accumulate(const Inst *d_inst, double *sp, int nyu, int nc, cudaStream_t st)
{
    const size_t n = (size_t)(nyu + 2) * nc;
    const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
    k_spectra_accumulate<<<blocks, 256, 0, st>>>(d_inst, sp);
}

}  // namespace lh
