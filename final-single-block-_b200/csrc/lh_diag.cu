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

#include <vector>

#include "lh_engine.h"
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

// Stats: stats() (stats.f90:1-97) at flagged steps.  nonlinear()
// calls it (FOU3D.f90:307-341) after ops_in_planes2 (FOU3D.f90:240) has run
// four_to_phys_u in place on planes 1..nyu of u1PL, u2PL_itp, u3PL
// (FOU3D.f90:1541) and of u1PL_itp, u2PL, u3PL_itp (FOU3D.f90:1584; v planes
// 1..nyv+1 at one rank).  So the sums of planes 1..nyu run over physical
// values on the dealiased Mx x Mz grid, while the wall planes 0 and nyu+1
// still hold the spectral coefficients modes_to_planes_UVP placed (re, im
// interleaved along x, kz rows mapped into the dealiased plane, zeros
// elsewhere).  The physical sums are evaluated from the spectral
// coefficients (k_stats_parseval), the coefficient sums in the reference's
// order (k_stats_spectral).  Accumulators acc[q][j], j = 0..nyu+1:
//   0 Um 1 U2m (u1)  2 Vm 3 V2m (u2)  4 Wm 5 W2m (u3)
//   6 UVm (u1 x u2 interpolated to u rows)  7 UWm (u1 x u3)
//   8 VWm (u2 x u3 interpolated to v rows)
//   9 Pm 10 P2m (the pressure planes of the latest output step, spectral)
//   11 wxm 12 wx2m (omega_x in physical space on the Nx x Nz grid)
constexpr int kStats = 13;
constexpr int kReduceThreads = 256;

// Spectral sums: rows 0..8 of the wall planes, and the P rows of planes
// 1..nyu from the pressure snapshot (plane nyu+1 of ppPL is empty).  The
// reference adds the entries of a plane in its storage order -- plane rows
// k = 1..Mz, then x entries -- which for the retained modes is column order
// (kz >= 0 rows first, then kz < 0) with re before im; zero entries add
// nothing.  One CTA per plane stages tiles of the plane's coefficients in
// shared memory, then lane 0 of warp q adds the tile into sum q in that
// order with explicitly rounded operations, so the sums match the host
// restatement bit for bit; the chains of different sums run in parallel.
constexpr int kSpecTile = 256;                  // columns per staged tile
constexpr int kSpecThreads = 9 * 32;            // one warp per sum

__global__ void __launch_bounds__(kSpecThreads) k_stats_spectral(const Inst *__restrict__ insts,
                                                                 const double2 *__restrict__ pp,
                                                                 double *__restrict__ acc)
{
    // term[q][2 c + part]: the rounded term entry (c, re/im) adds into sum q
    __shared__ double term[9][2 * kSpecTile];
    const Inst &I = insts[0];
    const int nyu = I.nyu, nyv = I.nyv, npl = nyu + 2, j = blockIdx.x;
    const bool wall = j == 0 || j == nyu + 1;
    if (!wall && !(pp && j >= 1 && j <= nyu)) return;
    const size_t nc = I.nc;
    const bool vrow = j <= nyv + 1;
    const int t = threadIdx.x, q = t >> 5, nq = wall ? 9 : 2, row = (wall ? 0 : 9) + q;
    const bool adder = (t & 31) == 0 && q < nq;
    double s = adder ? acc[row * npl + j] : 0.0;
    for (size_t c0 = 0; c0 < nc; c0 += kSpecTile) {
        const int cnt = (int)(nc - c0 < (size_t)kSpecTile ? nc - c0 : (size_t)kSpecTile);
        for (int c = t; c < cnt; c += kSpecThreads) {
            const size_t col = c0 + c, o = (size_t)j * nc + col;
            if (wall) {
                const double2 a2 = I.U1[o], w2 = I.U3[o];
                const double2 v2 = vrow ? I.U2[o] : make_double2(0.0, 0.0);
                const double2 vi2 = u2_at_u(I, col, j);
                const double2 wi2 = vrow ? u3_at_v(I, col, j) : make_double2(0.0, 0.0);
#pragma unroll
                for (int part = 0; part < 2; part++) {
                    const double a = part ? a2.y : a2.x, v = part ? v2.y : v2.x, w = part ? w2.y : w2.x;
                    const double vi = part ? vi2.y : vi2.x, wi = part ? wi2.y : wi2.x;
                    const int e = 2 * c + part;
                    term[0][e] = a;
                    term[1][e] = __dmul_rn(a, a);
                    term[2][e] = v;
                    term[3][e] = __dmul_rn(v, v);
                    term[4][e] = w;
                    term[5][e] = __dmul_rn(w, w);
                    term[6][e] = __dmul_rn(a, vi);
                    term[7][e] = __dmul_rn(a, w);
                    term[8][e] = __dmul_rn(v, wi);
                }
            } else {
                const double2 p = pp[(size_t)(j - 1) * nc + col];
                term[0][2 * c] = p.x;
                term[1][2 * c] = __dmul_rn(p.x, p.x);
                term[0][2 * c + 1] = p.y;
                term[1][2 * c + 1] = __dmul_rn(p.y, p.y);
            }
        }
        __syncthreads();
        if (adder) {
            const double *T = term[q];
            const int n = 2 * cnt;
#pragma unroll 8
            for (int e = 0; e < n; e++) s = __dadd_rn(s, T[e]);
        }
        __syncthreads();
    }
    if (adder) acc[row * npl + j] = s;
}

// Fixed-order block reduction of NQ sums (blockDim.x = kReduceThreads);
// the totals land in red[q * kReduceThreads].
template <int NQ>
__device__ __forceinline__ void block_sums(double (&s)[NQ], double *red)
{
    const int t = threadIdx.x;
#pragma unroll
    for (int q = 0; q < NQ; q++) red[q * kReduceThreads + t] = s[q];
    __syncthreads();
    for (int h = kReduceThreads / 2; h > 0; h >>= 1) {
        if (t < h) {
#pragma unroll
            for (int q = 0; q < NQ; q++) red[q * kReduceThreads + t] += red[q * kReduceThreads + t + h];
        }
        __syncthreads();
    }
}

// omega_x of planes j0..j0+cnt-1 (0 <= j <= nyu+1) in Nspec-sized planes
// [plane][Nz][Nx+2] (FOU3D.f90:314-336): u2 placed by modes_to_planes_phys
// (dk_phys = 0: row kr, planes 0..nyv+1), der_z_N's (0, kz) * u2 with the
// textbook complex product, der_yv_h_wx's (u3(j+1) - u3(j)) dthdyv(j)
// ddthetavi, then -wx + du3dy; plane nyu+1 is zero.
__global__ void k_wx_scatter(const Inst *__restrict__ insts, double *__restrict__ planes, int j0, int cnt)
{
    const Inst &I = insts[0];
    const int ign = I.Nx + 2, Nz = I.Nz, nxh = I.nxh;
    const size_t nc = I.nc, plane = (size_t)ign * Nz, total = plane * cnt;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t pl = e / plane;
        const int r = (int)(e - pl * plane), kr = r / ign, x = r - kr * ign, i = x >> 1;
        const int j = j0 + (int)pl;
        double val = 0.0;
        if (j <= I.nyv + 1 && i < nxh) {
            const size_t col = (size_t)kr * nxh + i;
            const double2 v = I.U2[(size_t)j * nc + col];
            const double2 a = I.U3[(size_t)(j + 1) * nc + col], b = I.U3[(size_t)j * nc + col];
            const double kz = I.kz[kr], dth = I.dthdyv[j];
            double dz, dy;
            if (x & 1) {
                dz = __dadd_rn(__dmul_rn(0.0, v.y), __dmul_rn(kz, v.x));
                dy = __dmul_rn(__dmul_rn(__dsub_rn(a.y, b.y), dth), I.ddthetavi);
            } else {
                dz = __dsub_rn(__dmul_rn(0.0, v.x), __dmul_rn(kz, v.y));
                dy = __dmul_rn(__dmul_rn(__dsub_rn(a.x, b.x), dth), I.ddthetavi);
            }
            val = __dadd_rn(-dz, dy);
        }
        planes[e] = val;
    }
}

// Physical-grid sums from the spectral coefficients.  four_to_phys_u on a
// dealiased plane gives u(p, q) = Re c_0(q) + sum_{i=1}^{Nx/2} 2 Re(c_i(q)
// e^{2 pi i i p / Mx}) with c_i(q) = sum_kz a(i, kz) e^{2 pi i kz q / Mz} (the
// imaginary part of mode 0 is dropped, rft_buff.f:78-81).  With Mx > Nx and
// Mz > Nz no two retained modes alias on the grid, so for two fields
//   sum_grid a b / (Mx Mz) = Re a(0,0) Re b(0,0)
//       + sum_{0<k<Nz/2} 2 Re(h_a(k) conj h_b(k))  + 1/2 Re(a(0,-Nz/2) conj b(0,-Nz/2))
//       + sum_{i>=1, all kz} 2 Re(a(i,kz) conj b(i,kz)),
//   h(k) = (a(0,k) + conj a(0,-k)) / 2,      sum_grid a / (Mx Mz) = Re a(0,0).
// four_to_phys_N on the Nspec grid keeps the kz = -Nz/2 row, which aliases
// +Nz/2, and the x Nyquist mode i = Nx/2 enters with its real part only:
//   sum_grid w^2 / (Nx Nz) = Q(0) + Q(Nx/2) + sum_{0<i<Nx/2, all kz} 2 |w(i,kz)|^2,
//   Q(i) = (Re w(i,0))^2 + sum_{0<k<Nz/2} 2 |h(k)|^2 + (Re w(i,-Nz/2))^2.
// These are the sums stats() takes over the transformed planes, evaluated
// without transforming them.

// omega_x's spectral coefficient at (col, v row j <= nyv+1): -(0, kz) u2 + du3dy
// in the operation order of der_z_N, der_yv_h_wx and FOU3D.f90:334
__device__ __forceinline__ double2 wx_hat(const Inst &I, size_t col, int kr, int j)
{
    const size_t nc = I.nc;
    const double2 v = I.U2[(size_t)j * nc + col];
    const double2 a = I.U3[(size_t)(j + 1) * nc + col], b = I.U3[(size_t)j * nc + col];
    const double kz = I.kz[kr], dth = I.dthdyv[j];
    const double dzr = __dsub_rn(__dmul_rn(0.0, v.x), __dmul_rn(kz, v.y));
    const double dzi = __dadd_rn(__dmul_rn(0.0, v.y), __dmul_rn(kz, v.x));
    const double dyr = __dmul_rn(__dmul_rn(__dsub_rn(a.x, b.x), dth), I.ddthetavi);
    const double dyi = __dmul_rn(__dmul_rn(__dsub_rn(a.y, b.y), dth), I.ddthetavi);
    return make_double2(__dadd_rn(-dzr, dyr), __dadd_rn(-dzi, dyi));
}

__device__ __forceinline__ double rdot(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ double2 hsym(double2 p, double2 m) { return make_double2(0.5 * (p.x + m.x), 0.5 * (p.y - m.y)); }
__device__ __forceinline__ double2 re_only(double2 a) { return make_double2(a.x, 0.0); }

// How a column enters a grid sum: its weight and whether it is replaced by
// h (paired with its -kz partner) or by its real part; weight 0 skips it.
struct ColRule {
    double wgt;
    bool paired, real;
};
__device__ __forceinline__ ColRule dealiased_rule(int i, int kr, int Nz)
{
    if (i > 0) return {2.0, false, false};
    if (kr == 0) return {1.0, false, true};
    if (kr < Nz / 2) return {2.0, true, false};
    if (kr == Nz / 2) return {0.5, false, false};
    return {0.0, false, false};
}
__device__ __forceinline__ ColRule nspec_rule(int i, int kr, int Nx, int Nz)
{
    if (i > 0 && i < Nx / 2) return {2.0, false, false};
    if (kr == 0 || kr == Nz / 2) return {1.0, false, true};
    if (kr < Nz / 2) return {2.0, true, false};
    return {0.0, false, false};
}

// Stats of planes 1..nyu (velocity rows) and of omega_x on planes 0..nyu+1,
// one CTA per plane j = blockIdx.x, columns reduced in a fixed tree.
__global__ void __launch_bounds__(kReduceThreads) k_stats_parseval(const Inst *__restrict__ insts,
                                                                   double *__restrict__ acc)
{
    __shared__ double red[7 * kReduceThreads];
    const Inst &I = insts[0];
    const int j = blockIdx.x, nyu = I.nyu, npl = nyu + 2, Nx = I.Nx, Nz = I.Nz, nxh = I.nxh;
    const size_t nc = I.nc;
    const bool inner = j >= 1 && j <= nyu, wxp = j <= I.nyv + 1;
    double s[7] = {};
    for (int col = threadIdx.x; col < (int)nc; col += kReduceThreads) {
        const int kr = col / nxh, i = col - kr * nxh;
        if (inner) {
            const ColRule r = dealiased_rule(i, kr, Nz);
            if (r.wgt != 0.0) {
                const size_t o = (size_t)j * nc + col;
                double2 a = I.U1[o], w = I.U3[o], v = I.U2[o];
                double2 vi = u2_at_u(I, col, j), wi = u3_at_v(I, col, j);
                if (r.paired) {
                    const size_t pc = (size_t)(Nz - kr) * nxh, po = (size_t)j * nc + pc;
                    a = hsym(a, I.U1[po]);
                    w = hsym(w, I.U3[po]);
                    v = hsym(v, I.U2[po]);
                    vi = hsym(vi, u2_at_u(I, pc, j));
                    wi = hsym(wi, u3_at_v(I, pc, j));
                } else if (r.real) {
                    a = re_only(a);
                    w = re_only(w);
                    v = re_only(v);
                    vi = re_only(vi);
                    wi = re_only(wi);
                }
                s[0] += r.wgt * rdot(a, a);
                s[1] += r.wgt * rdot(v, v);
                s[2] += r.wgt * rdot(w, w);
                s[3] += r.wgt * rdot(a, vi);
                s[4] += r.wgt * rdot(a, w);
                s[5] += r.wgt * rdot(v, wi);
            }
        }
        if (wxp) {
            const ColRule r = nspec_rule(i, kr, Nx, Nz);
            if (r.wgt != 0.0) {
                double2 x = wx_hat(I, col, kr, j);
                if (r.paired) x = hsym(x, wx_hat(I, (size_t)(Nz - kr) * nxh + i, Nz - kr, j));
                else if (r.real) x = re_only(x);
                s[6] += r.wgt * rdot(x, x);
            }
        }
    }
    block_sums<7>(s, red);
    if (threadIdx.x == 0) {
        const double n = (double)I.Mx * I.Mz, nn = (double)Nx * Nz;
        if (inner) {
            const size_t o = (size_t)j * nc;
            acc[0 * npl + j] += n * I.U1[o].x;
            acc[1 * npl + j] += n * red[0 * kReduceThreads];
            acc[2 * npl + j] += n * I.U2[o].x;
            acc[3 * npl + j] += n * red[1 * kReduceThreads];
            acc[4 * npl + j] += n * I.U3[o].x;
            acc[5 * npl + j] += n * red[2 * kReduceThreads];
            acc[6 * npl + j] += n * red[3 * kReduceThreads];
            acc[7 * npl + j] += n * red[4 * kReduceThreads];
            acc[8 * npl + j] += n * red[5 * kReduceThreads];
        }
        if (wxp) {
            acc[11 * npl + j] += nn * wx_hat(I, 0, 0, j).x;
            acc[12 * npl + j] += nn * red[6 * kReduceThreads];
        }
    }
}

size_t stats_doubles(int nyu) { return kStats * (size_t)(nyu + 2); }

namespace {
constexpr int kPlaneCols = 4, kPlaneRows = 4, kPlaneThreads = 256;
constexpr size_t kStatsBudget = 256u << 20;  // omega_x scratch bytes per pass

struct PlaneShape {
    unsigned nbz, nbx;
    size_t smz, smx;
};
PlaneShape plane_shape(int Mx, int Mz, int nxh)
{
    PlaneShape p;
    p.nbz = (unsigned)((nxh + kPlaneCols - 1) / kPlaneCols);
    p.nbx = (unsigned)(((Mz + 1) / 2 + kPlaneRows - 1) / kPlaneRows);
    p.smz = 2 * (size_t)Mz * kPlaneCols * sizeof(double2);
    p.smx = 2 * (size_t)Mx * kPlaneRows * sizeof(double2);
    return p;
}

unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

// inverse z then x transforms of nplanes planes (four_to_phys_u with the
// row zeroed, four_to_phys_N without)
cudaError_t planes_to_phys(const Inst *d_inst, const PlaneShape &p, double *planes, int nplanes, int zero_row,
                           cudaStream_t st)
{
    cudaError_t e = raise_smem_limit((const void *)k_plane_z_inv, p.smz);
    if (e == cudaSuccess) e = raise_smem_limit((const void *)k_plane_x_inv, p.smx);
    if (e != cudaSuccess) return e;
    k_plane_z_inv<<<nplanes * p.nbz, kPlaneThreads, p.smz, st>>>(d_inst, planes, kPlaneCols, zero_row);
    k_plane_x_inv<<<nplanes * p.nbx, kPlaneThreads, p.smx, st>>>(d_inst, planes, kPlaneRows);
    return cudaGetLastError();
}
}  // namespace

cudaError_t stats_prepare(const DevInstance &d, StatsScratch &s)
{
    if (s.planes) return cudaSuccess;
    const HostSetup &hs = d.hs;
    std::vector<int> rz, rx;
    std::vector<double> tz, tx;
    if (!cft_radices(hs.Nz, rz) || !rft_radices(hs.Nx, rx) || rz.size() > (size_t)kMaxRad ||
        rx.size() > (size_t)kMaxRad)
        return cudaErrorInvalidValue;
    cft_table(hs.Nz, tz);
    rft_table(hs.Nx, tx);
    const size_t per_n = (size_t)(hs.Nx + 2) * hs.Nz * sizeof(double);
    s.chunk_n = (int)std::max<size_t>(1, std::min<size_t>(hs.nyu + 2, kStatsBudget / per_n));
    s.bytes = per_n * s.chunk_n;
    cudaError_t e = cudaMalloc(&s.planes, s.bytes);
    if (e == cudaSuccess) e = cudaMalloc(&s.tw_n, (size_t)(hs.Nz + hs.Nx) * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&s.d_inst_n, sizeof(Inst));
    if (e == cudaSuccess) e = cudaMemcpy(s.tw_n, tz.data(), tz.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(s.tw_n + hs.Nz, tx.data(), tx.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        // the instance record with the transform sizes of the Nspec grid
        Inst n = d.inst;
        n.Mx = hs.Nx;
        n.Mz = hs.Nz;
        n.nradz = (int)rz.size();
        n.nradx = (int)rx.size();
        for (int k = 0; k < n.nradz; k++) n.radz[k] = rz[k];
        for (int k = 0; k < n.nradx; k++) n.radx[k] = rx[k];
        n.twz = s.tw_n;
        n.twx = s.tw_n + hs.Nz;
        e = cudaMemcpy(s.d_inst_n, &n, sizeof(Inst), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        double2 *pp = s.pp;
        s.pp = nullptr;
        stats_release(s);
        s.pp = pp;
    }
    return e;
}

void stats_release(StatsScratch &s)
{
    if (s.planes) cudaFree(s.planes);
    if (s.tw_n) cudaFree(s.tw_n);
    if (s.d_inst_n) cudaFree(s.d_inst_n);
    if (s.pp) cudaFree(s.pp);
    s = StatsScratch();
}

cudaError_t launch_stats_accumulate(const Inst *d_inst, const HostSetup &hs, const double2 *pp, double *acc,
                                    cudaStream_t st)
{
    const int npl = hs.nyu + 2;
    k_stats_spectral<<<npl, kSpecThreads, 0, st>>>(d_inst, pp, acc);
    k_stats_parseval<<<npl, kReduceThreads, 0, st>>>(d_inst, acc);
    return cudaGetLastError();
}

cudaError_t omega_x_planes(const Inst *d_inst, const HostSetup &hs, const StatsScratch &s, double *out,
                           cudaStream_t st)
{
    const PlaneShape pn = plane_shape(hs.Nx, hs.Nz, hs.nxh);
    const size_t plane_n = (size_t)(hs.Nx + 2) * hs.Nz;
    cudaError_t e = cudaSuccess;
    for (int j0 = 0; e == cudaSuccess && j0 <= hs.nyu + 1; j0 += s.chunk_n) {
        const int cnt = std::min(s.chunk_n, hs.nyu + 2 - j0);
        k_wx_scatter<<<grid_for(plane_n * cnt), 256, 0, st>>>(d_inst, s.planes, j0, cnt);
        e = planes_to_phys(s.d_inst_n, pn, s.planes, cnt, 0, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out + plane_n * j0, s.planes, plane_n * cnt * sizeof(double), cudaMemcpyDeviceToHost,
                                st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    return e;
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
