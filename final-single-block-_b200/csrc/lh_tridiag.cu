// Tridiagonal factor / solve entries of the C ABI and the scalar set-up of
// a continued run.
//
// The reference keeps its tridiagonal matrices in a(3, j[, column]) arrays
// (tridLU_3D.f90): LU_build / LU_buildP fill a(1,j) lower, a(2,j) main and
// a(3,j) upper diagonal; LU_dec / LU_decP overwrite a(2,j) with the inverse
// pivot and a(3,j) with the scaled upper diagonal, a(1,j) stays the lower
// diagonal of L.  These entries give a caller those factors (computed on the
// device with the reference's operation order), solve with factors the
// caller holds, and install a caller's pressure factors DG as the engine's.
// Compiled without FMA contraction, like the column pass, so every factor
// rounds as the reference's does.
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "lh_engine.h"
#include "lh_gpu.h"
#include "lh_kernels.cuh"

using namespace lh;

#include "lh_ctx_internal.h"

namespace {

int fail(lh_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

int cuda_fail(lh_ctx *c, cudaError_t e, const char *where)
{
    return fail(c, e == cudaErrorMemoryAllocation ? LH_ENOMEM : LH_ECUDA,
                std::string(where) + ": " + cudaGetErrorString(e));
}

// Rows of a grid: 2 = ugrid (0..nyu+1), 1 = vgrid (0..nyv+1), 3 = pgrid
// (1..nyu) -- the reference's jlim(1:2, grid) (start.f90:909-1070).
int grid_rows(const HostSetup &s, int grid)
{
    return grid == 2 ? s.nyu + 2 : grid == 1 ? s.nyv + 2 : grid == 3 ? s.nyu : 0;
}

// LU_build (tridLU_3D.f90:163-221) and LU_dec (:327-364) of every column of
// one velocity grid, written as a(3, j, column) with j from jlim(1, grid).
__global__ void k_lu_factor(const Inst *__restrict__ insts, int grid, double beta, double *__restrict__ a)
{
    const Inst &I = insts[0];
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= I.nc) return;
    const int i = col % I.nxh, kr = col / I.nxh;
    const double k2x = I.k2x[i], k2z = I.k2z[kr];
    const bool u = grid == 2;
    const int n = u ? I.nyu : I.nyv;  // interior rows 1..n, walls 0 and n+1
    const double *d = u ? I.dyu2i : I.dyv2i;
    double *A = a + (size_t)col * 3 * (n + 2);
    // LU_build: wall rows [0, 1, gw(1)] / [gw(2), 1, 0] on the u grid,
    // identity rows on the v grid
    A[0] = 0.0;
    A[1] = 1.0;
    A[2] = u ? I.gw1 : 0.0;
    for (int j = 1; j <= n; j++) {
        A[3 * j] = -beta * d[3 * j];
        A[3 * j + 1] = 1.0 - beta * (d[3 * j + 1] + k2x + k2z);
        A[3 * j + 2] = -beta * d[3 * j + 2];
    }
    A[3 * (n + 1)] = u ? I.gw2 : 0.0;
    A[3 * (n + 1) + 1] = 1.0;
    A[3 * (n + 1) + 2] = 0.0;
    // LU_dec
    A[1] = 1.0 / A[1];
    for (int j = 1; j <= n + 1; j++) {
        A[3 * (j - 1) + 2] = A[3 * (j - 1) + 2] * A[3 * (j - 1) + 1];
        A[3 * j + 1] = 1.0 / (A[3 * j + 1] - A[3 * j] * A[3 * (j - 1) + 2]);
    }
}

// The solve of LUsolU / LUsolP with given factors (tridLU_3D.f90:70-82,
// 115-128): x(j0) *= a(2,j0); x(j) = (x(j) - a(1,j) x(j-1)) a(2,j);
// x(j) -= a(3,j) x(j+1).  Column layout x(j, column), j fastest.
__global__ void k_lu_solve(int nc, int rows, const double *__restrict__ a, double2 *__restrict__ x)
{
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= nc) return;
    const double *A = a + (size_t)col * 3 * rows;
    double2 *X = x + (size_t)col * rows;
    double2 y = X[0];
    y = make_double2(y.x * A[1], y.y * A[1]);
    X[0] = y;
    for (int j = 1; j < rows; j++) {
        const double2 r = X[j];
        const double l = A[3 * j], iv = A[3 * j + 1];
        y = make_double2((r.x - l * y.x) * iv, (r.y - l * y.y) * iv);
        X[j] = y;
    }
    for (int j = rows - 2; j >= 0; j--) {
        const double2 r = X[j];
        const double f = A[3 * j + 2];
        y = make_double2(r.x - f * y.x, r.y - f * y.y);
        X[j] = y;
    }
}

// DG in the reference's a(3, j, column) layout (j = 1..nyu) from the
// engine's split storage: DG1[j] the column-independent lower diagonal
// (LU_buildP's a(1,j) = D_vec_b(j-1) G_vec_b(j-1), tridLU_3D.f90:260-266;
// zero at j = 1, where the reference never sets it), DG2 the inverse pivots,
// DG3 the scaled upper diagonals.
void dg_to_ref(const HostSetup &s, double *a)
{
    const int n = s.nyu, nc = s.nc;
    for (int col = 0; col < nc; col++)
        for (int j = 1; j <= n; j++) {
            double *A = a + ((size_t)col * n + (j - 1)) * 3;
            A[0] = j >= 2 ? s.DG1[j] : 0.0;
            A[1] = s.DG2[(size_t)(j - 1) * nc + col];
            A[2] = s.DG3[(size_t)(j - 1) * nc + col];
        }
}

}  // namespace

extern "C" int lh_tridiag_factor(lh_ctx *c, int grid, int kRK, double dt, double *a, size_t cap)
{
    if (!c) return LH_EINVAL;
    const HostSetup &s = c->dev.hs;
    const int rows = grid_rows(s, grid);
    if (!rows) return fail(c, LH_EINVAL, "grid must be 1 (v), 2 (u/w) or 3 (p)");
    if (grid != 3 && (kRK < 1 || kRK > 3)) return fail(c, LH_EINVAL, "kRK must be 1, 2 or 3");
    const size_t n = (size_t)3 * rows * s.nc;
    if (!a) return (int)n;
    if (cap < n) return fail(c, LH_EINVAL, "factor buffer too small");
    if (grid == 3) {
        dg_to_ref(s, a);
        return (int)n;
    }
    // beta = bRK(kRK) dt / Re (LU_build, tridLU_3D.f90:174); bRK = aRK
    const double bRK = kRK == 1 ? 4.0 / 15.0 : kRK == 2 ? 1.0 / 15.0 : 1.0 / 6.0;
    const double beta = bRK * dt / c->dev.desc.Re;
    double *d = nullptr;
    cudaError_t e = cudaMalloc(&d, n * sizeof(double));
    if (e != cudaSuccess) return cuda_fail(c, e, "tridiag_factor alloc");
    k_lu_factor<<<(s.nc + 127) / 128, 128, 0, c->st>>>(c->d_inst, grid, beta, d);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(a, d, n * sizeof(double), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(c, e, "tridiag_factor");
    return (int)n;
}

extern "C" int lh_tridiag_solve(lh_ctx *c, int grid, const double *a, double *x)
{
    if (!c || !a || !x) return fail(c, LH_EINVAL, "bad tridiag_solve arguments");
    const HostSetup &s = c->dev.hs;
    const int rows = grid_rows(s, grid);
    if (!rows) return fail(c, LH_EINVAL, "grid must be 1 (v), 2 (u/w) or 3 (p)");
    const size_t na = (size_t)3 * rows * s.nc, nx = (size_t)rows * s.nc;
    double *d_a = nullptr;
    double2 *d_x = nullptr;
    cudaError_t e = cudaMalloc(&d_a, na * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_x, nx * sizeof(double2));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_a, a, na * sizeof(double), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_x, x, nx * sizeof(double2), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) {
        k_lu_solve<<<(s.nc + 127) / 128, 128, 0, c->st>>>(s.nc, rows, d_a, d_x);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(x, d_x, nx * sizeof(double2), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(d_a);
    cudaFree(d_x);
    if (e != cudaSuccess) return cuda_fail(c, e, "tridiag_solve");
    return LH_OK;
}

extern "C" int lh_set_dg(lh_ctx *c, const double *a)
{
    if (!c || !a) return fail(c, LH_EINVAL, "bad set_dg arguments");
    HostSetup &s = c->dev.hs;
    const int n = s.nyu, nc = s.nc;
    // the engine keeps one lower diagonal for all columns, as LU_buildP forms it
    for (int col = 0; col < nc; col++)
        for (int j = 2; j <= n; j++)
            if (a[((size_t)col * n + (j - 1)) * 3] != a[(size_t)(j - 1) * 3])
                return fail(c, LH_EINVAL, "DG lower diagonal differs between columns (not LU_buildP's form)");
    std::vector<double> dg1(s.DG1.size(), 0.0), dg2(s.DG2.size()), dg3(s.DG3.size());
    for (int j = 2; j <= n; j++) dg1[j] = a[(size_t)(j - 1) * 3];
    for (int col = 0; col < nc; col++)
        for (int j = 1; j <= n; j++) {
            const double *A = a + ((size_t)col * n + (j - 1)) * 3;
            dg2[(size_t)(j - 1) * nc + col] = A[1];
            dg3[(size_t)(j - 1) * nc + col] = A[2];
        }
    const Inst &I = c->dev.inst;
    cudaError_t e = cudaMemcpyAsync(const_cast<double *>(I.DG1), dg1.data(), dg1.size() * 8, cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(const_cast<double *>(I.DG2), dg2.data(), dg2.size() * 8, cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(const_cast<double *>(I.DG3), dg3.data(), dg3.size() * 8, cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return cuda_fail(c, e, "set_dg");
    s.DG1.swap(dg1);
    s.DG2.swap(dg2);
    s.DG3.swap(dg3);
    return LH_OK;
}

extern "C" int lh_set_scalars(lh_ctx *c, double t, int iter, double mpgx)
{
    if (!c) return LH_EINVAL;
    if (!c->have_state) return fail(c, LH_ESTATE, "no state uploaded");
    if (iter < 0) return fail(c, LH_EINVAL, "iter < 0");
    const Inst &I = c->dev.inst;
    const double v[3] = {t, mpgx, (double)iter};
    cudaError_t e = cudaMemcpyAsync(I.sc + SC_T, &v[0], sizeof(double), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(I.sc + SC_MPGX, &v[1], sizeof(double), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(I.sc + SC_ITER, &v[2], sizeof(double), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return cuda_fail(c, e, "set_scalars");
    return LH_OK;
}
