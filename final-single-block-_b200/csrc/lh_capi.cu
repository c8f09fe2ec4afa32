// C ABI of the single-instance engine (include/lh_gpu.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "lh_engine.h"
#include "lh_gpu.h"
#include "lh_kernels.cuh"

using namespace lh;

#include "lh_ctx_internal.h"

static int fail(lh_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

static int cuda_fail(lh_ctx *c, cudaError_t e, const char *where)
{
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    return fail(c, e == cudaErrorMemoryAllocation ? LH_ENOMEM : LH_ECUDA, m);
}

#define CK(call, where)                                   \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, where); \
    } while (0)

extern "C" int lh_ctx_create(const lh_grid_desc *desc, lh_ctx **out)
{
    if (!desc || !out) return LH_EINVAL;
    *out = nullptr;
    lh_ctx *c = new (std::nothrow) lh_ctx();
    if (!c) return LH_ENOMEM;
    c->dev.desc = *desc;
    std::string why = build_setup(*desc, c->dev.hs);
    if (!why.empty()) {
        delete c;
        return LH_EINVAL;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        delete c;
        return LH_ECUDA;
    }
    cudaError_t e = cudaGetDevice(&c->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return LH_ECUDA;
    }
    const HostSetup &s = c->dev.hs;
    Tiles t = default_tiles(s.Mx, s.Mz, s.nxh, s.nyu);
    const char *gen = getenv("LH_GENERIC_FFT");
    e = instance_alloc(c->dev, t.chunk, c->st);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_inst, sizeof(Inst));
    if (e == cudaSuccess) e = cudaMemcpy(c->d_inst, &c->dev.inst, sizeof(Inst), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = plan_build(c->plan, {&c->dev}, gen && gen[0] == '1');
    if (e != cudaSuccess) {
        int code = e == cudaErrorMemoryAllocation ? LH_ENOMEM : LH_ECUDA;
        lh_ctx_destroy(c);
        return code;
    }
    *out = c;
    return LH_OK;
}

extern "C" int lh_ctx_destroy(lh_ctx *c)
{
    if (!c) return LH_OK;
    ctx_drop_graphs(c);
    if (c->ev_u) cudaEventDestroy(c->ev_u);
    if (c->ev_p) cudaEventDestroy(c->ev_p);
    if (c->st_up) cudaStreamDestroy(c->st_up);
    plan_free(c->plan);
    if (c->d_inst) cudaFree(c->d_inst);
    if (c->d_spec) cudaFree(c->d_spec);
    if (c->d_stats) cudaFree(c->d_stats);
    stats_release(c->stats_scr);
    instance_free(c->dev);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
    return LH_OK;
}

extern "C" const char *lh_last_error(const lh_ctx *c) { return c ? c->err.c_str() : "null context"; }

extern "C" int lh_get_sizes(const lh_ctx *c, lh_sizes *o)
{
    if (!c || !o) return LH_EINVAL;
    const HostSetup &s = c->dev.hs;
    o->Nx = s.Nx;
    o->Nz = s.Nz;
    o->Mx = s.Mx;
    o->Mz = s.Mz;
    o->nyu = s.nyu;
    o->nyv = s.nyv;
    o->ncols = s.nc;
    o->igal = s.Mx + 2;
    o->kgal = s.Mz;
    return LH_OK;
}

extern "C" int lh_get_grid(const lh_ctx *c, int which, double *out, int cap)
{
    if (!c) return LH_EINVAL;
    const HostSetup &s = c->dev.hs;
    const std::vector<double> *v = which == 0 ? &s.yu : which == 1 ? &s.yv : which == 2 ? &s.dthdyu
                                   : which == 3 ? &s.dthdyv : nullptr;
    if (!v) return LH_EINVAL;
    if (out && cap >= (int)v->size()) memcpy(out, v->data(), v->size() * sizeof(double));
    return (int)v->size();
}

extern "C" int lh_host_grid(const lh_grid_desc *desc, int which, double *out, int cap)
{
    if (!desc) return LH_EINVAL;
    HostSetup s;
    if (!build_setup(*desc, s).empty()) return LH_EINVAL;
    std::vector<double> sc = {s.gw1, s.gw2, s.gwbc, s.gwi1, s.gwi2, s.dtv};
    const std::vector<double> *v = which == 0 ? &s.yu : which == 1 ? &s.yv : which == 2 ? &s.dthdyu
                                   : which == 3 ? &s.dthdyv : which == 4 ? &sc : nullptr;
    if (!v) return LH_EINVAL;
    if (out && cap >= (int)v->size()) memcpy(out, v->data(), v->size() * sizeof(double));
    return (int)v->size();
}

extern "C" int lh_upload_state(lh_ctx *c, const double *u1, const double *u2, const double *u3, const double *p)
{
    if (!c || !u1 || !u2 || !u3) return fail(c, LH_EINVAL, "u1, u2 and u3 are required");
    CK(instance_upload(c->dev, u1, u2, u3, p, c->st), "upload");
    c->have_state = true;
    return LH_OK;
}

extern "C" int lh_download_state(lh_ctx *c, double *u1, double *u2, double *u3, double *p)
{
    if (!c) return LH_EINVAL;
    if (!c->have_state) return fail(c, LH_ESTATE, "no state uploaded");
    CK(instance_download(c->dev, u1, u2, u3, p, c->st), "download");
    return LH_OK;
}

extern "C" int lh_download_nu(lh_ctx *c, double *nu1, double *nu2, double *nu3)
{
    if (!c) return LH_EINVAL;
    const HostSetup &s = c->dev.hs;
    if (nu1) CK(download_field(c->dev, c->dev.inst.NU1, s.nyu, nu1, c->st), "download");
    if (nu2) CK(download_field(c->dev, c->dev.inst.NU2, s.nyv, nu2, c->st), "download");
    if (nu3) CK(download_field(c->dev, c->dev.inst.NU3, s.nyu, nu3, c->st), "download");
    CK(cudaStreamSynchronize(c->st), "download");
    return LH_OK;
}

static int check_err_word(lh_ctx *c)
{
    int h = 0;
    CK(cudaMemcpyAsync(&h, c->dev.inst.err, sizeof(int), cudaMemcpyDeviceToHost, c->st), "error word");
    CK(cudaStreamSynchronize(c->st), "synchronize");
    if (h & ERR_NONFINITE) return fail(c, LH_EDEVICE, "non-finite values in the state (time step unstable?)");
    return LH_OK;
}

extern "C" int lh_substep(lh_ctx *c, int kRK)
{
    if (!c) return LH_EINVAL;
    if (kRK < 1 || kRK > 3) return fail(c, LH_EINVAL, "kRK must be 1, 2 or 3");
    if (!c->have_state) return fail(c, LH_ESTATE, "no state uploaded");
    CK(launch_substep(c->plan, c->d_inst, kRK, c->dev.desc.dt_mode == LH_DT_CFL, c->st), "substep launch");
    return LH_OK;
}

// Capture one RK3 step; with wait_p (lh_step_host's first step) the first
// column pass waits for ev_p, the end of the p upload.
static int capture_step(lh_ctx *c, cudaEvent_t wait_p, cudaGraph_t *graph, cudaGraphExec_t *gexec)
{
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal), "graph capture");
    cudaError_t el = cudaSuccess;
    for (int k = 1; k <= 3 && el == cudaSuccess; k++)
        el = launch_substep(c->plan, c->d_inst, k, c->dev.desc.dt_mode == LH_DT_CFL, c->st, nullptr,
                            k == 1 ? wait_p : nullptr);
    cudaGraph_t g = nullptr;
    cudaError_t ee = cudaStreamEndCapture(c->st, &g);
    if (el != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_fail(c, el, "graph capture launch");
    }
    if (ee != cudaSuccess) return cuda_fail(c, ee, "graph capture end");
    *graph = g;
    CK(cudaGraphInstantiate(gexec, g, 0), "graph instantiate");
    return LH_OK;
}

static int ensure_graph(lh_ctx *c)
{
    if (c->gexec) return LH_OK;
    return capture_step(c, nullptr, &c->graph, &c->gexec);
}

extern "C" int lh_step(lh_ctx *c, int nsteps)
{
    if (!c) return LH_EINVAL;
    if (nsteps < 0) return fail(c, LH_EINVAL, "nsteps < 0");
    if (!c->have_state) return fail(c, LH_ESTATE, "no state uploaded");
    int rc = ensure_graph(c);
    if (rc) return rc;
    for (int s = 0; s < nsteps; s++) CK(cudaGraphLaunch(c->gexec, c->st), "graph launch");
    return LH_OK;
}

// Upload, nsteps steps, download.  u1, u2 and u3 upload first on st_up; p
// follows on st_up while the first substep's plane pass (which does not read
// p) runs on st, and the first column pass waits for it; the PCIe transfer
// of p is then hidden behind the plane pass.  Same operations and results as
// lh_upload_state + lh_step + lh_download_state.
extern "C" int lh_step_host(lh_ctx *c, double *u1, double *u2, double *u3, double *p, int nsteps)
{
    if (!c || !u1 || !u2 || !u3) return fail(c, LH_EINVAL, "u1, u2 and u3 are required");
    if (nsteps < 0) return fail(c, LH_EINVAL, "nsteps < 0");
    if (!c->st_up) {
        CK(cudaStreamCreateWithFlags(&c->st_up, cudaStreamNonBlocking), "upload stream");
        CK(cudaEventCreateWithFlags(&c->ev_u, cudaEventDisableTiming), "upload event");
        CK(cudaEventCreateWithFlags(&c->ev_p, cudaEventDisableTiming), "upload event");
    }
    // the upload reuses the staging field the previous call's download used
    CK(cudaStreamSynchronize(c->st), "synchronize");
    CK(instance_upload_p_last(c->dev, u1, u2, u3, p, c->st_up, c->ev_u), "upload");
    CK(cudaEventRecord(c->ev_p, c->st_up), "upload");
    c->have_state = true;
    CK(cudaStreamWaitEvent(c->st, c->ev_u, 0), "upload wait");
    if (nsteps == 0) {
        CK(cudaStreamWaitEvent(c->st, c->ev_p, 0), "upload wait");
    } else {
        int rc = LH_OK;
        if (!c->gexec_host) rc = capture_step(c, c->ev_p, &c->graph_host, &c->gexec_host);
        if (rc == LH_OK) rc = ensure_graph(c);
        if (rc) {
            cudaStreamSynchronize(c->st_up);
            return rc;
        }
        CK(cudaGraphLaunch(c->gexec_host, c->st), "graph launch");
        for (int s = 1; s < nsteps; s++) CK(cudaGraphLaunch(c->gexec, c->st), "graph launch");
    }
    CK(instance_download(c->dev, u1, u2, u3, p, c->st), "download");
    CK(cudaStreamSynchronize(c->st_up), "synchronize");
    return check_err_word(c);
}

extern "C" int lh_synchronize(lh_ctx *c)
{
    if (!c) return LH_EINVAL;
    CK(cudaStreamSynchronize(c->st), "synchronize");
    return check_err_word(c);
}

extern "C" int lh_get_scalars(lh_ctx *c, double *t, double *dt, int *iter, double *mpgx, double *Qx)
{
    if (!c) return LH_EINVAL;
    double sc[SC_COUNT];
    CK(cudaMemcpyAsync(sc, c->dev.inst.sc, sizeof(sc), cudaMemcpyDeviceToHost, c->st), "scalars");
    CK(cudaStreamSynchronize(c->st), "scalars");
    if (t) *t = sc[SC_T];
    if (dt) *dt = sc[SC_DT];
    if (iter) *iter = (int)sc[SC_ITER];
    if (mpgx) *mpgx = sc[SC_MPGX];
    if (Qx) *Qx = sc[SC_QX];
    return LH_OK;
}

// ---- spectra of flagged steps (spectra.f90:7-66) ---------------------------
extern "C" int lh_spectra_accumulate(lh_ctx *c)
{
    if (!c) return LH_EINVAL;
    if (!c->have_state) return fail(c, LH_ESTATE, "no state uploaded");
    const HostSetup &s = c->dev.hs;
    const size_t bytes = spectra_doubles(s.nyu, s.nyv, s.nc) * sizeof(double);
    if (!c->d_spec) {
        CK(cudaMalloc(&c->d_spec, bytes), "alloc spectra");
        CK(cudaMemsetAsync(c->d_spec, 0, bytes, c->st), "clear spectra");
        c->spec_count = 0;
    }
    launch_spectra_accumulate(c->d_inst, c->d_spec, s.nyu, s.nc, c->st);
    CK(cudaGetLastError(), "spectra launch");
    c->spec_count++;
    return LH_OK;
}

extern "C" int lh_spectra_reset(lh_ctx *c)
{
    if (!c) return LH_EINVAL;
    if (c->d_spec) {
        const HostSetup &s = c->dev.hs;
        CK(cudaMemsetAsync(c->d_spec, 0, spectra_doubles(s.nyu, s.nyv, s.nc) * sizeof(double), c->st), "reset");
    }
    c->spec_count = 0;
    return LH_OK;
}

extern "C" int lh_get_spectra(lh_ctx *c, int which, double *out, size_t cap, int *count)
{
    if (!c || which < 0 || which > 4) return fail(c, LH_EINVAL, "unknown spectrum");
    const HostSetup &s = c->dev.hs;
    const size_t nc = s.nc, nu = (size_t)(s.nyu + 2), nv = (size_t)(s.nyv + 2);
    const size_t rows = which == 1 ? nv : which == 4 ? (size_t)s.nyu : nu;
    const size_t off = which == 0 ? 0 : which == 1 ? nu : which == 2 ? nu + nv : which == 3 ? 2 * nu + nv : 3 * nu + nv;
    const size_t n = rows * nc;
    if (count) *count = c->spec_count;
    if (!out) return (int)n;
    if (cap < n) return fail(c, LH_EINVAL, "buffer too small");
    std::vector<double> plane(n, 0.0);
    if (c->d_spec) {
        CK(cudaMemcpyAsync(plane.data(), c->d_spec + off * nc, n * sizeof(double), cudaMemcpyDeviceToHost, c->st),
           "spectra download");
        CK(cudaStreamSynchronize(c->st), "spectra download");
    }
    // plane-major (row, column) -> the reference's sp(j, column), j fastest
    for (size_t j = 0; j < rows; j++)
        for (size_t col = 0; col < nc; col++) out[col * rows + j] = plane[j * nc + col];
    return (int)n;
}

// ---- stats of flagged output steps (stats.f90:1-97) ------------------------
extern "C" int lh_stats_accumulate(lh_ctx *c)
{
    if (!c) return LH_EINVAL;
    if (!c->have_state) return fail(c, LH_ESTATE, "no state uploaded");
    const HostSetup &s = c->dev.hs;
    const size_t bytes = stats_doubles(s.nyu) * sizeof(double);
    if (!c->d_stats) {
        CK(cudaMalloc(&c->d_stats, bytes), "alloc stats");
        CK(cudaMemsetAsync(c->d_stats, 0, bytes, c->st), "clear stats");
        c->stats_count = 0;
    }
    CK(launch_stats_accumulate(c->d_inst, s, c->stats_scr.pp, c->d_stats, c->st), "stats launch");
    c->stats_count++;
    return LH_OK;
}

extern "C" int lh_pressure_snapshot(lh_ctx *c)
{
    if (!c) return LH_EINVAL;
    if (!c->have_state) return fail(c, LH_ESTATE, "no state uploaded");
    const HostSetup &s = c->dev.hs;
    const size_t bytes = (size_t)s.nyu * s.nc * sizeof(double2);
    if (!c->stats_scr.pp) CK(cudaMalloc(&c->stats_scr.pp, bytes), "alloc pressure snapshot");
    CK(cudaMemcpyAsync(c->stats_scr.pp, c->dev.inst.P, bytes, cudaMemcpyDeviceToDevice, c->st), "pressure snapshot");
    return LH_OK;
}

extern "C" int lh_omega_x(lh_ctx *c, double *out, size_t cap)
{
    if (!c) return LH_EINVAL;
    const HostSetup &s = c->dev.hs;
    const size_t n = (size_t)(s.nyu + 2) * s.Nz * (s.Nx + 2);
    if (!out) return (int)n;
    if (!c->have_state) return fail(c, LH_ESTATE, "no state uploaded");
    if (cap < n) return fail(c, LH_EINVAL, "buffer too small");
    CK(stats_prepare(c->dev, c->stats_scr), "stats scratch");
    CK(omega_x_planes(c->d_inst, s, c->stats_scr, out, c->st), "omega_x");
    return (int)n;
}

extern "C" int lh_stats_reset(lh_ctx *c)
{
    if (!c) return LH_EINVAL;
    if (c->d_stats) CK(cudaMemsetAsync(c->d_stats, 0, stats_doubles(c->dev.hs.nyu) * sizeof(double), c->st), "reset");
    c->stats_count = 0;
    return LH_OK;
}

extern "C" int lh_get_stats(lh_ctx *c, double *out, size_t cap, int *count)
{
    if (!c) return LH_EINVAL;
    const size_t n = stats_doubles(c->dev.hs.nyu);
    if (count) *count = c->stats_count;
    if (!out) return (int)n;
    if (cap < n) return fail(c, LH_EINVAL, "buffer too small");
    if (!c->d_stats) {
        memset(out, 0, n * sizeof(double));
        return (int)n;
    }
    CK(cudaMemcpyAsync(out, c->d_stats, n * sizeof(double), cudaMemcpyDeviceToHost, c->st), "stats download");
    CK(cudaStreamSynchronize(c->st), "stats download");
    return (int)n;
}

extern "C" int lh_error_div(lh_ctx *c, double *err)
{
    if (!c || !err) return LH_EINVAL;
    double *d = nullptr;
    CK(cudaMalloc(&d, sizeof(double)), "alloc");
    cudaMemsetAsync(d, 0, sizeof(double), c->st);
    k_divmax<<<120, 256, 0, c->st>>>(c->d_inst, d);
    cudaError_t e = cudaMemcpyAsync(err, d, sizeof(double), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(c, e, "error_div");
    return LH_OK;
}

extern "C" int lh_get_intermediate(lh_ctx *c, int which, double *out, size_t cap)
{
    if (!c) return LH_EINVAL;
    const HostSetup &s = c->dev.hs;
    const Inst &I = c->dev.inst;
    const double2 *src;
    int len;
    switch (which) {
    case 0: src = I.NXZ1; len = s.nyu; break;
    case 1: src = I.NXZ2; len = s.nyv; break;
    case 2: src = I.NXZ3; len = s.nyu; break;
    case 3: src = I.UVF; len = s.nyv + 2; break;
    case 4: src = I.VVC; len = s.nyu + 2; break;
    case 5: src = I.WVF; len = s.nyv + 2; break;
    default: return fail(c, LH_EINVAL, "unknown intermediate");
    }
    const size_t n = (size_t)2 * len * s.nc;
    if (!out) return (int)n;
    if (cap < n) return fail(c, LH_EINVAL, "buffer too small");
    CK(download_field(c->dev, src, len, out, c->st), "intermediate");
    CK(cudaStreamSynchronize(c->st), "intermediate");
    return (int)n;
}

// ---- plane transforms -------------------------------------------------------
static int plane_transform(lh_ctx *c, double *planes, int nplanes, int sgn)
{
    if (!c || !planes || nplanes <= 0) return fail(c, LH_EINVAL, "bad plane arguments");
    const HostSetup &s = c->dev.hs;
    const int ig = s.Mx + 2;
    const size_t bytes = (size_t)ig * s.Mz * nplanes * sizeof(double);
    double *d = nullptr;
    CK(cudaMalloc(&d, bytes), "alloc planes");
    cudaError_t e = cudaMemcpyAsync(d, planes, bytes, cudaMemcpyHostToDevice, c->st);
    const int bc = 4, br = 4, thr = 256;
    const size_t smz = 2 * (size_t)s.Mz * bc * sizeof(double2), smx = 2 * (size_t)s.Mx * br * sizeof(double2);
    const int nbz = (s.nxh + bc - 1) / bc, nbx = ((s.Mz + 1) / 2 + br - 1) / br;
    if (e == cudaSuccess) {
        if (sgn > 0) {
            raise_smem_limit((const void *)k_plane_z_inv, smz);
            raise_smem_limit((const void *)k_plane_x_inv, smx);
            k_plane_z_inv<<<nplanes * nbz, thr, smz, c->st>>>(c->d_inst, d, bc, 1);
            k_plane_x_inv<<<nplanes * nbx, thr, smx, c->st>>>(c->d_inst, d, br);
        } else {
            raise_smem_limit((const void *)k_plane_z_fwd, smz);
            raise_smem_limit((const void *)k_plane_x_fwd, smx);
            k_plane_x_fwd<<<nplanes * nbx, thr, smx, c->st>>>(c->d_inst, d, br);
            k_plane_z_fwd<<<nplanes * nbz, thr, smz, c->st>>>(c->d_inst, d, bc);
            k_plane_zero_row<<<nplanes, 256, 0, c->st>>>(c->d_inst, d);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(planes, d, bytes, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(c, e, "plane transform");
    return LH_OK;
}

extern "C" int lh_four_to_phys(lh_ctx *c, double *planes, int nplanes) { return plane_transform(c, planes, nplanes, +1); }
extern "C" int lh_phys_to_four(lh_ctx *c, double *planes, int nplanes) { return plane_transform(c, planes, nplanes, -1); }

// ---- tridiagonal unit entries -------------------------------------------------
extern "C" int lh_lusolu(lh_ctx *c, int grid, int kRK, double dt, const double *rhs, double *u)
{
    if (!c || !rhs || !u || (grid != 1 && grid != 2) || kRK < 1 || kRK > 3)
        return fail(c, LH_EINVAL, "bad lusolu arguments");
    const HostSetup &s = c->dev.hs;
    const int len = grid == 2 ? s.nyu + 2 : s.nyv + 2;
    const size_t n = (size_t)len * s.nc;
    double2 *d_r = nullptr, *d_u = nullptr;
    double *d_f = nullptr;
    CK(cudaMalloc(&d_r, n * sizeof(double2)), "alloc");
    cudaError_t e = cudaMalloc(&d_u, n * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&d_f, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->dev.stage, rhs, n * sizeof(double2), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) {
        dim3 g((s.nc + 31) / 32, (len + 31) / 32), b(32, 8);
        k_col_to_plane<<<g, b, 0, c->st>>>(c->dev.stage, d_r, len, s.nc);
        k_lusolu<<<(s.nc + 127) / 128, 128, 0, c->st>>>(c->d_inst, grid, kRK, dt, d_r, d_u, d_f);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = download_field(c->dev, d_u, len, u, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(d_r);
    cudaFree(d_u);
    cudaFree(d_f);
    if (e != cudaSuccess) return cuda_fail(c, e, "lusolu");
    return LH_OK;
}

extern "C" int lh_lusolp(lh_ctx *c, double *x)
{
    if (!c || !x) return fail(c, LH_EINVAL, "bad lusolp arguments");
    const HostSetup &s = c->dev.hs;
    const int len = s.nyu;
    const size_t n = (size_t)len * s.nc;
    double2 *d_x = nullptr;
    CK(cudaMalloc(&d_x, n * sizeof(double2)), "alloc");
    cudaError_t e = cudaMemcpyAsync(c->dev.stage, x, n * sizeof(double2), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) {
        dim3 g((s.nc + 31) / 32, (len + 31) / 32), b(32, 8);
        k_col_to_plane<<<g, b, 0, c->st>>>(c->dev.stage, d_x, len, s.nc);
        k_lusolp<<<(s.nc + 127) / 128, 128, 0, c->st>>>(c->d_inst, d_x);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = download_field(c->dev, d_x, len, x, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(d_x);
    if (e != cudaSuccess) return cuda_fail(c, e, "lusolp");
    return LH_OK;
}

extern "C" int lh_get_stream(lh_ctx *c, void **stream)
{
    if (!c || !stream) return LH_EINVAL;
    *stream = (void *)c->st;
    return LH_OK;
}

extern "C" int lh_profile(lh_ctx *c, int nsteps, double *ms, int *launches)
{
    if (!c || !ms || !launches || nsteps < 1) return LH_EINVAL;
    if (!c->have_state) return fail(c, LH_ESTATE, "no state uploaded");
    LaunchTimer t;
    CK(cudaEventCreate(&t.ev[0]), "event");
    CK(cudaEventCreate(&t.ev[1]), "event");
    cudaError_t e = cudaSuccess;
    const bool cfl = c->dev.desc.dt_mode == LH_DT_CFL;
    for (int s = 0; s < nsteps && e == cudaSuccess; s++)
        for (int k = 1; k <= 3 && e == cudaSuccess; k++) e = launch_substep(c->plan, c->d_inst, k, cfl, c->st, &t);
    cudaEventDestroy(t.ev[0]);
    cudaEventDestroy(t.ev[1]);
    if (e != cudaSuccess) return cuda_fail(c, e, "profile");
    for (int k = 0; k < 5; k++) {
        ms[k] = t.ms[k];
        launches[k] = t.n[k];
    }
    return LH_OK;
}
