/*
 * lh_gpu.h -- C ABI of the B200 (sm_100a) FP64 time-step engine for the
 * LittleHarsh channel DNS.
 *
 * The entry points replace, one for one, the reference subroutines that sit
 * under the Fortran main loop (reference file:line given beside each).  All
 * arrays use the reference's own layouts so a Fortran caller can pass its
 * arrays unchanged through iso_c_binding:
 *
 *   column fields   complex(8) x(jlim(1,grid):jlim(2,grid), column), j fastest,
 *                   interleaved (re, im) doubles.  Column order is the
 *                   reference's np=1 order: k = 1..Nz (z mode), i = 0..Nx/2
 *                   inner (start.f90:964-981).
 *                     u1, u3 : j = 0 .. nyu+1   (nyu = ny-1)
 *                     u2     : j = 0 .. nyv+1   (nyv = ny-2)
 *                     p      : j = 1 .. nyu
 *   plane arrays    real(8) xPL(Ngal_x+2, Ngal_z), x fastest, (re, im) pairs
 *                   for spectral planes (FOU3D.f90:734).
 *
 * Every function returns 0 on success and a negative LH_E* code on failure;
 * lh_last_error() gives a message.  Device faults are reported through a
 * device error word, never by trapping.  One caller thread per context.
 */
#ifndef LH_GPU_H
#define LH_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LH_OK 0
#define LH_EINVAL -1   /* bad argument or unsupported size */
#define LH_ECUDA -2    /* CUDA runtime error */
#define LH_ENOMEM -3   /* device allocation failed / over budget */
#define LH_EDEVICE -4  /* device-side error word set (non-finite state, ...) */
#define LH_ESTATE -5   /* call out of order (no state uploaded, ...) */

#define LH_GRID_POLY 0 /* reference polynomial grid, start.f90:665-806 */
#define LH_GRID_TANH 1 /* tanh(gamma s)/tanh(gamma) stretching (extension) */

#define LH_DT_CFL 0    /* reference CFL rule at kRK=1, FOU3D.f90:290-303 */
#define LH_DT_FIXED 1  /* fixed dt (extension used by the benchmark configs) */

/* Instance description: the values start.f90 reads from input.in
 * (start.f90:85-252) plus the two extensions above. */
typedef struct lh_grid_desc {
    int Nx, Nz;          /* Fourier modes Nspec_x, Nspec_z (Ngal = 3N/2) */
    int ny;              /* input ny: v faces 0..ny-1 */
    double Re;           /* bulk Reynolds number */
    double alp, bet;     /* box wavenumbers, Lx = 2pi/alp, Lz = 2pi/bet */
    double mpgx;         /* mean pressure gradient (flpress = 1) */
    int flag_ctpress;    /* 1: constant pressure gradient, 0: constant flow rate */
    int grid_type;       /* LH_GRID_* */
    double dyq;          /* poly grid: dymax/dymin */
    int ppp;             /* poly grid: exponent */
    double gamma;        /* tanh grid: stretching */
    int dt_mode;         /* LH_DT_* */
    double CFL;          /* CFL number (LH_DT_CFL) */
    double dt;           /* time step (LH_DT_FIXED) */
} lh_grid_desc;

typedef struct lh_ctx lh_ctx;

/* Sizes of one instance: [Nx, Nz, Mx, Mz, nyu, nyv, ncols, igal, kgal] */
typedef struct lh_sizes {
    int Nx, Nz, Mx, Mz, nyu, nyv, ncols, igal, kgal;
} lh_sizes;

/* ---- context: replaces start() set-up, start.f90:53-662 -------------- */
int lh_ctx_create(const lh_grid_desc *desc, lh_ctx **out);
int lh_ctx_destroy(lh_ctx *ctx);
const char *lh_last_error(const lh_ctx *ctx);
int lh_get_sizes(const lh_ctx *ctx, lh_sizes *out);
/* Grid arrays as built on the host: which = 0 yu, 1 yv, 2 dthdyu, 3 dthdyv
 * (lengths nyu+2 / nyv+2).  Returns the element count. */
int lh_get_grid(const lh_ctx *ctx, int which, double *out, int cap);

/* Host-only set-up query (needs no GPU): the same arrays as lh_get_grid for a
 * description, or, for which = 4, the scalars [gw1, gw2, gw_bc, gwi1, gwi2,
 * dtv] (start.f90:476, 518-537).  Returns the element count or LH_EINVAL. */
int lh_host_grid(const lh_grid_desc *desc, int which, double *out, int cap);

/* ---- state: replaces getini/read_in (start.f90:1221-1997) ------------- */
/* Host arrays in the reference column layout (see above).  p may be NULL
 * (zero pressure).  Resets Nu (littleharsh.f90:127-129), t and iter. */
int lh_upload_state(lh_ctx *ctx, const double *u1, const double *u2,
                    const double *u3, const double *p);
int lh_download_state(lh_ctx *ctx, double *u1, double *u2, double *u3,
                      double *p);
/* Nu1, Nu2, Nu3 (interior rows) of the last substep, column layout:
 * Nu1/Nu3 j = 1..nyu, Nu2 j = 1..nyv.  Any pointer may be NULL. */
int lh_download_nu(lh_ctx *ctx, double *nu1, double *nu2, double *nu3);

/* ---- the RK3 step: replaces the loop body littleharsh.f90:165-231 ---- */
/* One substep kRK = 1..3: RHS0_u1/2/3, nonlinear, solveU x3,
 * flowrate correction (flag_ctpress = 0), solveP, v_corr. */
int lh_substep(lh_ctx *ctx, int kRK);
/* nsteps full RK3 steps (captured once in a CUDA graph and replayed). */
int lh_step(lh_ctx *ctx, int nsteps);
/* t, dt, iter, mpgx, Qx (flow rate of the (0,0) mode) */
int lh_get_scalars(lh_ctx *ctx, double *t, double *dt, int *iter,
                   double *mpgx, double *Qx);
/* Host-buffer step for callers that keep the state on the host: upload,
 * nsteps RK3 steps, download (the Fortran drop-in call).  Same results as
 * lh_upload_state + lh_step + lh_download_state; p is uploaded beside the
 * first substep's plane pass.  Synchronous: returns after the download. */
int lh_step_host(lh_ctx *ctx, double *u1, double *u2, double *u3, double *p,
                 int nsteps);
int lh_synchronize(lh_ctx *ctx);
/* The CUDA stream (cudaStream_t) every call of this context is ordered on. */
int lh_get_stream(lh_ctx *ctx, void **stream);
/* Autotuner of the launch shapes (no counterpart in the reference, whose
 * shapes are fixed by FFTPACK's factorisation, cft_buff.f:141-163,
 * rft_buff.f:133-160): the plane pipeline's tile bounds (x modes per
 * z-inverse CTA, z rows per x-products CTA, x modes per z-forward CTA), the
 * plane-staging budget and the number of column-pass launches for this
 * context's size, chosen by timing RK3 steps of a scratch instance (the
 * context's state is not touched; its current state is copied in so the CFL
 * step is the run's).  None of them changes any arithmetic: the states stay
 * bit-identical.  Results are cached per GPU name and (Mz, Mx, nyu) in the
 * file LH_TUNE_CACHE (default lh_tune_cache.txt beside the library) and in a
 * process-wide table that every later plan of that size -- contexts and
 * batches -- uses.  force = 1 measures even when the cache has the size.
 * params (may be NULL) receives [cbz, rbx, cbf, staging_mb, col_waves,
 * source], source 1 = measured now, 2 = read from the cache.  Allocates one
 * scratch instance for the duration of the call. */
int lh_autotune(lh_ctx *ctx, int force, int *params);
/* Runs nsteps RK3 steps launch by launch with CUDA events around every
 * kernel and returns, per kernel class (0 z-inverse, 1 x-products,
 * 2 z-forward, 3 dt, 4 column), the summed milliseconds and launch counts. */
int lh_profile(lh_ctx *ctx, int nsteps, double *ms, int *launches);
/* max |div| after the last projection (error(), littleharsh.f90:370-409) */
int lh_error_div(lh_ctx *ctx, double *err);

/* ---- spectra of flagged steps: replace spectra() (spectra.f90:7-66), which
 * nonlinear() calls every nstat steps at kRK = 1 (FOU3D.f90:76-81, 137-141).
 * lh_spectra_accumulate adds the current state's terms into accumulators that
 * stay on the device: spU/spV/spW += |u1|^2 / |u2|^2 / |u3|^2, spUV +=
 * Re(u1 conj(u2 interpolated to the u rows by interp_v)), spP += |p|^2, per
 * (y row, column).  Call it between steps where the reference's flag would be
 * set; it is queued on the context's stream.  lh_get_spectra copies one of
 * them out in the reference layout sp(j, column), rows fastest: which 0 spU
 * and 2 spW and 3 spUV (rows 0..nyu+1), 1 spV (0..nyv+1), 4 spP (1..nyu);
 * *count (optional) receives the accumulations since the last reset.  Returns
 * the element count; out = NULL only queries it.  The first accumulation
 * allocates the accumulators (5 x ncols x ny doubles). */
int lh_spectra_accumulate(lh_ctx *ctx);
int lh_spectra_reset(lh_ctx *ctx);
int lh_get_spectra(lh_ctx *ctx, int which, double *out, size_t cap, int *count);

/* ---- stats of flagged steps: replace stats() (stats.f90:1-97), which
 * nonlinear() calls every nstat steps at kRK = 1 (FOU3D.f90:76-81, 290,
 * 307-341), after ops_in_planes2 (FOU3D.f90:240) has transformed planes
 * 1..nyu of its plane arrays to physical space in place (FOU3D.f90:1541,
 * 1584).  lh_stats_accumulate adds into acc[13][nyu+2], j = 0..nyu+1:
 *   0 Um 1 U2m  2 Vm 3 V2m  4 Wm 5 W2m  6 UVm (u1 x u2 interpolated to the
 *   u rows)  7 UWm  8 VWm (u2 x u3 interpolated to the v rows) -- sums over
 *   the physical Mx x Mz grid on planes 1..nyu, over the spectral
 *   coefficients (re and im entries) on the wall planes 0 and nyu+1;
 *   9 Pm 10 P2m -- over the spectral coefficients of the pressure planes of
 *   the latest lh_pressure_snapshot (zero before the first), planes 1..nyu;
 *   11 wxm 12 wx2m -- over omega_x = -d(u2)/dz + d(u3)/dy at the v faces in
 *   physical space on the Nx x Nz grid (FOU3D.f90:314-338), planes 0..nyu+1.
 * The physical-grid sums are evaluated from the spectral coefficients by
 * Parseval's identity on the transform grid (the same sums; no transform
 * runs).  lh_get_stats copies out acc and the count of accumulations. */
int lh_stats_accumulate(lh_ctx *ctx);
int lh_stats_reset(lh_ctx *ctx);
int lh_get_stats(lh_ctx *ctx, double *out, size_t cap, int *count);
/* ppPL <- p: nonlinear() refills the pressure planes at every output step
 * (FOU3D.f90:149-152) and stats() reads them (stats.f90:45-52); call it
 * where the reference's output flag is set, before that step's stats. */
int lh_pressure_snapshot(lh_ctx *ctx);
/* omega_x of the current state as nonlinear() forms it for stats()
 * (modes_to_planes_phys, der_z_N, der_yv_h_wx, four_to_phys_N; FOU3D.f90:
 * 314-338): (nyu+2) planes j = 0..nyu+1 of (Nx+2) x Nz doubles, x fastest,
 * physical values in x = 1..Nx, host pointer.  Returns the element count;
 * out = NULL only queries it.  The first call allocates a transform scratch
 * of at most 256 MB. */
int lh_omega_x(lh_ctx *ctx, double *out, size_t cap);

/* ---- nonlinear-term intermediates of the last substep (parity) -------- */
/* which: 0 Nu1 x/z part, 1 Nu2 x/z part, 2 Nu3 x/z part (FOU3D.f90:259-261
 * before the y-flux sum), 3 uv_f (j=0..nyv+1), 4 vv_c (j=0..nyu+1),
 * 5 wv_f (j=0..nyv+1).  Column layout.  Returns the element count. */
int lh_get_intermediate(lh_ctx *ctx, int which, double *out, size_t cap);

/* ---- plane transforms: replace four_to_phys_u (FOU3D.f90:653-679) and --
 * phys_to_four_du (FOU3D.f90:1654-1672), i.e. cft/rft on a plane.
 * nplanes planes of igal*kgal doubles, host pointers, in place. */
int lh_four_to_phys(lh_ctx *ctx, double *planes, int nplanes);
int lh_phys_to_four(lh_ctx *ctx, double *planes, int nplanes);

/* ---- tridiagonal solves: replace LUsolU (tridLU_3D.f90:38-94, with
 * LU_build :163-221 and LU_dec :327-364) and LUsolP (tridLU_3D.f90:98-132
 * with the DG factors of LU_buildP/LU_decP :224-297, :366-407).
 * grid: 2 = u/w (j = 0..nyu+1), 1 = v (j = 0..nyv+1).  beta = bRK*dt/Re is
 * taken from kRK and dt.  Column layout, host pointers. */
int lh_lusolu(lh_ctx *ctx, int grid, int kRK, double dt, const double *rhs,
              double *u);
int lh_lusolp(lh_ctx *ctx, double *x);

/* ---- tridiagonal factors in the reference's a(3, j, column) layout -----
 * (tridLU_3D.f90): a(1,j) lower diagonal, a(2,j) inverse pivot, a(3,j)
 * scaled upper diagonal, j from jlim(1,grid), 3 doubles per row, rows
 * fastest within a column.  grid: 2 = u/w (j = 0..nyu+1), 1 = v (j =
 * 0..nyv+1), 3 = p (j = 1..nyu).
 *
 * lh_tridiag_factor replaces LU_build + LU_dec (tridLU_3D.f90:163-221,
 * 327-364) of every column for RK substep kRK and time step dt (grid 1, 2;
 * computed on the device with the reference's operation order), and, for
 * grid = 3, returns the pressure factors DG of LU_buildP + LU_decP
 * (tridLU_3D.f90:224-297, 366-407; start.f90:636) the engine uses (kRK, dt
 * ignored).  Returns the double count 3 x rows x ncols; a = NULL only
 * queries it, cap is the capacity of a in doubles.
 * lh_tridiag_solve replaces the solve of LUsolU / LUsolP with factors the
 * caller holds (tridLU_3D.f90:70-82, 115-128): x is x(j, column), complex,
 * solved in place.
 * lh_set_dg installs a caller's DG (the start.f90:636 array, grid 3 layout)
 * as the engine's pressure factors; its lower diagonal a(1,j) must be the
 * same in every column, as LU_buildP forms it (LH_EINVAL otherwise). */
int lh_tridiag_factor(lh_ctx *ctx, int grid, int kRK, double dt, double *a, size_t cap);
int lh_tridiag_solve(lh_ctx *ctx, int grid, const double *a, double *x);
int lh_set_dg(lh_ctx *ctx, const double *a);

/* ---- continuing a run: getini with flag_init = 2 (start.f90:1268-1282)
 * takes t and iter from the restart file's header and keeps its mpgx.  Call
 * after lh_upload_state (which starts t and iter at 0 and mpgx at the
 * description's); the state must be the complete one (read_in at one rank
 * leaves the top ghost plane of u1/u3 at zero, which changes the next step). */
int lh_set_scalars(lh_ctx *ctx, double t, int iter, double mpgx);

/* Allocation-free LUsolU for callers that cannot allocate device memory
 * per call (inside CUDA-graph capture, in a loop that must not hit the
 * synchronisation of cudaMalloc/cudaFree, or with device memory owned by
 * another allocator).  No counterpart in the reference.  rhs_dev and u_dev
 * are device arrays the caller owns, in the engine's plane-major layout:
 * complex element (j, column) at j*ncols + column, rows 0..nyu+1 (grid 2)
 * or 0..nyv+1 (grid 1); they may be the same array.  The only scratch is a
 * fixed file-scope device array of 2^21 doubles (16 MiB, held on every GPU
 * that loads the library); rows x columns above that return LH_EINVAL.
 * The first call on a device looks the array's device address up
 * (cudaGetSymbolAddress), so make it before any stream capture.  Calls are
 * ordered on the context's stream; calls that overlap on the GPU (other
 * streams, other contexts on the same device) share the scratch and race.
 * Every call overwrites the scratch rows it uses before reading them. */
int lh_lusolu_noalloc(lh_ctx *ctx, int grid, int kRK, double dt,
                      const double *rhs_dev, double *u_dev);

/* ---- batched / served instances ------------------------------------- */
typedef struct lh_batch lh_batch;
/* A batch owns many independent instances of uneven size that advance in
 * shared launches.  HBM budget in bytes (0 = no limit). */
int lh_batch_create(size_t hbm_budget, lh_batch **out);
int lh_batch_destroy(lh_batch *b);
const char *lh_batch_last_error(const lh_batch *b);
/* Bytes of device memory one instance of this description needs. */
size_t lh_instance_bytes(const lh_grid_desc *desc);
/* Admit an instance (returns its slot id >= 0) with its initial state in
 * the column layout; LH_ENOMEM when the budget is exhausted. */
int lh_batch_add(lh_batch *b, const lh_grid_desc *desc, const double *u1,
                 const double *u2, const double *u3, const double *p,
                 int *slot);
int lh_batch_remove(lh_batch *b, int slot);
/* Advance every live instance by nsteps RK3 steps in shared launches. */
int lh_batch_step(lh_batch *b, int nsteps);
int lh_batch_download(lh_batch *b, int slot, double *u1, double *u2,
                      double *u3, double *p);
int lh_batch_scalars(lh_batch *b, int slot, double *t, double *dt, int *iter);
/* Restore a snapshot of a live instance (lh_batch_download + lh_batch_scalars,
 * or a restart file): set t, iter and mpgx of an admitted instance, as
 * lh_set_scalars does for a context (getini with flag_init = 2,
 * start.f90:1268-1282). */
int lh_batch_set_scalars(lh_batch *b, int slot, double t, int iter, double mpgx);
int lh_batch_count(const lh_batch *b);
int lh_batch_synchronize(lh_batch *b);

#ifdef __cplusplus
}
#endif
#endif /* LH_GPU_H */
