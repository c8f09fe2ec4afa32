/*
 * TEST INFRASTRUCTURE -- parity oracle, not part of the product.
 *
 * C restatement of the reference's RK3 time-step path (LittleHarsh channel
 * DNS, Fortran 90 + MPI) at one MPI rank.  Each function cites the reference
 * file:line it follows.  Arrays keep the reference's layouts:
 *   column fields  x(j, column), j fastest, complex(8) as (re, im) pairs,
 *                  j = jlim(1,grid) .. jlim(2,grid)   (start.f90:1009-1026)
 *   plane fields   xPL(igal, kgal, j), igal = Ngal_x + 2, kgal = Ngal_z
 * Only tests/, the smoke check and the CPU-baseline leg of bench.py load it.
 */
#ifndef LH_ORACLE_H
#define LH_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define LHO_FFT_MAXN 1024

typedef struct {
    int n;
    double dn1;
    int ifac[32];
    double wa[2 * LHO_FFT_MAXN];
} lho_cfft;

typedef struct {
    int n;
    double dn1;
    int ifac[32];
    double wa[LHO_FFT_MAXN];
} lho_rfft;

int lho_cfft_init(lho_cfft *t, int n);
int lho_rfft_init(lho_rfft *t, int n);
void lho_cfft_pass(const lho_cfft *t, int sgn, double *c, double *ch);
void lho_rfftf(const lho_rfft *t, double *c, double *ch);
void lho_rfftb(const lho_rfft *t, double *c, double *ch);
/* work: 4n doubles (cft) / n doubles (rft) */
void lho_cft(double *c, int ise, int isa, int m, int iopt, const lho_cfft *t,
             double *work);
void lho_rft(double *c, int isa, int m, int iopt, const lho_rfft *t,
             double *work);

/* grid families */
#define LHO_GRID_POLY 0 /* reference ygrid, start.f90:665-806 */
#define LHO_GRID_TANH 1 /* tanh(gamma s)/tanh(gamma) extension */

/* time-step modes */
#define LHO_DT_CFL 0   /* reference: dt from CFL at kRK=1 (FOU3D.f90:290-303) */
#define LHO_DT_FIXED 1 /* extension: fixed dt */

typedef struct {
    int Nx, Nz, ny;        /* Nspec_x, Nspec_z, input ny */
    double Re, alp, bet;
    double mpgx;           /* prescribed mean pressure gradient */
    int flag_ctpress;      /* 1 const pressure gradient, 0 const flow rate */
    int grid_type;
    double dyq;            /* poly: dymax/dymin */
    int ppp;               /* poly: exponent */
    double gamma;          /* tanh stretching */
    int dt_mode;
    double CFL;
    double dt_fixed;
    int nthreads;          /* OpenMP threads (0 = runtime default) */
} lho_params;

typedef struct lho_ctx lho_ctx;

lho_ctx *lho_create(const lho_params *p);
void lho_destroy(lho_ctx *c);

/* sizes: [Nx, Nz, Mx, Mz, nyu, nyv, nyp, ncols, igal, kgal] */
void lho_sizes(const lho_ctx *c, int *out10);

/* Grid and metric arrays as the reference builds them.  which:
 *  0 yu(0:nyu+1)  1 yv(0:nyv+1)  2 dthdyu  3 dthdyv
 *  4 dyu2i(3,0:nyu+1)  5 dyv2i(3,0:nyv+1)
 *  6 scalars [gw1, gw2, gw_bc_u1, gw_bc_u3, gwi1, gwi2, dtv, ddthetavi]
 *  7 k1F_x imag parts (0:Nx/2)   8 k1F_z imag parts (1:Nz)
 *  9 k2F_x  10 k2F_z  11 DG(3, 1:nyp+1?, ncols) -> 3*nyp_p*ncols doubles
 * returns number of doubles copied */
int lho_get_array(const lho_ctx *c, int which, double *out, int cap);

/* state in reference column layout, complex as (re,im):
 * field 0 u1 (0:nyu+1), 1 u2 (0:nyv+1), 2 u3, 3 p (1:nyu), 4 Nu1 (1:nyu),
 * 5 Nu2 (1:nyv), 6 Nu3, 7 div (1:nyu), 8 psi */
int lho_field_len(const lho_ctx *c, int field);
void lho_set_field(lho_ctx *c, int field, const double *src);
void lho_get_field(const lho_ctx *c, int field, double *dst);

/* scalars: 0 t, 1 dt, 2 dti, 3 mpgx, 4 Qx, 5 QxT, 6 iter, 7 dtc */
double lho_get_scalar(const lho_ctx *c, int which);
void lho_set_scalar(lho_ctx *c, int which, double v);

/* one RK3 substep (littleharsh.f90:169-220), kRK in 1..3 */
void lho_substep(lho_ctx *c, int kRK);
/* nsteps full RK3 steps (littleharsh.f90:163-233) */
void lho_step(lho_ctx *c, int nsteps);

/* nonlinear() intermediates captured by the last substep, column layout:
 * 0 Nu1 xz-part, 1 Nu2 xz-part, 2 Nu3 xz-part (before the y-flux sum),
 * 3 uv_f (0:nyv+1), 4 vv_c (0:nyu+1), 5 wv_f (0:nyv+1) */
int lho_get_intermediate(const lho_ctx *c, int which, double *dst, int cap);

/* plane transforms on one plane (igal x kgal reals), FOU3D.f90:653-679 and
 * FOU3D.f90:1654-1672 */
void lho_four_to_phys(lho_ctx *c, double *plane);
void lho_phys_to_four(lho_ctx *c, double *plane);

/* derivative masks, FOU3D.f90:420-523 (plane in/out, igal x kgal) */
void lho_der_x(const lho_ctx *c, const double *u, double *dudx);
void lho_der_z(const lho_ctx *c, const double *u, double *dudz);

/* LUsolU on every column for one grid (tridLU_3D.f90:38-94); grid 2 = u, 1 = v.
 * rhs and u in column layout; uses current dt and kRK. */
void lho_lusolu(lho_ctx *c, int grid, int kRK, const double *rhs, double *u);
/* LU_build + LU_dec (tridLU_3D.f90:163-221, 327-364) of every column of grid
 * (2 u/w, 1 v) at RK substep kRK with the context's dt: a(3, j, column) */
void lho_lu_factor(const lho_ctx *c, int grid, int kRK, double *a);
/* LUsolP on every column (tridLU_3D.f90:98-132), in place */
void lho_lusolp(const lho_ctx *c, double *x);

/* max |div| over columns (littleharsh.f90:370-409) */
double lho_error_div(const lho_ctx *c);

/* spectra() at a flagged step (spectra.f90:7-66, called from nonlinear at
 * FOU3D.f90:137-141): add the current state's terms into sp arrays in the
 * reference layout sp(j, column), j fastest: spU, spW and spUV over u rows
 * 0..nyu+1 (spUV with u2 interpolated to the u rows by interp_v), spV over
 * v rows 0..nyv+1, spP over p rows 1..nyu. */
void lho_spectra(lho_ctx *c, double *spU, double *spV, double *spW, double *spUV, double *spP);

/* stats (stats.f90:1-97): add the plane sums of the current state into
 * acc[13][nyu+2] (Um U2m Vm V2m Wm W2m UVm UWm VWm over planes 0..nyu+1, in
 * physical space on planes 1..nyu and over the spectral coefficients on the
 * wall planes, as nonlinear() holds them when it calls stats (FOU3D.f90:
 * 240, 307-341); Pm P2m over planes 1..nyu+1 of the latest pressure
 * snapshot; wxm wx2m over the physical omega_x of lho_omega_x). */
void lho_stats(lho_ctx *c, double *acc);
/* ppPL <- p as nonlinear() does at output steps (FOU3D.f90:149-152); the
 * snapshot is zero until the first call */
void lho_pressure_snapshot(lho_ctx *c);
/* der_z_N (FOU3D.f90:525-546) on an (Nx+2) x Nz real plane viewed as complex
 * (0:Nx/2, Nz): dudz = kz(k) u with kz_im the imaginary parts of kz(1:Nz) */
void lho_der_z_n(const double *u, double *dudz, const double *kz_im, int Nx, int Nz);
/* omega_x of the current state at planes 0..nyu+1 (FOU3D.f90:314-338):
 * (nyu+2) planes of (Nx+2) x Nz reals, physical values at i = 1..Nx */
void lho_omega_x(lho_ctx *c, double *wx);

/* generic mode-count helpers for the 2-D (i,k) <-> plane map */
int lho_column_i(const lho_ctx *c, int column);   /* 1-based column */
int lho_column_k(const lho_ctx *c, int column);
int lho_column_row(const lho_ctx *c, int column); /* k - dk (1-based row) */

#ifdef __cplusplus
}
#endif
#endif
