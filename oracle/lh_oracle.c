/*
 * TEST INFRASTRUCTURE -- parity oracle, not part of the product.
 *
 * C restatement of the reference's time-step path for one MPI rank
 * (mpirun -np 1): start.f90 set-up (ygrid, def_k, proc_lims_*, RK
 * coefficients, grid weights, LU_buildP/LU_decP), littleharsh.f90's RK3
 * loop body (RHS0_u1/u2/u3, solveU, solveP, v_corr, flow-rate bookkeeping),
 * FOU3D.f90's nonlinear() with interp_u/v, modes_to_planes_UVP,
 * ops_in_planes2, planes_to_modes_UVP/NUVP, der_x/der_z/der_yu_h/der_yv_h and
 * dtc_calc, and tridLU_3D.f90's factor/solve routines.  Arithmetic is written
 * in the reference's operation order; complex*real products are component-
 * wise, complex*complex products use the textbook formula.  The build uses
 * -ffp-contract=off so no fused multiply-adds are introduced.
 *
 * OpenMP (when enabled) splits planes and columns across threads; every
 * result is independent of the thread count (the only reduction is a max).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "lh_oracle.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#define UGRID 2
#define VGRID 1
#define PGRID 3

struct lho_ctx {
    lho_params prm;
    int Nx, Nz, Mx, Mz;
    int nyv, nyu, nyp;
    int ncols, nxh, igal, kgal;
    /* grids, 0-based storage mirroring Fortran lower bound 0 */
    double *yu, *yv, *dthdyu, *dthdyv, *dyu2i, *dyv2i;
    double gw[2], gw_bc_u1, gw_bc_u3, gwi[2];
    double dtheta, dthetai, ddthetavi, dthetavi;
    double dtv;
    double aRK[3], bRK[3], gRK[3], cRK[3], dRK[3];
    double *k1x, *k1z, *k2x, *k2z; /* imag parts of im*k, and -k^2 */
    int *col_i, *col_k, *col_row;
    double *DG;
    lho_cfft cz;
    lho_rfft rx;
    lho_cfft czN; /* buffC_z: cft of length Nspec_z (start.f90:414-421) */
    lho_rfft rxN; /* buffR_x: rft of length Nspec_x */
    double *pp;   /* p as ppPL last held it (FOU3D.f90:151-152), column layout */
    /* column fields (re,im pairs) */
    double *u1, *u2, *u3, *p, *psi, *div;
    double *Nu1, *Nu2, *Nu3, *du1, *du2, *du3;
    double *u1_itp, *u2_itp, *u3_itp;
    double *Nu1_dy, *Nu2_dy, *Nu3_dy;
    double *uv_f, *vv_c, *wv_f;
    double *sav_nxz[3];
    /* planes */
    double *u1PL, *u2PL, *u3PL, *u1PL_itp, *u2PL_itp, *u3PL_itp;
    double *Nu1PL, *Nu2PL, *Nu3PL;
    double *uu_cPL, *uw_cPL, *vv_cPL, *ww_cPL, *uv_fPL, *wv_fPL;
    double *a_ugrid, *a_vgrid; /* LU factor scratch per thread */
    double *u11;
    /* scalars */
    double t, dt, dti, dtc, Qx, QxT, mpgx, dgx;
    int iter, kRK;
    int nthr;
};

/* ------------------------------------------------------------------ */
/* layout helpers                                                       */
static int jlo(int grid) { return grid == PGRID ? 1 : 0; }
static int jlen(const lho_ctx *c, int grid)
{
    if (grid == UGRID) return c->nyu + 2; /* 0 .. nyu+1 */
    if (grid == VGRID) return c->nyv + 2; /* 0 .. nyv+1 */
    return c->nyu;                        /* 1 .. nyu */
}
/* complex column element (j, column), column 1-based */
#define CX(x, lo, len, j, col) ((x) + 2 * ((size_t)((j) - (lo)) + (size_t)(len) * ((col) - 1)))
/* plane element (i, k, j), i,k 1-based; plane lower bound 0 */
#define PL(c, x, i, k, j) ((x) + ((size_t)((i) - 1) + (size_t)(c)->igal * ((size_t)((k) - 1) + (size_t)(c)->kgal * (size_t)(j))))
#define PLANE(c, x, j) ((x) + (size_t)(c)->igal * (size_t)(c)->kgal * (size_t)(j))

/* integer power by binary powering, the way a Fortran real**integer is
 * evaluated for a run-time exponent */
static double powi(double x, int m)
{
    unsigned n = m < 0 ? (unsigned)(-m) : (unsigned)m;
    double y = (n % 2) ? x : 1.0;
    while (n >>= 1) {
        x = x * x;
        if (n % 2) y = y * x;
    }
    return m < 0 ? 1.0 / y : y;
}

static double *zalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

/* ------------------------------------------------------------------ */
/* ygrid (start.f90:665-806) and the tanh extension                     */
static void ygrid(lho_ctx *c)
{
    int nn = c->nyv + 1;
    c->yu = zalloc(nn + 2);
    c->yv = zalloc(nn + 1);
    c->dthdyu = zalloc(nn + 2);
    c->dthdyv = zalloc(nn + 1);
    c->dyu2i = zalloc(3 * (nn + 2));
    c->dyv2i = zalloc(3 * (nn + 1));
    double *yu = c->yu, *yv = c->yv;
    c->dtheta = 1.0;
    c->dthetai = 1.0 / c->dtheta;
    c->ddthetavi = 1.0 / c->dtheta;
    double qqq = nn / 2.0;
    if (c->prm.grid_type == LHO_GRID_POLY) {
        int ppp = c->prm.ppp;
        double dyq = c->prm.dyq;
        double bbb = (dyq - 1.0) / (qqq * (1.0 - powi(qqq, ppp - 1) +
                                           dyq * ((1.0 - qqq) * powi(qqq, ppp - 1) - powi(1.0 - qqq, ppp))));
        double aaa = (1.0 - bbb * powi(qqq, ppp)) / qqq;
        yu[0] = aaa * (-1.0 + .5 - qqq) + bbb * powi(-1.0 + .5 - qqq, ppp);
        for (int j = 0; j <= nn; j++) {
            yv[j] = aaa * (j - qqq) + bbb * powi(j - qqq, ppp);
            yu[j + 1] = aaa * (j + .5 - qqq) + bbb * powi(j + .5 - qqq, ppp);
        }
        c->dthdyu[0] = 1.0 / (aaa + ppp * bbb * powi(-1.0 + .5 - qqq, ppp - 1));
        for (int j = 0; j <= nn; j++) {
            c->dthdyv[j] = 1.0 / (aaa + ppp * bbb * powi(j - qqq, ppp - 1));
            c->dthdyu[j + 1] = 1.0 / (aaa + ppp * bbb * powi(j + .5 - qqq, ppp - 1));
        }
    } else {
        /* y(s) = tanh(gamma*s)/tanh(gamma), s = (j - q)/q; dtheta/dy is the
         * inverse of dy/dj evaluated analytically. */
        double g = c->prm.gamma, tg = tanh(g);
#define TANHY(x) (tanh(g * ((x) - qqq) / qqq) / tg)
#define TANHD(x) (1.0 / (g * (1.0 - tanh(g * ((x) - qqq) / qqq) * tanh(g * ((x) - qqq) / qqq)) / (qqq * tg)))
        yu[0] = TANHY(-1.0 + .5);
        c->dthdyu[0] = TANHD(-1.0 + .5);
        for (int j = 0; j <= nn; j++) {
            yv[j] = TANHY((double)j);
            yu[j + 1] = TANHY(j + .5);
            c->dthdyv[j] = TANHD((double)j);
            c->dthdyu[j + 1] = TANHD(j + .5);
        }
#undef TANHY
#undef TANHD
    }
    double *du = c->dyu2i, *dv = c->dyv2i;
#define DU(r, j) du[(r) - 1 + 3 * (j)]
#define DV(r, j) dv[(r) - 1 + 3 * (j)]
    int j = 0;
    DU(1, j) = 0.0;
    DU(2, j) = -2.0 / ((yu[j + 1] - yu[j]) * (yu[j + 1] - yu[j]));
    DU(3, j) = 1.0 / ((yu[j + 1] - yu[j]) * (yu[j + 1] - yu[j]));
    DV(1, j) = 0.0;
    DV(2, j) = -2.0 / ((yv[j + 1] - yv[j]) * (yv[j + 1] - yv[j]));
    DV(3, j) = 1.0 / ((yv[j + 1] - yv[j]) * (yv[j + 1] - yv[j]));
    for (j = 1; j <= nn - 1; j++) {
        DU(1, j) = 2.0 / ((yu[j] - yu[j - 1]) * (yu[j + 1] - yu[j - 1]));
        DU(2, j) = -2.0 / ((yu[j + 1] - yu[j]) * (yu[j] - yu[j - 1]));
        DU(3, j) = 2.0 / ((yu[j + 1] - yu[j]) * (yu[j + 1] - yu[j - 1]));
        DV(1, j) = 2.0 / ((yv[j] - yv[j - 1]) * (yv[j + 1] - yv[j - 1]));
        DV(2, j) = -2.0 / ((yv[j + 1] - yv[j]) * (yv[j] - yv[j - 1]));
        DV(3, j) = 2.0 / ((yv[j + 1] - yv[j]) * (yv[j + 1] - yv[j - 1]));
    }
    j = nn;
    DU(1, j) = 2.0 / ((yu[j] - yu[j - 1]) * (yu[j + 1] - yu[j - 1]));
    DU(2, j) = -2.0 / ((yu[j + 1] - yu[j]) * (yu[j] - yu[j - 1]));
    DU(3, j) = 2.0 / ((yu[j + 1] - yu[j]) * (yu[j + 1] - yu[j - 1]));
    DV(1, j) = 1.0 / ((yv[j] - yv[j - 1]) * (yv[j] - yv[j - 1]));
    DV(2, j) = -2.0 / ((yv[j] - yv[j - 1]) * (yv[j] - yv[j - 1]));
    DV(3, j) = 0.0;
    j = nn + 1;
    DU(1, j) = 1.0 / ((yu[j] - yu[j - 1]) * (yu[j] - yu[j - 1]));
    DU(2, j) = -2.0 / ((yu[j] - yu[j - 1]) * (yu[j] - yu[j - 1]));
    DU(3, j) = 0.0;
#undef DU
#undef DV
}

/* def_k (start.f90:809-902) */
static void def_k(lho_ctx *c)
{
    int nxh = c->Nx / 2 + 1;
    c->k1x = zalloc(nxh);
    c->k2x = zalloc(nxh);
    c->k1z = zalloc(c->Nz);
    c->k2z = zalloc(c->Nz);
    for (int i = 0; i <= c->Nx / 2; i++) {
        c->k1x[i] = c->prm.alp * i;
        c->k2x[i] = -((c->prm.alp * i) * (c->prm.alp * i));
    }
    for (int k = 1; k <= c->Nz / 2; k++) {
        c->k1z[k - 1] = c->prm.bet * (k - 1);
        c->k2z[k - 1] = -((c->prm.bet * (k - 1)) * (c->prm.bet * (k - 1)));
    }
    for (int k = c->Nz / 2 + 1; k <= c->Nz; k++) {
        c->k1z[k - 1] = -(c->prm.bet * (c->Nz - k + 1));
        c->k2z[k - 1] = -((c->prm.bet * (c->Nz - k + 1)) * (c->prm.bet * (c->Nz - k + 1)));
    }
}

/* proc_lims_columns at np = 1 (start.f90:909-1070): k-major column list
 * with the z-shift dk = Nz - Mz for k > Nz/2 */
static void proc_lims_columns(lho_ctx *c)
{
    int nc = (c->Nx / 2 + 1) * c->Nz;
    c->col_i = (int *)calloc(nc + 1, sizeof(int));
    c->col_k = (int *)calloc(nc + 1, sizeof(int));
    c->col_row = (int *)calloc(nc + 1, sizeof(int));
    int column = 0;
    for (int k = 1; k <= c->Nz / 2; k++)
        for (int i = 0; i <= c->Nx / 2; i++) {
            column++;
            c->col_i[column] = i;
            c->col_k[column] = k;
        }
    for (int k = c->Nz - c->Nz / 2 + 1; k <= c->Nz; k++)
        for (int i = 0; i <= c->Nx / 2; i++) {
            column++;
            c->col_i[column] = i;
            c->col_k[column] = k;
        }
    for (int col = 1; col <= nc; col++) {
        int dk = c->col_k[col] > c->Nz / 2 ? c->Nz - c->Mz : 0;
        c->col_row[col] = c->col_k[col] - dk;
    }
}

/* LU_buildP + LU_decP (tridLU_3D.f90:224-297, 366-407), called at
 * start.f90:636 */
static void lu_buildp(lho_ctx *c)
{
    int ns = 1, ne = c->nyu, len = ne - ns + 1, nc = c->ncols;
    c->DG = zalloc((size_t)3 * len * nc);
    double *Db = zalloc(len + 2), *Gb = zalloc(len + 2), *Dt = zalloc(len + 2), *Gt = zalloc(len + 2);
    /* arrays indexed ns-1 .. ne+1 -> offset +1 */
#define V(a, j) a[(j) - ns + 1]
    for (int j = ns; j <= ne; j++) {
        V(Db, j - 1) = -c->ddthetavi * c->dthdyu[j];
        V(Gb, j) = -c->ddthetavi * c->dthdyv[j];
        V(Dt, j) = c->ddthetavi * c->dthdyu[j];
        V(Gt, j + 1) = c->ddthetavi * c->dthdyv[j];
    }
#define A(r, j, col) c->DG[((r) - 1) + 3 * ((size_t)((j) - ns) + (size_t)len * ((col) - 1))]
    for (int col = 1; col <= nc; col++) {
        double k2x = c->k2x[c->col_i[col]], k2z = c->k2z[c->col_k[col] - 1];
        A(2, ns, col) = (V(Dt, ns) * V(Gb, ns)) + k2x + k2z;
        A(3, ns, col) = (V(Dt, ns) * V(Gt, ns + 1));
        A(2, ne, col) = (V(Db, ne - 1) * V(Gt, ne)) + k2x + k2z;
        A(1, ne, col) = (V(Db, ne - 1) * V(Gb, ne - 1));
        for (int j = ns + 1; j <= ne - 1; j++) {
            A(2, j, col) = (V(Db, j - 1) * V(Gt, j)) + (V(Dt, j) * V(Gb, j)) + k2x + k2z;
            A(1, j, col) = (V(Db, j - 1) * V(Gb, j - 1));
            A(3, j, col) = (V(Dt, j) * V(Gt, j + 1));
        }
    }
    /* gauge row of the (0,0) mode */
    A(1, ns, 1) = 0.0;
    A(2, ns, 1) = 1.0 / ((c->yu[1 + 1] - c->yu[1]) * (c->yu[1 + 1] - c->yu[1]));
    A(3, ns, 1) = 0.0;
    for (int col = 1; col <= nc; col++) {
        A(2, ns, col) = 1.0 / A(2, ns, col);
        for (int j = ns + 1; j <= ne; j++) {
            A(3, j - 1, col) = A(3, j - 1, col) * A(2, j - 1, col);
            A(2, j, col) = 1.0 / (A(2, j, col) - A(1, j, col) * A(3, j - 1, col));
        }
    }
#undef A
#undef V
    free(Db);
    free(Gb);
    free(Dt);
    free(Gt);
}

lho_ctx *lho_create(const lho_params *p)
{
    if (p->Nx < 2 || p->Nz < 2 || (p->Nx & 1) || (p->Nz & 1) || p->ny < 5) return NULL;
    lho_ctx *c = (lho_ctx *)calloc(1, sizeof(lho_ctx));
    c->prm = *p;
    c->Nx = p->Nx;
    c->Nz = p->Nz;
    /* start.f90:124-136 : Nspec = 2*Ngal/3 -> Ngal = 3*Nspec/2 */
    c->Mx = 3 * p->Nx / 2;
    c->Mz = 3 * p->Nz / 2;
    c->nyv = p->ny - 2;
    c->nyu = c->nyv + 1;
    c->nyp = c->nyv;
    c->nxh = c->Nx / 2 + 1;
    c->ncols = c->nxh * c->Nz;
    c->igal = c->Mx + 2;
    c->kgal = c->Mz;
    c->nthr = 1;
#ifdef _OPENMP
    c->nthr = p->nthreads > 0 ? p->nthreads : omp_get_max_threads();
#endif
    if (lho_cfft_init(&c->cz, c->Mz) != 0 || lho_rfft_init(&c->rx, c->Mx) != 0 ||
        lho_cfft_init(&c->czN, c->Nz) != 0 || lho_rfft_init(&c->rxN, c->Nx) != 0) {
        free(c);
        return NULL;
    }
    ygrid(c);
    def_k(c);
    /* start.f90:439-453 */
    c->aRK[0] = 4.0 / 15.0;
    c->aRK[1] = 1.0 / 15.0;
    c->aRK[2] = 1.0 / 6.0;
    c->bRK[0] = 4.0 / 15.0;
    c->bRK[1] = 1.0 / 15.0;
    c->bRK[2] = 1.0 / 6.0;
    c->gRK[0] = 8.0 / 15.0;
    c->gRK[1] = 5.0 / 12.0;
    c->gRK[2] = 3.0 / 4.0;
    c->cRK[0] = 0.0;
    c->cRK[1] = -17.0 / 60.0;
    c->cRK[2] = -5.0 / 12.0;
    c->dRK[0] = 8.0 / 15.0;
    c->dRK[1] = 2.0 / 15.0;
    c->dRK[2] = 1.0 / 3.0;
    /* start.f90:476 */
    c->dtv = p->Re / (-c->k2x[c->Nx / 2] - c->k2z[c->Nz / 2 - 1] +
                      4.0 / ((c->yv[1] - c->yv[0]) * (c->yv[1] - c->yv[0])));
    proc_lims_columns(c);
    /* start.f90:518-537 */
    double *yu = c->yu, *yv = c->yv;
    int nyu = c->nyu, nyv = c->nyv;
    c->gw[0] = -(yv[0] - yu[0]) / (yv[0] - yu[1]);
    c->gw[1] = (yu[nyu + 1] - yv[nyv + 1]) / (yv[nyv + 1] - yu[nyu]);
    c->gw_bc_u1 = (yu[0] - yv[0]) / (yu[1] - yv[0]);
    c->gw_bc_u3 = (yu[0] - yv[0]) / (yu[1] - yv[0]);
    c->gwi[0] = (yu[0] - yu[1]) / (yv[0] - yu[1]);
    c->gwi[1] = (yu[nyu + 1] - yu[nyu]) / (yv[nyv + 1] - yu[nyu]);
    /* dthetavi (declaration.f90:66) is never assigned by the reference, so
     * the zero-initialised module variable makes dtc_calc's v-term
     * 1/(u2m*dthetavi) = +inf (FOU3D.f90:642): it never sets dt. */
    c->dthetavi = 0.0;
    lu_buildp(c);

    size_t nc = c->ncols;
    size_t lu = jlen(c, UGRID), lv = jlen(c, VGRID), lp = jlen(c, PGRID);
    c->u1 = zalloc(2 * lu * nc);
    c->u2 = zalloc(2 * lv * nc);
    c->u3 = zalloc(2 * lu * nc);
    c->p = zalloc(2 * lp * nc);
    c->psi = zalloc(2 * lp * nc);
    c->div = zalloc(2 * lp * nc);
    c->Nu1 = zalloc(2 * (lu - 2) * nc);
    c->Nu2 = zalloc(2 * (lv - 2) * nc);
    c->Nu3 = zalloc(2 * (lu - 2) * nc);
    c->du1 = zalloc(2 * lu * nc);
    c->du2 = zalloc(2 * lv * nc);
    c->du3 = zalloc(2 * lu * nc);
    c->u1_itp = zalloc(2 * lv * nc);
    c->u2_itp = zalloc(2 * lu * nc);
    c->u3_itp = zalloc(2 * lv * nc);
    c->Nu1_dy = zalloc(2 * (lu - 2) * nc);
    c->Nu2_dy = zalloc(2 * (lv - 2) * nc);
    c->Nu3_dy = zalloc(2 * (lu - 2) * nc);
    c->uv_f = zalloc(2 * lv * nc);
    c->vv_c = zalloc(2 * lu * nc);
    c->wv_f = zalloc(2 * lv * nc);
    c->sav_nxz[0] = zalloc(2 * (lu - 2) * nc);
    c->sav_nxz[1] = zalloc(2 * (lv - 2) * nc);
    c->sav_nxz[2] = zalloc(2 * (lu - 2) * nc);
    size_t plane = (size_t)c->igal * c->kgal;
    size_t npl = nyu + 2; /* planes 0 .. nyu+1 */
    c->u1PL = zalloc(plane * npl);
    c->u2PL = zalloc(plane * npl);
    c->u3PL = zalloc(plane * npl);
    c->u1PL_itp = zalloc(plane * npl);
    c->u2PL_itp = zalloc(plane * npl);
    c->u3PL_itp = zalloc(plane * npl);
    c->Nu1PL = zalloc(plane * npl);
    c->Nu2PL = zalloc(plane * npl);
    c->Nu3PL = zalloc(plane * npl);
    c->uu_cPL = zalloc(plane * npl);
    c->uw_cPL = zalloc(plane * npl);
    c->vv_cPL = zalloc(plane * npl);
    c->ww_cPL = zalloc(plane * npl);
    c->uv_fPL = zalloc(plane * npl);
    c->wv_fPL = zalloc(plane * npl);
    c->a_ugrid = zalloc((size_t)3 * lu * c->nthr);
    c->a_vgrid = zalloc((size_t)3 * lv * c->nthr);
    c->u11 = zalloc(nyu + 2);
    c->mpgx = p->mpgx;
    c->dt = p->dt_fixed;
    c->dti = p->dt_fixed > 0 ? 1.0 / p->dt_fixed : 0.0;
    return c;
}

void lho_destroy(lho_ctx *c)
{
    if (!c) return;
    double **bufs[] = {&c->yu, &c->yv, &c->dthdyu, &c->dthdyv, &c->dyu2i, &c->dyv2i, &c->k1x, &c->k1z,
                       &c->k2x, &c->k2z, &c->DG, &c->u1, &c->u2, &c->u3, &c->p, &c->psi, &c->div,
                       &c->Nu1, &c->Nu2, &c->Nu3, &c->du1, &c->du2, &c->du3, &c->u1_itp, &c->u2_itp,
                       &c->u3_itp, &c->Nu1_dy, &c->Nu2_dy, &c->Nu3_dy, &c->uv_f, &c->vv_c, &c->wv_f,
                       &c->sav_nxz[0], &c->sav_nxz[1], &c->sav_nxz[2], &c->u1PL, &c->u2PL, &c->u3PL,
                       &c->u1PL_itp, &c->u2PL_itp, &c->u3PL_itp, &c->Nu1PL, &c->Nu2PL, &c->Nu3PL,
                       &c->uu_cPL, &c->uw_cPL, &c->vv_cPL, &c->ww_cPL, &c->uv_fPL, &c->wv_fPL,
                       &c->a_ugrid, &c->a_vgrid, &c->u11, &c->pp};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); i++) free(*bufs[i]);
    free(c->col_i);
    free(c->col_k);
    free(c->col_row);
    free(c);
}

void lho_sizes(const lho_ctx *c, int *o)
{
    o[0] = c->Nx;
    o[1] = c->Nz;
    o[2] = c->Mx;
    o[3] = c->Mz;
    o[4] = c->nyu;
    o[5] = c->nyv;
    o[6] = c->nyp;
    o[7] = c->ncols;
    o[8] = c->igal;
    o[9] = c->kgal;
}

static int copy_out(double *out, int cap, const double *src, int n)
{
    if (out && cap >= n) memcpy(out, src, sizeof(double) * n);
    return n;
}

int lho_get_array(const lho_ctx *c, int which, double *out, int cap)
{
    int nu = c->nyu + 2, nv = c->nyv + 2;
    switch (which) {
    case 0: return copy_out(out, cap, c->yu, nu);
    case 1: return copy_out(out, cap, c->yv, nv);
    case 2: return copy_out(out, cap, c->dthdyu, nu);
    case 3: return copy_out(out, cap, c->dthdyv, nv);
    case 4: return copy_out(out, cap, c->dyu2i, 3 * nu);
    case 5: return copy_out(out, cap, c->dyv2i, 3 * nv);
    case 6: {
        double s[8] = {c->gw[0], c->gw[1], c->gw_bc_u1, c->gw_bc_u3, c->gwi[0], c->gwi[1], c->dtv, c->ddthetavi};
        return copy_out(out, cap, s, 8);
    }
    case 7: return copy_out(out, cap, c->k1x, c->nxh);
    case 8: return copy_out(out, cap, c->k1z, c->Nz);
    case 9: return copy_out(out, cap, c->k2x, c->nxh);
    case 10: return copy_out(out, cap, c->k2z, c->Nz);
    case 11: return copy_out(out, cap, c->DG, 3 * c->nyu * c->ncols);
    default: return -1;
    }
}

static double *field_ptr(const lho_ctx *c, int f, int *len)
{
    size_t nc = c->ncols;
    int lu = jlen(c, UGRID), lv = jlen(c, VGRID), lp = jlen(c, PGRID);
    switch (f) {
    case 0: *len = 2 * lu * nc; return c->u1;
    case 1: *len = 2 * lv * nc; return c->u2;
    case 2: *len = 2 * lu * nc; return c->u3;
    case 3: *len = 2 * lp * nc; return c->p;
    case 4: *len = 2 * (lu - 2) * nc; return c->Nu1;
    case 5: *len = 2 * (lv - 2) * nc; return c->Nu2;
    case 6: *len = 2 * (lu - 2) * nc; return c->Nu3;
    case 7: *len = 2 * lp * nc; return c->div;
    case 8: *len = 2 * lp * nc; return c->psi;
    default: *len = 0; return NULL;
    }
}

int lho_field_len(const lho_ctx *c, int f)
{
    int n;
    field_ptr(c, f, &n);
    return n;
}

static double flowrate_im(const lho_ctx *c, const double *u1col);

void lho_set_field(lho_ctx *c, int f, const double *src)
{
    int n;
    double *p = field_ptr(c, f, &n);
    if (p) memcpy(p, src, sizeof(double) * n);
    if (f == 0) {
        /* getini after read_in (start.f90:1258-1267): Qx of the initial
         * field; the constant flow-rate mode keeps it as its target QxT */
        c->Qx = flowrate_im(c, c->u1);
        if (c->prm.flag_ctpress != 1) c->QxT = c->Qx;
        c->t = 0.0;
        c->iter = 0;
    }
}

void lho_get_field(const lho_ctx *c, int f, double *dst)
{
    int n;
    double *p = field_ptr(c, f, &n);
    if (p) memcpy(dst, p, sizeof(double) * n);
}

int lho_get_intermediate(const lho_ctx *c, int which, double *dst, int cap)
{
    size_t nc = c->ncols;
    int lu = jlen(c, UGRID), lv = jlen(c, VGRID);
    switch (which) {
    case 0: return copy_out(dst, cap, c->sav_nxz[0], 2 * (lu - 2) * nc);
    case 1: return copy_out(dst, cap, c->sav_nxz[1], 2 * (lv - 2) * nc);
    case 2: return copy_out(dst, cap, c->sav_nxz[2], 2 * (lu - 2) * nc);
    case 3: return copy_out(dst, cap, c->uv_f, 2 * lv * nc);
    case 4: return copy_out(dst, cap, c->vv_c, 2 * lu * nc);
    case 5: return copy_out(dst, cap, c->wv_f, 2 * lv * nc);
    default: return -1;
    }
}

double lho_get_scalar(const lho_ctx *c, int w)
{
    switch (w) {
    case 0: return c->t;
    case 1: return c->dt;
    case 2: return c->dti;
    case 3: return c->mpgx;
    case 4: return c->Qx;
    case 5: return c->QxT;
    case 6: return c->iter;
    case 7: return c->dtc;
    default: return 0.0;
    }
}

void lho_set_scalar(lho_ctx *c, int w, double v)
{
    switch (w) {
    case 0: c->t = v; break;
    case 1: c->dt = v; c->dti = 1.0 / v; break;
    case 2: c->dti = v; break;
    case 3: c->mpgx = v; break;
    case 4: c->Qx = v; break;
    case 5: c->QxT = v; break;
    case 6: c->iter = (int)v; break;
    case 7: c->dtc = v; break;
    }
}

int lho_column_i(const lho_ctx *c, int col) { return c->col_i[col]; }
int lho_column_k(const lho_ctx *c, int col) { return c->col_k[col]; }
int lho_column_row(const lho_ctx *c, int col) { return c->col_row[col]; }

/* ------------------------------------------------------------------ */
/* linear terms                                                         */

/* laplacian_U / laplacian_V (littleharsh.f90:281-368) fused into RHS0_u*
 * (littleharsh.f90:682-856) */
static void rhs0(lho_ctx *c, int kRK)
{
    int k = kRK - 1;
    double C1 = c->aRK[k] / c->prm.Re;
    double C2 = -c->cRK[k];
    int nc = c->ncols, lu = jlen(c, UGRID), lv = jlen(c, VGRID), lp = jlen(c, PGRID);
    int nyu = c->nyu;
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int col = 1; col <= nc; col++) {
        int i = c->col_i[col], kk = c->col_k[col];
        double k2x = c->k2x[i], k2z = c->k2z[kk - 1];
        /* u1 and u3 */
        for (int f = 0; f < 2; f++) {
            double *u = f == 0 ? c->u1 : c->u3;
            double *du = f == 0 ? c->du1 : c->du3;
            double *Nu = f == 0 ? c->Nu1 : c->Nu3;
            /* C3 = -dRK*k1F (real times purely imaginary complex) */
            double kim = f == 0 ? c->k1x[i] : c->k1z[kk - 1];
            double C3r = -c->dRK[k] * 0.0, C3i = -c->dRK[k] * kim;
            for (int j = 1; j <= nyu; j++) {
                const double *um = CX(u, 0, lu, j - 1, col), *u0 = CX(u, 0, lu, j, col),
                             *up = CX(u, 0, lu, j + 1, col);
                double d1 = c->dyu2i[0 + 3 * j], d2 = c->dyu2i[1 + 3 * j], d3 = c->dyu2i[2 + 3 * j];
                double cen = k2x + k2z + d2;
                double Lr = d1 * um[0] + cen * u0[0] + d3 * up[0];
                double Li = d1 * um[1] + cen * u0[1] + d3 * up[1];
                const double *nu = CX(Nu, 1, lu - 2, j, col);
                const double *pp = CX(c->p, 1, lp, j, col);
                double pr = C3r * pp[0] - C3i * pp[1];
                double pi = C3r * pp[1] + C3i * pp[0];
                double *d = CX(du, 0, lu, j, col);
                d[0] = C1 * Lr + C2 * nu[0] + pr;
                d[1] = C1 * Li + C2 * nu[1] + pi;
            }
        }
        /* u2 */
        for (int j = 1; j <= c->nyv; j++) {
            const double *um = CX(c->u2, 0, lv, j - 1, col), *u0 = CX(c->u2, 0, lv, j, col),
                         *up = CX(c->u2, 0, lv, j + 1, col);
            double d1 = c->dyv2i[0 + 3 * j], d2 = c->dyv2i[1 + 3 * j], d3 = c->dyv2i[2 + 3 * j];
            double cen = k2x + k2z + d2;
            double Lr = d1 * um[0] + cen * u0[0] + d3 * up[0];
            double Li = d1 * um[1] + cen * u0[1] + d3 * up[1];
            double C3 = -c->dRK[k] * c->ddthetavi * c->dthdyv[j];
            const double *nu = CX(c->Nu2, 1, lv - 2, j, col);
            const double *pp1 = CX(c->p, 1, lp, j + 1, col), *pp0 = CX(c->p, 1, lp, j, col);
            double *d = CX(c->du2, 0, lv, j, col);
            d[0] = C1 * Lr + C2 * nu[0] + C3 * (pp1[0] - pp0[0]);
            d[1] = C1 * Li + C2 * nu[1] + C3 * (pp1[1] - pp0[1]);
        }
    }
    /* mean pressure gradient on mode (0,0), littleharsh.f90:727-733 */
    double C1m = -c->dRK[k] * c->mpgx;
    for (int j = 1; j <= nyu; j++) CX(c->du1, 0, lu, j, 1)[0] += C1m;
}

/* ------------------------------------------------------------------ */
/* nonlinear (FOU3D.f90:51-371)                                         */

/* interp_u (FOU3D.f90:373-392): u/w centres -> v faces */
static void interp_u(lho_ctx *c, double *u_itp, const double *u)
{
    int nc = c->ncols, lu = jlen(c, UGRID), lv = jlen(c, VGRID);
    const double *yu = c->yu, *yv = c->yv;
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int col = 1; col <= nc; col++)
        for (int j = 0; j <= c->nyv + 1; j++) {
            const double *a = CX(u, 0, lu, j + 1, col), *b = CX(u, 0, lu, j, col);
            double w1 = yv[j] - yu[j], w2 = yu[j + 1] - yv[j], d = yu[j + 1] - yu[j];
            double *o = CX(u_itp, 0, lv, j, col);
            o[0] = (w1 * a[0] + w2 * b[0]) / d;
            o[1] = (w1 * a[1] + w2 * b[1]) / d;
        }
}

/* interp_v (FOU3D.f90:394-418): v faces -> u/w centres */
static void interp_v(lho_ctx *c, double *u_itp, const double *u)
{
    int nc = c->ncols, lu = jlen(c, UGRID), lv = jlen(c, VGRID);
    const double *yu = c->yu, *yv = c->yv;
    int nyu = c->nyu, nyv = c->nyv;
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int col = 1; col <= nc; col++) {
        for (int j = 1; j <= nyu; j++) {
            const double *a = CX(u, 0, lv, j, col), *b = CX(u, 0, lv, j - 1, col);
            double w1 = yu[j] - yv[j - 1], w2 = yv[j] - yu[j], d = yv[j] - yv[j - 1];
            double *o = CX(u_itp, 0, lu, j, col);
            o[0] = (w1 * a[0] + w2 * b[0]) / d;
            o[1] = (w1 * a[1] + w2 * b[1]) / d;
        }
        double *o0 = CX(u_itp, 0, lu, 0, col), *o1 = CX(u_itp, 0, lu, 1, col);
        const double *v0 = CX(u, 0, lv, 0, col);
        for (int r = 0; r < 2; r++) o0[r] = c->gwi[0] * (v0[r] - o1[r]) + o1[r];
        double *oT = CX(u_itp, 0, lu, nyu + 1, col), *oT1 = CX(u_itp, 0, lu, nyu, col);
        const double *vT = CX(u, 0, lv, nyv + 1, col);
        for (int r = 0; r < 2; r++) oT[r] = c->gwi[1] * (vT[r] - oT1[r]) + oT1[r];
    }
}

/* plane range of modes_to_planes_UVP / planes_to_modes_UVP at np = 1
 * (FOU3D.f90:743-751, 1732-1744; start.f90:1158-1194) */
static void uvp_range(const lho_ctx *c, int grid, int *jmin, int *jmax)
{
    int nyg = grid == UGRID ? c->nyu : (grid == VGRID ? c->nyv : c->nyp);
    int nyg_lb = grid == PGRID ? 1 : 0;
    int jlim1 = grid == PGRID ? 1 : 0;
    int jlim2 = grid == UGRID ? c->nyu + 1 : (grid == VGRID ? c->nyv + 1 : c->nyu);
    int pl1 = grid == PGRID ? 2 : 1, pl2 = c->nyu;
    int a = pl1 > jlim1 + 1 ? pl1 : jlim1 + 1;
    int b = pl2 < jlim2 - 1 ? pl2 : jlim2 - 1;
    if (a == nyg_lb + 1 && b >= a) a = a - 1;
    if (b == nyg && b >= a) b = b + 1;
    *jmin = a;
    *jmax = b;
}

/* modes_to_planes_UVP self part (FOU3D.f90:718-759) */
static void modes_to_planes(lho_ctx *c, double *xPL, const double *x, int grid)
{
    int jmin, jmax, len = jlen(c, grid), lo = jlo(grid);
    uvp_range(c, grid, &jmin, &jmax);
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int j = jmin; j <= jmax; j++)
        for (int col = 1; col <= c->ncols; col++) {
            int i = c->col_i[col], k = c->col_row[col];
            const double *v = CX(x, lo, len, j, col);
            *PL(c, xPL, 2 * i + 1, k, j) = v[0];
            *PL(c, xPL, 2 * i + 2, k, j) = v[1];
        }
}

/* planes_to_modes_UVP self part (FOU3D.f90:1694-1753) */
static void planes_to_modes_uvp(lho_ctx *c, double *x, const double *xPL, int grid)
{
    int jmin, jmax, len = jlen(c, grid), lo = jlo(grid);
    uvp_range(c, grid, &jmin, &jmax);
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int j = jmin; j <= jmax; j++)
        for (int col = 1; col <= c->ncols; col++) {
            int i = c->col_i[col], k = c->col_row[col];
            double *v = CX(x, lo, len, j, col);
            v[0] = *PL(c, xPL, 2 * i + 1, k, j);
            v[1] = *PL(c, xPL, 2 * i + 2, k, j);
        }
}

/* planes_to_modes_NUVP self part (FOU3D.f90:1911-1957): interior planes */
static void planes_to_modes_nuvp(lho_ctx *c, double *x, const double *xPL, int grid)
{
    int jlim2 = grid == UGRID ? c->nyu + 1 : c->nyv + 1;
    int jmin = 1, jmax = c->nyu < jlim2 - 1 ? c->nyu : jlim2 - 1;
    int len = jlim2 - 1;
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int j = jmin; j <= jmax; j++)
        for (int col = 1; col <= c->ncols; col++) {
            int i = c->col_i[col], k = c->col_row[col];
            double *v = CX(x, 1, len, j, col);
            v[0] = *PL(c, xPL, 2 * i + 1, k, j);
            v[1] = *PL(c, xPL, 2 * i + 2, k, j);
        }
}

static void four_to_phys_plane(lho_ctx *c, double *u, double *work)
{
    /* FOU3D.f90:668-677 for one field */
    for (int i = 1; i <= c->igal; i++) u[(i - 1) + c->igal * (c->Mz / 2)] = 0.0;
    lho_cft(u, c->igal, 2, (c->Nx + 2) / 2, 1, &c->cz, work);
    lho_rft(u, c->igal, c->Mz, 1, &c->rx, work);
}

static void phys_to_four_plane(lho_ctx *c, double *u, double *work)
{
    /* FOU3D.f90:1667-1670 */
    lho_rft(u, c->igal, c->Mz, -1, &c->rx, work);
    lho_cft(u, c->igal, 2, (c->Nx + 2) / 2, -1, &c->cz, work);
    for (int i = 1; i <= c->igal; i++) u[(i - 1) + c->igal * (c->Mz / 2)] = 0.0;
}

void lho_four_to_phys(lho_ctx *c, double *plane)
{
    double *w = zalloc(4 * (size_t)(c->Mx > c->Mz ? c->Mx : c->Mz) + 8);
    four_to_phys_plane(c, plane, w);
    free(w);
}

void lho_phys_to_four(lho_ctx *c, double *plane)
{
    double *w = zalloc(4 * (size_t)(c->Mx > c->Mz ? c->Mx : c->Mz) + 8);
    phys_to_four_plane(c, plane, w);
    free(w);
}

/* complex (im*kr) * (ur, ui) with the textbook product: (0*ur - kr*ui, 0*ui + kr*ur) */
static inline void mul_ik(double kr, const double *u, double *o)
{
    o[0] = 0.0 * u[0] - kr * u[1];
    o[1] = 0.0 * u[1] + kr * u[0];
}

/* der_x (FOU3D.f90:420-458) on the complex view u(0:Ngal_x/2, Ngal_z) */
void lho_der_x(const lho_ctx *c, const double *u, double *dudx)
{
    int Nx = c->Nx, Nz = c->Nz, Mx = c->Mx, Mz = c->Mz, ig = c->igal;
#define UC(i, k) (u + 2 * (i) + (size_t)ig * ((k) - 1))
#define DC(i, k) (dudx + 2 * (i) + (size_t)ig * ((k) - 1))
    for (int k = 1; k <= Nz / 2; k++) {
        for (int i = 0; i <= Nx / 2; i++) mul_ik(c->k1x[i], UC(i, k), DC(i, k));
        for (int i = Nx / 2 + 1; i <= Mx / 2; i++) DC(i, k)[0] = DC(i, k)[1] = 0.0;
    }
    for (int k = Nz / 2 + 1; k <= Mz - Nz / 2 + 1; k++)
        for (int i = 0; i <= Mx / 2; i++) DC(i, k)[0] = DC(i, k)[1] = 0.0;
    for (int k = Mz - Nz / 2 + 2; k <= Mz; k++) {
        for (int i = 0; i <= Nx / 2; i++) mul_ik(c->k1x[i], UC(i, k), DC(i, k));
        for (int i = Nx / 2 + 1; i <= Mx / 2; i++) DC(i, k)[0] = DC(i, k)[1] = 0.0;
    }
}

/* der_z (FOU3D.f90:483-523) */
void lho_der_z(const lho_ctx *c, const double *u, double *dudz)
{
    int Nx = c->Nx, Nz = c->Nz, Mx = c->Mx, Mz = c->Mz, ig = c->igal;
    int dk2 = Nz - Mz;
#undef DC
#define DC(i, k) (dudz + 2 * (i) + (size_t)ig * ((k) - 1))
    for (int k = 1; k <= Nz / 2; k++) {
        for (int i = 0; i <= Nx / 2; i++) mul_ik(c->k1z[k - 1], UC(i, k), DC(i, k));
        for (int i = Nx / 2 + 1; i <= Mx / 2; i++) DC(i, k)[0] = DC(i, k)[1] = 0.0;
    }
    for (int k = Nz / 2 + 1; k <= Mz - Nz / 2 + 1; k++)
        for (int i = 0; i <= Mx / 2; i++) DC(i, k)[0] = DC(i, k)[1] = 0.0;
    for (int k = Mz - Nz / 2 + 2; k <= Mz; k++) {
        int k2 = k + dk2;
        for (int i = 0; i <= Nx / 2; i++) mul_ik(c->k1z[k2 - 1], UC(i, k), DC(i, k));
        for (int i = Nx / 2 + 1; i <= Mx / 2; i++) DC(i, k)[0] = DC(i, k)[1] = 0.0;
    }
#undef UC
#undef DC
}

/* ops_in_planes2 (FOU3D.f90:1514-1652) */
static void ops_in_planes2(lho_ctx *c)
{
    int Mx = c->Mx, Mz = c->Mz, ig = c->igal;
    size_t plane = (size_t)ig * c->kgal;
    int nwork = 4 * (Mx > Mz ? Mx : Mz) + 8;
#pragma omp parallel num_threads(c->nthr)
    {
        double *w = zalloc(nwork);
        double *d1 = zalloc(plane), *d2 = zalloc(plane);
#pragma omp for schedule(static)
        for (int j = 1; j <= c->nyu; j++) {
            double *u1 = PLANE(c, c->u1PL, j), *u2 = PLANE(c, c->u2PL_itp, j), *u3 = PLANE(c, c->u3PL, j);
            four_to_phys_plane(c, u1, w);
            four_to_phys_plane(c, u2, w);
            four_to_phys_plane(c, u3, w);
            double *uu = PLANE(c, c->uu_cPL, j), *uw = PLANE(c, c->uw_cPL, j);
            double *vv = PLANE(c, c->vv_cPL, j), *ww = PLANE(c, c->ww_cPL, j);
            for (int k = 0; k < Mz; k++)
                for (int i = 0; i < Mx; i++) {
                    size_t q = i + (size_t)ig * k;
                    uu[q] = u1[q] * u1[q];
                    uw[q] = u1[q] * u3[q];
                    vv[q] = u2[q] * u2[q];
                    ww[q] = u3[q] * u3[q];
                }
            phys_to_four_plane(c, uu, w);
            phys_to_four_plane(c, uw, w);
            phys_to_four_plane(c, vv, w);
            phys_to_four_plane(c, ww, w);
            double *N1 = PLANE(c, c->Nu1PL, j), *N3 = PLANE(c, c->Nu3PL, j);
            lho_der_x(c, uu, d1);
            lho_der_z(c, uw, d2);
            for (int k = 0; k < Mz; k++)
                for (int i = 0; i < Mx; i++) N1[i + (size_t)ig * k] = d1[i + (size_t)ig * k] + d2[i + (size_t)ig * k];
            lho_der_x(c, uw, d1);
            lho_der_z(c, ww, d2);
            for (int k = 0; k < Mz; k++)
                for (int i = 0; i < Mx; i++) N3[i + (size_t)ig * k] = d1[i + (size_t)ig * k] + d2[i + (size_t)ig * k];
        }
#pragma omp for schedule(static)
        for (int j = 1; j <= c->nyu; j++) {
            double *u1 = PLANE(c, c->u1PL_itp, j), *u2 = PLANE(c, c->u2PL, j), *u3 = PLANE(c, c->u3PL_itp, j);
            four_to_phys_plane(c, u1, w);
            four_to_phys_plane(c, u2, w);
            four_to_phys_plane(c, u3, w);
            double *uv = PLANE(c, c->uv_fPL, j), *wv = PLANE(c, c->wv_fPL, j);
            for (int k = 0; k < Mz; k++)
                for (int i = 0; i < Mx; i++) {
                    size_t q = i + (size_t)ig * k;
                    uv[q] = u1[q] * u2[q];
                    wv[q] = u3[q] * u2[q];
                }
            phys_to_four_plane(c, uv, w);
            phys_to_four_plane(c, wv, w);
            double *N2 = PLANE(c, c->Nu2PL, j);
            lho_der_x(c, uv, d1);
            lho_der_z(c, wv, d2);
            for (int k = 0; k < Mz; k++)
                for (int i = 0; i < Mx; i++) N2[i + (size_t)ig * k] = d1[i + (size_t)ig * k] + d2[i + (size_t)ig * k];
        }
        free(w);
        free(d1);
        free(d2);
    }
}

/* dtc_calc (FOU3D.f90:613-651) with its explicit-shape dummies: dummy plane
 * j of u1/u2/u3 is actual plane j-1 of the arrays passed in (planes 0..nyu
 * are allocated from jgal-1), so the scan covers actual planes 0..nyu-1 and
 * pairs dthdyv(j) with actual plane j-1. */
static double dtc_calc(lho_ctx *c)
{
    size_t plane = (size_t)c->igal * c->kgal;
    int npl = c->nyu; /* dummy planes 1..nyu */
    double u1m = 0.0, u3m = 0.0, u2m = 1e-6;
    for (size_t q = 0; q < plane * npl; q++) {
        double a = fabs(c->u1PL[q]);
        if (a > u1m) u1m = a;
        double b = fabs(c->u3PL[q]);
        if (b > u3m) u3m = b;
    }
    for (int jd = 1; jd <= npl; jd++) {
        const double *pl = PLANE(c, c->u2PL, jd - 1);
        for (int k = 0; k < c->kgal; k++)
            for (int i = 0; i < c->igal - 2; i++) {
                double v = fabs(pl[i + (size_t)c->igal * k]) * c->dthdyv[jd];
                if (v > u2m) u2m = v;
            }
    }
    double a = 1.0 / (c->prm.alp * (c->Nx / 2) * u1m);
    double b = 1.0 / (c->prm.bet * (c->Nz / 2) * u3m);
    double d = 1.0 / (u2m * c->dthetavi);
    double m = a < b ? a : b;
    return m < d ? m : d;
}

static void nonlinear(lho_ctx *c, int kRK)
{
    size_t plane = (size_t)c->igal * c->kgal;
    size_t npl = c->nyu + 2;
    int nc = c->ncols, lu = jlen(c, UGRID), lv = jlen(c, VGRID);
    /* FOU3D.f90:98-118 */
    memset(c->u1PL_itp, 0, sizeof(double) * plane * npl);
    memset(c->u2PL_itp, 0, sizeof(double) * plane * npl);
    memset(c->u3PL_itp, 0, sizeof(double) * plane * npl);
    interp_u(c, c->u1_itp, c->u1);
    interp_v(c, c->u2_itp, c->u2);
    interp_u(c, c->u3_itp, c->u3);
    memset(c->u1PL, 0, sizeof(double) * plane * npl);
    memset(c->u2PL, 0, sizeof(double) * plane * npl);
    memset(c->u3PL, 0, sizeof(double) * plane * npl);
    memset(c->Nu1PL, 0, sizeof(double) * plane * npl);
    memset(c->Nu2PL, 0, sizeof(double) * plane * npl);
    memset(c->Nu3PL, 0, sizeof(double) * plane * npl);
    /* FOU3D.f90:126-131 */
    modes_to_planes(c, c->u1PL, c->u1, UGRID);
    modes_to_planes(c, c->u2PL, c->u2, VGRID);
    modes_to_planes(c, c->u3PL, c->u3, UGRID);
    modes_to_planes(c, c->u1PL_itp, c->u1_itp, VGRID);
    modes_to_planes(c, c->u2PL_itp, c->u2_itp, UGRID);
    modes_to_planes(c, c->u3PL_itp, c->u3_itp, VGRID);
    ops_in_planes2(c);
    /* FOU3D.f90:248-261 */
    planes_to_modes_uvp(c, c->uv_f, c->uv_fPL, VGRID);
    planes_to_modes_uvp(c, c->vv_c, c->vv_cPL, UGRID);
    planes_to_modes_uvp(c, c->wv_f, c->wv_fPL, VGRID);
    planes_to_modes_nuvp(c, c->Nu1, c->Nu1PL, UGRID);
    planes_to_modes_nuvp(c, c->Nu2, c->Nu2PL, VGRID);
    planes_to_modes_nuvp(c, c->Nu3, c->Nu3PL, UGRID);
    memcpy(c->sav_nxz[0], c->Nu1, sizeof(double) * 2 * (lu - 2) * nc);
    memcpy(c->sav_nxz[1], c->Nu2, sizeof(double) * 2 * (lv - 2) * nc);
    memcpy(c->sav_nxz[2], c->Nu3, sizeof(double) * 2 * (lu - 2) * nc);
    /* der_yu_h / der_yv_h and the sum (FOU3D.f90:268-281, 550-590) */
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int col = 1; col <= nc; col++) {
        for (int j = 1; j <= c->nyu; j++) {
            const double *a = CX(c->uv_f, 0, lv, j, col), *b = CX(c->uv_f, 0, lv, j - 1, col);
            const double *e = CX(c->wv_f, 0, lv, j, col), *f = CX(c->wv_f, 0, lv, j - 1, col);
            double *n1 = CX(c->Nu1, 1, lu - 2, j, col), *n3 = CX(c->Nu3, 1, lu - 2, j, col);
            double m = c->dthdyu[j], dv = c->ddthetavi;
            for (int r = 0; r < 2; r++) {
                double d1 = (a[r] - b[r]) * m * dv;
                double d3 = (e[r] - f[r]) * m * dv;
                n1[r] = n1[r] + d1;
                n3[r] = n3[r] + d3;
            }
        }
        for (int j = 1; j <= c->nyv; j++) {
            const double *a = CX(c->vv_c, 0, lu, j + 1, col), *b = CX(c->vv_c, 0, lu, j, col);
            double *n2 = CX(c->Nu2, 1, lv - 2, j, col);
            double m = c->dthdyv[j], dv = c->ddthetavi;
            for (int r = 0; r < 2; r++) {
                double d2 = (a[r] - b[r]) * m * dv;
                n2[r] = n2[r] + d2;
            }
        }
    }
    /* CFL (FOU3D.f90:290-303) */
    if (kRK == 1) {
        if (c->prm.dt_mode == LHO_DT_CFL) {
            c->dtc = dtc_calc(c);
            double a = 2.5 * c->dtv, b = c->prm.CFL * c->dtc;
            c->dt = a < b ? a : b;
        } else {
            c->dt = c->prm.dt_fixed;
        }
        c->dti = 1.0 / c->dt;
        c->t = c->t + c->dt;
    }
    /* FOU3D.f90:359-368 */
    double C1 = -c->gRK[kRK - 1];
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int col = 1; col <= nc; col++) {
        for (int j = 1; j <= c->nyu; j++) {
            double *d1 = CX(c->du1, 0, lu, j, col), *d3 = CX(c->du3, 0, lu, j, col);
            const double *n1 = CX(c->Nu1, 1, lu - 2, j, col), *n3 = CX(c->Nu3, 1, lu - 2, j, col);
            for (int r = 0; r < 2; r++) {
                d1[r] = d1[r] + C1 * n1[r];
                d3[r] = d3[r] + C1 * n3[r];
            }
        }
        for (int j = 1; j <= c->nyv; j++) {
            double *d2 = CX(c->du2, 0, lv, j, col);
            const double *n2 = CX(c->Nu2, 1, lv - 2, j, col);
            for (int r = 0; r < 2; r++) d2[r] = d2[r] + C1 * n2[r];
        }
    }
}

/* ------------------------------------------------------------------ */
/* tridiagonal solves                                                   */

/* LU_build + LU_dec (tridLU_3D.f90:163-221, 327-364) for one column */
static void lu_build_dec(const lho_ctx *c, int grid, int col, int kRK, double *a)
{
    int ns = 0, ne = grid == UGRID ? c->nyu + 1 : c->nyv + 1;
    double beta = c->bRK[kRK - 1] * c->dt / c->prm.Re;
    double k2x = c->k2x[c->col_i[col]], k2z = c->k2z[c->col_k[col] - 1];
    const double *d = grid == UGRID ? c->dyu2i : c->dyv2i;
#define A(r, j) a[(r) - 1 + 3 * ((j) - ns)]
    A(1, ns) = 0.0;
    A(2, ns) = 1.0;
    A(3, ns) = grid == UGRID ? c->gw[0] : 0.0;
    for (int j = ns + 1; j <= ne - 1; j++) {
        A(1, j) = -beta * d[0 + 3 * j];
        A(2, j) = 1.0 - beta * (d[1 + 3 * j] + k2x + k2z);
        A(3, j) = -beta * d[2 + 3 * j];
    }
    A(1, ne) = grid == UGRID ? c->gw[1] : 0.0;
    A(2, ne) = 1.0;
    A(3, ne) = 0.0;
    A(2, ns) = 1.0 / A(2, ns);
    for (int j = ns + 1; j <= ne; j++) {
        A(3, j - 1) = A(3, j - 1) * A(2, j - 1);
        A(2, j) = 1.0 / (A(2, j) - A(1, j) * A(3, j - 1));
    }
#undef A
}

/* LUsolU (tridLU_3D.f90:38-94) for every column */
static void lusolu(lho_ctx *c, int grid, int kRK, const double *rhs, double *u)
{
    int ns = 0, ne = grid == UGRID ? c->nyu + 1 : c->nyv + 1, len = ne - ns + 1;
#pragma omp parallel num_threads(c->nthr)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *a = (grid == UGRID ? c->a_ugrid : c->a_vgrid) + (size_t)3 * len * tid;
#pragma omp for schedule(static)
        for (int col = 1; col <= c->ncols; col++) {
            lu_build_dec(c, grid, col, kRK, a);
#define A(r, j) a[(r) - 1 + 3 * ((j) - ns)]
            const double *rh0 = CX(rhs, 0, len, ns, col);
            double *u0 = CX(u, 0, len, ns, col);
            u0[0] = rh0[0] * A(2, ns);
            u0[1] = rh0[1] * A(2, ns);
            for (int j = ns + 1; j <= ne; j++) {
                const double *rh = CX(rhs, 0, len, j, col);
                const double *um = CX(u, 0, len, j - 1, col);
                double *uj = CX(u, 0, len, j, col);
                uj[0] = (rh[0] - A(1, j) * um[0]) * A(2, j);
                uj[1] = (rh[1] - A(1, j) * um[1]) * A(2, j);
            }
            for (int j = ne - 1; j >= ns; j--) {
                double *uj = CX(u, 0, len, j, col);
                const double *up = CX(u, 0, len, j + 1, col);
                uj[0] = uj[0] - A(3, j) * up[0];
                uj[1] = uj[1] - A(3, j) * up[1];
            }
#undef A
        }
    }
}

void lho_lusolu(lho_ctx *c, int grid, int kRK, const double *rhs, double *u) { lusolu(c, grid, kRK, rhs, u); }

/* LU_build + LU_dec of every column of a velocity grid, a(3, j, column) */
void lho_lu_factor(const lho_ctx *c, int grid, int kRK, double *a)
{
    int len = grid == UGRID ? c->nyu + 2 : c->nyv + 2;
    for (int col = 1; col <= c->ncols; col++) lu_build_dec(c, grid, col, kRK, a + (size_t)3 * len * (col - 1));
}

/* LUsolP (tridLU_3D.f90:98-132) */
void lho_lusolp(const lho_ctx *c, double *x)
{
    int ns = 1, ne = c->nyu, len = ne - ns + 1;
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int col = 1; col <= c->ncols; col++) {
#define G(r, j) c->DG[((r) - 1) + 3 * ((size_t)((j) - ns) + (size_t)len * (col - 1))]
        double *x0 = CX(x, 1, len, ns, col);
        x0[0] = x0[0] * G(2, ns);
        x0[1] = x0[1] * G(2, ns);
        for (int j = ns + 1; j <= ne; j++) {
            double *xj = CX(x, 1, len, j, col);
            const double *xm = CX(x, 1, len, j - 1, col);
            xj[0] = (xj[0] - G(1, j) * xm[0]) * G(2, j);
            xj[1] = (xj[1] - G(1, j) * xm[1]) * G(2, j);
        }
        for (int j = ne - 1; j >= ns; j--) {
            double *xj = CX(x, 1, len, j, col);
            const double *xp = CX(x, 1, len, j + 1, col);
            xj[0] = xj[0] - G(3, j) * xp[0];
            xj[1] = xj[1] - G(3, j) * xp[1];
        }
#undef G
    }
}

/* solveU (littleharsh.f90:863-894) */
static void solve_u(lho_ctx *c, double *u, double *du, int grid, int kRK)
{
    int len = jlen(c, grid), ne = len - 1;
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int col = 1; col <= c->ncols; col++) {
        double *d0 = CX(du, 0, len, 0, col);
        d0[0] = d0[1] = 0.0;
        for (int j = 1; j <= ne - 1; j++) {
            double *d = CX(du, 0, len, j, col);
            const double *uu = CX(u, 0, len, j, col);
            d[0] = uu[0] + c->dt * d[0];
            d[1] = uu[1] + c->dt * d[1];
        }
        double *dT = CX(du, 0, len, ne, col);
        dT[0] = dT[1] = 0.0;
    }
    lusolu(c, grid, kRK, du, u);
}

/* divergence (littleharsh.f90:242-278) */
static void divergence(lho_ctx *c)
{
    int lu = jlen(c, UGRID), lv = jlen(c, VGRID), lp = jlen(c, PGRID);
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int col = 1; col <= c->ncols; col++) {
        double kx = c->k1x[c->col_i[col]], kz = c->k1z[c->col_k[col] - 1];
        for (int j = 1; j <= c->nyu; j++) {
            double a[2], b[2];
            mul_ik(kx, CX(c->u1, 0, lu, j, col), a);
            mul_ik(kz, CX(c->u3, 0, lu, j, col), b);
            const double *v0 = CX(c->u2, 0, lv, j, col), *vm = CX(c->u2, 0, lv, j - 1, col);
            double m = c->ddthetavi * c->dthdyu[j];
            double *d = CX(c->div, 1, lp, j, col);
            d[0] = a[0] + b[0] + m * (v0[0] - vm[0]);
            d[1] = a[1] + b[1] + m * (v0[1] - vm[1]);
        }
    }
}

/* solveP (littleharsh.f90:626-680) */
static void solve_p(lho_ctx *c, int kRK)
{
    int lp = jlen(c, PGRID);
    double dtirk = c->dti / (c->aRK[kRK - 1] + c->bRK[kRK - 1]);
    divergence(c);
    size_t n = (size_t)lp * c->ncols;
    for (size_t q = 0; q < 2 * n; q++) c->psi[q] = dtirk * c->div[q];
    c->psi[0] = 0.0;
    c->psi[1] = 0.0;
    lho_lusolp(c, c->psi);
    for (size_t q = 0; q < 2 * n; q++) c->p[q] = c->p[q] + c->psi[q];
}

/* v_corr (littleharsh.f90:896-993) */
static void v_corr(lho_ctx *c, int kRK)
{
    int lu = jlen(c, UGRID), lv = jlen(c, VGRID), lp = jlen(c, PGRID);
    double dtrk = c->dt * (c->aRK[kRK - 1] + c->bRK[kRK - 1]);
    double dtrk_u2 = dtrk * c->ddthetavi;
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int col = 1; col <= c->ncols; col++) {
        /* kx = dtrk*k1F_x(i): (dtrk*0, dtrk*kxr) */
        double kxr = dtrk * c->k1x[c->col_i[col]], kxre = dtrk * 0.0;
        double kzr = dtrk * c->k1z[c->col_k[col] - 1], kzre = dtrk * 0.0;
        for (int j = 1; j <= c->nyu; j++) {
            const double *ps = CX(c->psi, 1, lp, j, col);
            double *u = CX(c->u1, 0, lu, j, col);
            double pr = kxre * ps[0] - kxr * ps[1], pi = kxre * ps[1] + kxr * ps[0];
            u[0] = u[0] - pr;
            u[1] = u[1] - pi;
        }
        double *a0 = CX(c->u1, 0, lu, 0, col), *a1 = CX(c->u1, 0, lu, 1, col);
        a0[0] = c->gw_bc_u1 * a1[0];
        a0[1] = c->gw_bc_u1 * a1[1];
        double *aT = CX(c->u1, 0, lu, c->nyu + 1, col), *aT1 = CX(c->u1, 0, lu, c->nyu, col);
        aT[0] = c->gw_bc_u1 * aT1[0];
        aT[1] = c->gw_bc_u1 * aT1[1];
        for (int j = 1; j <= c->nyv; j++) {
            const double *p1 = CX(c->psi, 1, lp, j + 1, col), *p0 = CX(c->psi, 1, lp, j, col);
            double *v = CX(c->u2, 0, lv, j, col);
            double m = dtrk_u2 * c->dthdyv[j];
            v[0] = v[0] - m * (p1[0] - p0[0]);
            v[1] = v[1] - m * (p1[1] - p0[1]);
        }
        double *v0 = CX(c->u2, 0, lv, 0, col), *vT = CX(c->u2, 0, lv, c->nyv + 1, col);
        v0[0] = v0[1] = vT[0] = vT[1] = 0.0;
        for (int j = 1; j <= c->nyu; j++) {
            const double *ps = CX(c->psi, 1, lp, j, col);
            double *u = CX(c->u3, 0, lu, j, col);
            double pr = kzre * ps[0] - kzr * ps[1], pi = kzre * ps[1] + kzr * ps[0];
            u[0] = u[0] - pr;
            u[1] = u[1] - pi;
        }
        double *w0 = CX(c->u3, 0, lu, 0, col), *w1 = CX(c->u3, 0, lu, 1, col);
        w0[0] = c->gw_bc_u3 * w1[0];
        w0[1] = c->gw_bc_u3 * w1[1];
        double *wT = CX(c->u3, 0, lu, c->nyu + 1, col), *wT1 = CX(c->u3, 0, lu, c->nyu, col);
        wT[0] = c->gw_bc_u3 * wT1[0];
        wT[1] = c->gw_bc_u3 * wT1[1];
    }
    divergence(c);
}

/* flowrateIm (littleharsh.f90:473-492): Re(u) on the u grid, yv widths */
static double flowrate_im(const lho_ctx *c, const double *u1col)
{
    double Qu = 0.0;
    int nn = c->nyv;
    for (int j = 1; j <= nn + 1; j++) Qu = Qu + (c->yv[j] - c->yv[j - 1]) * u1col[2 * j];
    return Qu;
}

/* flowrate_corr (littleharsh.f90:515-548) with LUsol0/LU_build0
 * (tridLU_3D.f90:134-160, 299-325).  flowrateRe's dummy is declared
 * u(1:nn+2) and receives u11(0:nn+2), so its u(j) is u11(j-1). */
static void flowrate_corr(lho_ctx *c, int kRK)
{
    int nn = c->nyv, ns = 0, ne = nn + 2;
    double *u11 = c->u11;
    double bdt = -c->dRK[kRK - 1] * c->dt;
    u11[0] = 0.0;
    for (int j = 1; j <= nn + 1; j++) u11[j] = bdt;
    u11[nn + 2] = 0.0;
    double *a = zalloc((size_t)3 * (ne - ns + 1));
#define A(r, j) a[(r) - 1 + 3 * ((j) - ns)]
    double beta = c->bRK[kRK - 1] * c->dt / c->prm.Re;
    A(1, ns) = 0.0;
    A(2, ns) = 1.0;
    A(3, ns) = c->gw[0];
    for (int j = ns + 1; j <= ne - 1; j++) {
        A(1, j) = -beta * c->dyu2i[0 + 3 * j];
        A(2, j) = 1.0 - beta * c->dyu2i[1 + 3 * j];
        A(3, j) = -beta * c->dyu2i[2 + 3 * j];
    }
    A(1, ne) = c->gw[1];
    A(2, ne) = 1.0;
    A(3, ne) = 0.0;
    A(2, ns) = 1.0 / A(2, ns);
    for (int j = ns + 1; j <= ne; j++) {
        A(3, j - 1) = A(3, j - 1) * A(2, j - 1);
        A(2, j) = 1.0 / (A(2, j) - A(1, j) * A(3, j - 1));
    }
    u11[ns] = u11[ns] * A(2, ns);
    for (int j = ns + 1; j <= ne; j++) u11[j] = (u11[j] - A(1, j) * u11[j - 1]) * A(2, j);
    for (int j = ne - 1; j >= ns; j--) u11[j] = u11[j] - A(3, j) * u11[j + 1];
#undef A
    free(a);
    double Qx1 = 0.0;
    for (int j = 1; j <= nn + 1; j++) Qx1 = Qx1 + (c->yv[j] - c->yv[j - 1]) * u11[j - 1];
    double Qx0 = flowrate_im(c, c->u1);
    double g = (c->QxT - Qx0) / Qx1;
    c->mpgx = c->mpgx + g;
    c->dgx = g;
    for (int j = 0; j <= nn + 2; j++) c->u1[2 * j] = c->u1[2 * j] + g * u11[j];
}

void lho_substep(lho_ctx *c, int kRK)
{
    c->kRK = kRK;
    rhs0(c, kRK);
    nonlinear(c, kRK);
    solve_u(c, c->u1, c->du1, UGRID, kRK);
    solve_u(c, c->u2, c->du2, VGRID, kRK);
    solve_u(c, c->u3, c->du3, UGRID, kRK);
    if (c->prm.flag_ctpress == 0) flowrate_corr(c, kRK);
    solve_p(c, kRK);
    v_corr(c, kRK);
}

void lho_step(lho_ctx *c, int nsteps)
{
    for (int s = 0; s < nsteps; s++) {
        for (int k = 1; k <= 3; k++) lho_substep(c, k);
        if (c->prm.flag_ctpress == 1) c->Qx = flowrate_im(c, c->u1);
        c->iter = c->iter + 1;
    }
}

/* spectra (spectra.f90:7-66): buildsp per field, buildspUV with u2_itp */
void lho_spectra(lho_ctx *c, double *spU, double *spV, double *spW, double *spUV, double *spP)
{
    const int nc = c->ncols, lu = jlen(c, UGRID), lv = jlen(c, VGRID), lp = jlen(c, PGRID);
    double *itp = (double *)malloc(sizeof(double) * 2 * (size_t)lu * nc);
    interp_v(c, itp, c->u2);
    for (int col = 1; col <= nc; col++) {
        for (int j = 0; j < lu; j++) {
            const size_t q = (size_t)(col - 1) * lu + j;
            const double *a = CX(c->u1, 0, lu, j, col), *w = CX(c->u3, 0, lu, j, col), *v = CX(itp, 0, lu, j, col);
            spU[q] = spU[q] + a[0] * a[0] + a[1] * a[1];
            spW[q] = spW[q] + w[0] * w[0] + w[1] * w[1];
            spUV[q] = spUV[q] + a[0] * v[0] + a[1] * v[1];
        }
        for (int j = 0; j < lv; j++) {
            const size_t q = (size_t)(col - 1) * lv + j;
            const double *a = CX(c->u2, 0, lv, j, col);
            spV[q] = spV[q] + a[0] * a[0] + a[1] * a[1];
        }
        for (int j = 1; j <= lp; j++) {
            const size_t q = (size_t)(col - 1) * lp + (j - 1);
            const double *a = CX(c->p, 1, lp, j, col);
            spP[q] = spP[q] + a[0] * a[0] + a[1] * a[1];
        }
    }
    free(itp);
}

/* The pressure planes stats() reads: nonlinear() refills ppPL from p at
 * every output step (FOU3D.f90:149-152), and stats() runs only at kRK = 1
 * (FOU3D.f90:290-341), so it sees p as of the latest output step. */
void lho_pressure_snapshot(lho_ctx *c)
{
    const size_t n = 2 * (size_t)jlen(c, PGRID) * c->ncols;
    if (!c->pp) c->pp = zalloc(n);
    memcpy(c->pp, c->p, n * sizeof(double));
}

/* der_z_N (FOU3D.f90:525-546): dudz(i,k) = kz(k) u(i,k) on the complex view
 * (0:Nx/2, Nz) of an (Nx+2) x Nz real plane, every row, no masking; kz_im
 * holds the imaginary parts of kz(1:Nz) */
void lho_der_z_n(const double *u, double *dudz, const double *kz_im, int Nx, int Nz)
{
    const int ign = Nx + 2;
    for (int k = 1; k <= Nz; k++)
        for (int i = 0; i <= Nx / 2; i++)
            mul_ik(kz_im[k - 1], u + 2 * i + (size_t)ign * (k - 1), dudz + 2 * i + (size_t)ign * (k - 1));
}

/* omega_x at the v faces as nonlinear() forms it before stats()
 * (FOU3D.f90:314-338), plane by plane: u2PLN = 0 and modes_to_planes_phys
 * of u2 (FOU3D.f90:816-860: dk_phys = 0, planes 0..nyv+1), der_z_N with
 * k1F_z, der_yv_h_wx (FOU3D.f90:592-610) placed the same way, wx = -wx +
 * du3dy over planes 0..nyu+1 (FOU3D.f90:331-336) and four_to_phys_N
 * (FOU3D.f90:700-714: cft then rft of the Nspec sizes, no row zeroed).
 * Plane nyu+1, which the transposes never write, holds zeros.
 * wx: (nyu+2) planes of (Nx+2) x Nz reals. */
void lho_omega_x(lho_ctx *c, double *wx)
{
    const int Nx = c->Nx, Nz = c->Nz, ign = Nx + 2, nyv = c->nyv, nyu = c->nyu;
    const int lu = jlen(c, UGRID), lv = jlen(c, VGRID);
    const size_t plane = (size_t)ign * Nz;
    const int nwork = 4 * (Nx > Nz ? Nx : Nz) + 8;
#pragma omp parallel num_threads(c->nthr)
    {
        double *w = zalloc(nwork), *u2pl = zalloc(plane), *dy = zalloc(plane);
#pragma omp for schedule(static)
        for (int j = 0; j <= nyu + 1; j++) {
            double *P = wx + plane * j;
            memset(u2pl, 0, plane * sizeof(double));
            memset(dy, 0, plane * sizeof(double));
            if (j <= nyv + 1) {
                const double dth = c->dthdyv[j];
                for (int col = 1; col <= c->ncols; col++) {
                    const int i = c->col_i[col], k = c->col_k[col];
                    const double *v = CX(c->u2, 0, lv, j, col);
                    const double *a = CX(c->u3, 0, lu, j + 1, col), *b = CX(c->u3, 0, lu, j, col);
                    const size_t o = 2 * (size_t)i + (size_t)ign * (k - 1);
                    u2pl[o] = v[0];
                    u2pl[o + 1] = v[1];
                    dy[o] = (a[0] - b[0]) * dth * c->ddthetavi;
                    dy[o + 1] = (a[1] - b[1]) * dth * c->ddthetavi;
                }
            }
            lho_der_z_n(u2pl, P, c->k1z, Nx, Nz);
            for (size_t e = 0; e < plane; e++) P[e] = -P[e] + dy[e];
            lho_cft(P, ign, 2, (Nx + 2) / 2, 1, &c->czN, w);
            lho_rft(P, ign, Nz, 1, &c->rxN, w);
        }
        free(w);
        free(u2pl);
        free(dy);
    }
}

/* stats (stats.f90:1-97) at a flagged output step.  nonlinear() calls it
 * (FOU3D.f90:307-341) after ops_in_planes2 (FOU3D.f90:240), which has run
 * four_to_phys_u in place on planes 1..nyu of u1PL, u2PL_itp, u3PL
 * (FOU3D.f90:1541) and of u1PL_itp, u2PL, u3PL_itp (FOU3D.f90:1584; the v
 * planes reach nyv+1 = nyu at one rank).  So on those planes the sums run over
 * physical values, on the wall planes 0 and nyu+1 over the spectral
 * coefficients modes_to_planes_UVP placed (zeros where it placed none):
 * entries i = 1..igal-2, rows k = 1..kgal, planes limPL_incw (0..nyu+1 for u
 * and v, 1..nyu+1 for p).  P sums read the pressure planes of the latest
 * lho_pressure_snapshot (spectral, as modes_to_planes_UVP left them); wx sums
 * run over the physical omega_x of lho_omega_x, i = 1..Nx, k = 1..Nz.
 * acc[q*(nyu+2) + j]: q 0 Um, 1 U2m, 2 Vm, 3 V2m, 4 Wm, 5 W2m, 6 UVm (u1 x
 * u2PL_itp), 7 UWm, 8 VWm (u2 x u3PL_itp), 9 Pm, 10 P2m, 11 wxm, 12 wx2m. */
void lho_stats(lho_ctx *c, double *acc)
{
    const int nyu = c->nyu, nc = c->ncols, lu = jlen(c, UGRID), lv = jlen(c, VGRID);
    const int Nx = c->Nx, Nz = c->Nz, ign = Nx + 2;
    const size_t plane = (size_t)c->igal * c->kgal, npl = (size_t)nyu + 2, planeN = (size_t)ign * Nz;
    double *P1 = zalloc(plane * npl), *P2 = zalloc(plane * npl), *P3 = zalloc(plane * npl);
    double *P2i = zalloc(plane * npl), *P3i = zalloc(plane * npl), *PP = zalloc(plane * npl);
    double *WX = zalloc(planeN * npl);
    double *u2i = zalloc(2 * (size_t)lu * nc), *u3i = zalloc(2 * (size_t)lv * nc);
    interp_v(c, u2i, c->u2);
    interp_u(c, u3i, c->u3);
    modes_to_planes(c, P1, c->u1, UGRID);
    modes_to_planes(c, P2, c->u2, VGRID);
    modes_to_planes(c, P3, c->u3, UGRID);
    modes_to_planes(c, P2i, u2i, UGRID);
    modes_to_planes(c, P3i, u3i, VGRID);
    if (c->pp) modes_to_planes(c, PP, c->pp, PGRID);
    lho_omega_x(c, WX);
    const int nwork = 4 * (c->Mx > c->Mz ? c->Mx : c->Mz) + 8;
#pragma omp parallel num_threads(c->nthr)
    {
        double *w = zalloc(nwork);
#pragma omp for schedule(static)
        for (int j = 1; j <= nyu; j++) {
            four_to_phys_plane(c, PLANE(c, P1, j), w);
            four_to_phys_plane(c, PLANE(c, P2i, j), w);
            four_to_phys_plane(c, PLANE(c, P3, j), w);
            four_to_phys_plane(c, PLANE(c, P2, j), w);
            four_to_phys_plane(c, PLANE(c, P3i, j), w);
        }
        free(w);
    }
#pragma omp parallel for schedule(static) num_threads(c->nthr)
    for (int j = 0; j <= nyu + 1; j++) {
        double *Um = acc + 0 * npl + j, *U2m = acc + 1 * npl + j, *Vm = acc + 2 * npl + j, *V2m = acc + 3 * npl + j;
        double *Wm = acc + 4 * npl + j, *W2m = acc + 5 * npl + j, *UVm = acc + 6 * npl + j, *UWm = acc + 7 * npl + j;
        double *VWm = acc + 8 * npl + j, *Pm = acc + 9 * npl + j, *P2m = acc + 10 * npl + j;
        double *wxm = acc + 11 * npl + j, *wx2m = acc + 12 * npl + j;
        for (int k = 1; k <= c->kgal; k++)
            for (int i = 1; i <= c->igal - 2; i++) {
                const double a = *PL(c, P1, i, k, j), v = *PL(c, P2, i, k, j), w = *PL(c, P3, i, k, j);
                const double vi = *PL(c, P2i, i, k, j), wi = *PL(c, P3i, i, k, j);
                *Um = *Um + a;
                *U2m = *U2m + a * a;
                *Vm = *Vm + v;
                *V2m = *V2m + v * v;
                *Wm = *Wm + w;
                *W2m = *W2m + w * w;
                *UVm = *UVm + a * vi;
                *UWm = *UWm + a * w;
                *VWm = *VWm + v * wi;
                if (j >= 1) {
                    const double q = *PL(c, PP, i, k, j);
                    *Pm = *Pm + q;
                    *P2m = *P2m + q * q;
                }
            }
        const double *X = WX + planeN * j;
        for (int k = 1; k <= Nz; k++)
            for (int i = 1; i <= Nx; i++) {
                const double x = X[(i - 1) + (size_t)ign * (k - 1)];
                *wxm = *wxm + x;
                *wx2m = *wx2m + x * x;
            }
    }
    free(P1);
    free(P2);
    free(P3);
    free(P2i);
    free(P3i);
    free(PP);
    free(WX);
    free(u2i);
    free(u3i);
}

double lho_error_div(const lho_ctx *c)
{
    size_t n = (size_t)jlen(c, PGRID) * c->ncols;
    double e = 0.0;
    for (size_t q = 0; q < n; q++) {
        double a = hypot(c->div[2 * q], c->div[2 * q + 1]);
        if (a > e) e = a;
    }
    return e;
}
