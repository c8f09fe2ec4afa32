// Column pass of one RK3 substep: everything that couples a (kx, kz) mode
// along y.  One thread owns one column and sweeps y four times:
//
//   A (up)   RHS0_u1/u2/u3 (littleharsh.f90:682-856, laplacian_U/V :281-368),
//            the y-flux derivatives and the Nu sum (FOU3D.f90:268-281,
//            550-590), du += -g Nu (:359-368), the solveU right-hand side
//            (littleharsh.f90:878-890) and the forward elimination of the
//            three Helmholtz systems.  The LU factors of LU_build/LU_dec
//            (tridLU_3D.f90:163-221, 327-364) are formed on the fly; u and w
//            share one factorisation (the reference rebuilds it per field).
//   B (down) back substitution (tridLU_3D.f90:80-82), flow-rate correction
//            for flag_ctpress = 0 (column 0 only, littleharsh.f90:515-548),
//            divergence and the Poisson right-hand side (:645-658).
//   C (up)   LUsolP forward sweep with the set-up DG factors (:118-124).
//   D (down) LUsolP back sweep, p += psi, v_corr and the ghost rows
//            (littleharsh.f90:896-993).
//
// Intermediate y rows are written in place into the state arrays; the
// scaled upper diagonals go to FACU/FACV for the back substitution.
#include "lh_core.cuh"

namespace lh {

struct RK {
    double a, b, g, c, d;
};

__device__ __forceinline__ RK rk_coeffs(int kRK)
{
    // start.f90:439-453
    RK r;
    if (kRK == 1) {
        r.a = 4.0 / 15.0; r.b = 4.0 / 15.0; r.g = 8.0 / 15.0; r.c = 0.0; r.d = 8.0 / 15.0;
    } else if (kRK == 2) {
        r.a = 1.0 / 15.0; r.b = 1.0 / 15.0; r.g = 5.0 / 12.0; r.c = -17.0 / 60.0; r.d = 2.0 / 15.0;
    } else {
        r.a = 1.0 / 6.0; r.b = 1.0 / 6.0; r.g = 3.0 / 4.0; r.c = -5.0 / 12.0; r.d = 1.0 / 3.0;
    }
    return r;
}

__device__ __forceinline__ double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }

// Per-thread asynchronous row prefetch.  Each thread streams the rows of
// its own column through a ring of kStages shared-memory stages with
// cp.async, so a sweep keeps kStages-1 rows of loads in flight while it
// works on the current row; slots are [stage][slot][lane] so the 32 lanes of
// a warp touch 512 contiguous bytes.
constexpr int kColThreads = 32;
constexpr int kStages = 8;
constexpr int kSlotsA = 13, kSlotsB = 4, kSlotsC = 2, kSlotsD = 6;

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp16(double2 *s, const double2 *g)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(s)), "l"(g));
}
__device__ __forceinline__ void cp8(double *s, const double *g)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(s)), "l"(g));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

struct Ring {
    double2 *base;
    int nslot, lane;
    __device__ double2 *at(int stage, int slot) const { return base + ((stage * nslot + slot) * kColThreads + lane); }
};

size_t column_smem_bytes() { return (size_t)kStages * kSlotsA * kColThreads * sizeof(double2); }

__global__ void __launch_bounds__(kColThreads) k_column(const Inst *__restrict__ insts, const Work *__restrict__ work,
                                                        int kRK)
{
    extern __shared__ double2 ring_mem[];
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    const int lane = threadIdx.x;
    const int col = w.j * kColThreads + lane;
    if (col >= I.nc) return;  // whole-warp granularity except the last block; no block barriers below
    const int nc = I.nc, nxh = I.nxh, nyu = I.nyu, nyv = I.nyv;
    const int i = col % nxh, kr = col / nxh;
    const RK rk = rk_coeffs(kRK);
    const double dt = I.sc[SC_DT];
    const double Re = I.Re;
    const double C1 = rk.a / Re, C2 = -rk.c, G = -rk.g;
    const double kxr = I.kx[i], kzr = I.kz[kr];
    const double k2x = I.k2x[i], k2z = I.k2z[kr];
    const double beta = rk.b * dt / Re;
    // C3 = -dRK*k1F: (-0, -(d k)); C3*p = ((d k) p.im, -((d k) p.re))
    const double dC3x = rk.d * kxr, dC3z = rk.d * kzr;
    const double ddv = I.ddthetavi;
    const bool mean = (col == 0);
    const double C1m = -rk.d * I.sc[SC_MPGX];

    double2 *U1 = I.U1 + col, *U2 = I.U2 + col, *U3 = I.U3 + col, *P = I.P + col;
    double2 *N1 = I.NU1 + col, *N2 = I.NU2 + col, *N3 = I.NU3 + col;
    const double2 *X1 = I.NXZ1 + col, *X2 = I.NXZ2 + col, *X3 = I.NXZ3 + col;
    const double2 *UVF = I.UVF + col, *WVF = I.WVF + col, *VVC = I.VVC + col;
    double *FU = I.FACU + col, *FV = I.FACV + col;
    double2 *PS = I.PSI + col;
    const double *du = I.dyu2i, *dv = I.dyv2i;

    // ---------------- A: right-hand sides and forward elimination --------
    Ring ra{ring_mem, kSlotsA, lane};
    auto fillA = [&](int j) {  // inputs of row j (1..nyu)
        const int st = (j - 1) % kStages;
        const size_t o = (size_t)j * nc, on = o - nc;
        cp16(ra.at(st, 0), U1 + o + nc);
        cp16(ra.at(st, 1), U3 + o + nc);
        cp16(ra.at(st, 4), N1 + on);
        cp16(ra.at(st, 5), N3 + on);
        cp16(ra.at(st, 7), X1 + on);
        cp16(ra.at(st, 8), X3 + on);
        cp16(ra.at(st, 10), UVF + o);
        cp16(ra.at(st, 11), WVF + o);
        if (j <= nyv) {
            cp16(ra.at(st, 2), U2 + o + nc);
            cp16(ra.at(st, 3), P + o);  // p(j+1)
            cp16(ra.at(st, 6), N2 + on);
            cp16(ra.at(st, 9), X2 + on);
            cp16(ra.at(st, 12), VVC + o + nc);
        }
    };
    // row 0: rhs = 0 and a = [0, 1, gw1] (u, w) / [0, 1, 0] (v)
    double2 u1m = U1[0], u1c = U1[(size_t)nc], u3m = U3[0], u3c = U3[(size_t)nc];
    double2 u2m = U2[0], u2c = U2[(size_t)nc];
    double2 uvf_prev = UVF[0], wvf_prev = WVF[0];
    double2 vvc_c = VVC[(size_t)nc];
    double2 p_c = P[0];  // p(1)
    double a3u = I.gw1 * 1.0;
    double a3v = 0.0 * 1.0;
    double2 y1p = make_double2(0.0, 0.0), y3p = y1p, y2p = y1p;
    for (int r = 0; r < kStages - 1; r++) {
        if (1 + r <= nyu) fillA(1 + r);
        cp_commit();
    }
    U1[0] = y1p;
    U3[0] = y3p;
    U2[0] = y2p;
    FU[0] = a3u;
    FV[0] = a3v;
    for (int j = 1; j <= nyu; j++) {
        cp_wait<kStages - 2>();
        const int st = (j - 1) % kStages;
        const size_t o = (size_t)j * nc;
        const size_t on = o - nc;
        const double2 u1p = *ra.at(st, 0), u3p = *ra.at(st, 1);
        const double2 n1o = *ra.at(st, 4), n3o = *ra.at(st, 5);
        const double2 x1 = *ra.at(st, 7), x3 = *ra.at(st, 8);
        const double2 uvf = *ra.at(st, 10), wvf = *ra.at(st, 11);
        double2 u2p, p_n, n2o, x2, vvn;
        if (j <= nyv) {
            u2p = *ra.at(st, 2);
            p_n = *ra.at(st, 3);
            n2o = *ra.at(st, 6);
            x2 = *ra.at(st, 9);
            vvn = *ra.at(st, 12);
        }
        if (j + kStages - 1 <= nyu) fillA(j + kStages - 1);
        cp_commit();

        const double d1 = du[3 * j], d2 = du[3 * j + 1], d3 = du[3 * j + 2];
        const double cen = k2x + k2z + d2;
        double2 L1 = make_double2(d1 * u1m.x + cen * u1c.x + d3 * u1p.x, d1 * u1m.y + cen * u1c.y + d3 * u1p.y);
        double2 L3 = make_double2(d1 * u3m.x + cen * u3c.x + d3 * u3p.x, d1 * u3m.y + cen * u3c.y + d3 * u3p.y);
        double2 du1 = make_double2(C1 * L1.x + C2 * n1o.x + dC3x * p_c.y, C1 * L1.y + C2 * n1o.y + -(dC3x * p_c.x));
        double2 du3 = make_double2(C1 * L3.x + C2 * n3o.x + dC3z * p_c.y, C1 * L3.y + C2 * n3o.y + -(dC3z * p_c.x));
        if (mean) du1.x = du1.x + C1m;
        const double m = I.dthdyu[j];
        const double2 nu1 = make_double2(x1.x + (uvf.x - uvf_prev.x) * m * ddv, x1.y + (uvf.y - uvf_prev.y) * m * ddv);
        const double2 nu3 = make_double2(x3.x + (wvf.x - wvf_prev.x) * m * ddv, x3.y + (wvf.y - wvf_prev.y) * m * ddv);
        N1[on] = nu1;
        N3[on] = nu3;
        du1 = make_double2(du1.x + G * nu1.x, du1.y + G * nu1.y);
        du3 = make_double2(du3.x + G * nu3.x, du3.y + G * nu3.y);
        const double2 r1 = make_double2(u1c.x + dt * du1.x, u1c.y + dt * du1.y);
        const double2 r3 = make_double2(u3c.x + dt * du3.x, u3c.y + dt * du3.y);
        const double a1 = -beta * d1;
        const double a2 = 1.0 - beta * (d2 + k2x + k2z);
        const double a3 = -beta * d3;
        const double inv = 1.0 / (a2 - a1 * a3u);
        const double2 y1 = make_double2((r1.x - a1 * y1p.x) * inv, (r1.y - a1 * y1p.y) * inv);
        const double2 y3 = make_double2((r3.x - a1 * y3p.x) * inv, (r3.y - a1 * y3p.y) * inv);
        a3u = a3 * inv;
        U1[o] = y1;
        U3[o] = y3;
        FU[o] = a3u;
        y1p = y1;
        y3p = y3;
        u1m = u1c;
        u1c = u1p;
        u3m = u3c;
        u3c = u3p;
        uvf_prev = uvf;
        wvf_prev = wvf;
        if (j <= nyv) {
            const double e1 = dv[3 * j], e2 = dv[3 * j + 1], e3 = dv[3 * j + 2];
            const double cenv = k2x + k2z + e2;
            const double2 L2 = make_double2(e1 * u2m.x + cenv * u2c.x + e3 * u2p.x, e1 * u2m.y + cenv * u2c.y + e3 * u2p.y);
            const double mv = I.dthdyv[j];
            const double C3 = -rk.d * ddv * mv;
            double2 du2 = make_double2(C1 * L2.x + C2 * n2o.x + C3 * (p_n.x - p_c.x),
                                       C1 * L2.y + C2 * n2o.y + C3 * (p_n.y - p_c.y));
            const double2 nu2 = make_double2(x2.x + (vvn.x - vvc_c.x) * mv * ddv, x2.y + (vvn.y - vvc_c.y) * mv * ddv);
            N2[on] = nu2;
            du2 = make_double2(du2.x + G * nu2.x, du2.y + G * nu2.y);
            const double2 r2 = make_double2(u2c.x + dt * du2.x, u2c.y + dt * du2.y);
            const double b1 = -beta * e1;
            const double b2 = 1.0 - beta * (e2 + k2x + k2z);
            const double b3 = -beta * e3;
            const double invv = 1.0 / (b2 - b1 * a3v);
            const double2 y2 = make_double2((r2.x - b1 * y2p.x) * invv, (r2.y - b1 * y2p.y) * invv);
            a3v = b3 * invv;
            U2[o] = y2;
            FV[o] = a3v;
            y2p = y2;
            u2m = u2c;
            u2c = u2p;
            vvc_c = vvn;
            p_c = p_n;
        }
    }
    cp_wait<0>();
    // top rows, rhs = 0: u/w a = [gw2, 1, 0], v a = [0, 1, 0]
    {
        const double inv = 1.0 / (1.0 - I.gw2 * a3u);
        const double2 y1 = make_double2((0.0 - I.gw2 * y1p.x) * inv, (0.0 - I.gw2 * y1p.y) * inv);
        const double2 y3 = make_double2((0.0 - I.gw2 * y3p.x) * inv, (0.0 - I.gw2 * y3p.y) * inv);
        U1[(size_t)(nyu + 1) * nc] = y1;
        U3[(size_t)(nyu + 1) * nc] = y3;
        y1p = y1;
        y3p = y3;
        const double invv = 1.0 / (1.0 - 0.0 * a3v);
        const double2 y2 = make_double2((0.0 - 0.0 * y2p.x) * invv, (0.0 - 0.0 * y2p.y) * invv);
        U2[(size_t)(nyv + 1) * nc] = y2;
        y2p = y2;
    }
    __threadfence_block();

    // ---------------- B: back substitution and divergence ---------------
    const double dtirk = (1.0 / dt) / (rk.a + rk.b);
    const bool div_inline = I.flag_ctpress != 0;
    Ring rb{ring_mem, kSlotsB, lane};
    auto fillB = [&](int j) {  // row j (nyu .. 0)
        const int st = (nyu - j) % kStages;
        const size_t o = (size_t)j * nc;
        cp16(rb.at(st, 0), U1 + o);
        cp16(rb.at(st, 1), U3 + o);
        cp8(&rb.at(st, 3)->x, FU + o);
        if (j <= nyv) {
            cp16(rb.at(st, 2), U2 + o);
            cp8(&rb.at(st, 3)->y, FV + o);
        }
    };
    for (int r = 0; r < kStages - 1; r++) {
        if (nyu - r >= 0) fillB(nyu - r);
        cp_commit();
    }
    double2 v1 = y1p, v3 = y3p;  // rows j+1 of u1, u3
    double2 v2 = y2p;            // u2 at row nyv+1 = nyu
    for (int j = nyu; j >= 0; j--) {
        cp_wait<kStages - 2>();
        const int st = (nyu - j) % kStages;
        const size_t o = (size_t)j * nc;
        const double2 y1 = *rb.at(st, 0), y3 = *rb.at(st, 1);
        const double2 ff = *rb.at(st, 3);
        double2 y2 = make_double2(0.0, 0.0);
        if (j <= nyv) y2 = *rb.at(st, 2);
        if (j - (kStages - 1) >= 0) fillB(j - (kStages - 1));
        cp_commit();
        const double f = ff.x;
        const double2 n1 = make_double2(y1.x - f * v1.x, y1.y - f * v1.y);
        const double2 n3 = make_double2(y3.x - f * v3.x, y3.y - f * v3.y);
        U1[o] = n1;
        U3[o] = n3;
        double2 n2 = v2;
        if (j <= nyv) {
            const double fv = ff.y;
            n2 = make_double2(y2.x - fv * v2.x, y2.y - fv * v2.y);
            U2[o] = n2;
        }
        if (div_inline && j + 1 <= nyu) {
            // div(j+1) = i kx u1 + i kz u3 + dthdyu (u2(j+1) - u2(j)), psi = dtirk div
            const int jp = j + 1;
            const double mm = ddv * I.dthdyu[jp];
            const double2 d = make_double2(-(kxr * v1.y) + -(kzr * v3.y) + mm * (v2.x - n2.x),
                                           kxr * v1.x + kzr * v3.x + mm * (v2.y - n2.y));
            double2 ps = cscale(dtirk, d);
            if (mean && jp == 1) ps = make_double2(0.0, 0.0);  // gauge, littleharsh.f90:656-658
            PS[(size_t)(jp - 1) * nc] = ps;
        }
        v1 = n1;
        v3 = n3;
        v2 = n2;
    }
    cp_wait<0>();

    if (!div_inline) {
        __threadfence_block();
        if (mean) {
            // flowrate_corr (littleharsh.f90:515-548): u11 from LUsol0 with
            // LU_build0 (tridLU_3D.f90:299-325); flowrateRe's dummy
            // u(1:nn+2) receives u11(0:nn+2), so it sums u11(j-1).
            double *u11 = I.U11, *f11 = I.F11;
            const int ne = nyu + 1;
            const double bdt = -rk.d * dt;
            double a3p = I.gw1 * 1.0;
            double yp = 0.0 * 1.0;
            u11[0] = yp;
            f11[0] = a3p;
            for (int j = 1; j <= ne; j++) {
                double a1, a2, a3, rr;
                if (j < ne) {
                    a1 = -beta * du[3 * j];
                    a2 = 1.0 - beta * du[3 * j + 1];
                    a3 = -beta * du[3 * j + 2];
                    rr = bdt;
                } else {
                    a1 = I.gw2;
                    a2 = 1.0;
                    a3 = 0.0;
                    rr = 0.0;
                }
                const double inv = 1.0 / (a2 - a1 * a3p);
                yp = (rr - a1 * yp) * inv;
                a3p = a3 * inv;
                u11[j] = yp;
                f11[j] = a3p;
            }
            double up = yp;
            for (int j = ne - 1; j >= 0; j--) {
                up = u11[j] - f11[j] * up;
                u11[j] = up;
            }
            double Qx1 = 0.0, Qx0 = 0.0;
            for (int j = 1; j <= nyv + 1; j++) Qx1 = Qx1 + (I.yv[j] - I.yv[j - 1]) * u11[j - 1];
            for (int j = 1; j <= nyv + 1; j++) Qx0 = Qx0 + (I.yv[j] - I.yv[j - 1]) * U1[(size_t)j * nc].x;
            const double g = (I.sc[SC_QXT] - Qx0) / Qx1;
            I.sc[SC_MPGX] = I.sc[SC_MPGX] + g;
            I.sc[SC_DGX] = g;
            for (int j = 0; j <= ne; j++) {
                double2 u = U1[(size_t)j * nc];
                u.x = u.x + g * u11[j];
                U1[(size_t)j * nc] = u;
            }
        }
        double2 v2m = U2[0];
        for (int jp = 1; jp <= nyu; jp++) {
            const double2 a = U1[(size_t)jp * nc], c3 = U3[(size_t)jp * nc];
            const double2 v2c = U2[(size_t)jp * nc];
            const double mm = ddv * I.dthdyu[jp];
            const double2 d = make_double2(-(kxr * a.y) + -(kzr * c3.y) + mm * (v2c.x - v2m.x),
                                           kxr * a.x + kzr * c3.x + mm * (v2c.y - v2m.y));
            double2 ps = cscale(dtirk, d);
            if (mean && jp == 1) ps = make_double2(0.0, 0.0);
            PS[(size_t)(jp - 1) * nc] = ps;
            v2m = v2c;
        }
    }
    __threadfence_block();

    // ---------------- C: LUsolP forward sweep ------------------------------
    const double *G2 = I.DG2 + col, *G3 = I.DG3 + col;
    Ring rc{ring_mem, kSlotsC, lane};
    auto fillC = [&](int j) {  // row j (2 .. nyu)
        const int st = (j - 2) % kStages;
        const size_t o = (size_t)(j - 1) * nc;
        cp16(rc.at(st, 0), PS + o);
        cp8(&rc.at(st, 1)->x, G2 + o);
    };
    for (int r = 0; r < kStages - 1; r++) {
        if (2 + r <= nyu) fillC(2 + r);
        cp_commit();
    }
    double2 xp = cscale(G2[0], PS[0]);
    PS[0] = xp;
    for (int j = 2; j <= nyu; j++) {
        cp_wait<kStages - 2>();
        const int st = (j - 2) % kStages;
        const double2 x = *rc.at(st, 0);
        const double g2 = rc.at(st, 1)->x;
        if (j + kStages - 1 <= nyu) fillC(j + kStages - 1);
        cp_commit();
        const double g1 = I.DG1[j];
        xp = make_double2((x.x - g1 * xp.x) * g2, (x.y - g1 * xp.y) * g2);
        PS[(size_t)(j - 1) * nc] = xp;
    }
    cp_wait<0>();
    __threadfence_block();

    // ---------------- D: LUsolP back sweep, p += psi, v_corr --------------
    const double dtrk = dt * (rk.a + rk.b);
    const double kxd = dtrk * kxr, kzd = dtrk * kzr;
    const double dtrk_u2 = dtrk * ddv;
    Ring rd{ring_mem, kSlotsD, lane};
    auto fillD = [&](int j) {  // row j (nyu .. 1)
        const int st = (nyu - j) % kStages;
        const size_t o = (size_t)(j - 1) * nc, ou = (size_t)j * nc;
        cp16(rd.at(st, 0), PS + o);
        cp16(rd.at(st, 1), P + o);
        cp16(rd.at(st, 2), U1 + ou);
        cp16(rd.at(st, 3), U3 + ou);
        if (j <= nyv) cp16(rd.at(st, 4), U2 + ou);
        if (j < nyu) cp8(&rd.at(st, 5)->x, G3 + o);
    };
    for (int r = 0; r < kStages - 1; r++) {
        if (nyu - r >= 1) fillD(nyu - r);
        cp_commit();
    }
    double2 psn = make_double2(0.0, 0.0);  // psi(j+1)
    bool bad = false;
    for (int j = nyu; j >= 1; j--) {
        cp_wait<kStages - 2>();
        const int st = (nyu - j) % kStages;
        const double2 x = *rd.at(st, 0), p = *rd.at(st, 1);
        double2 a = *rd.at(st, 2), c3 = *rd.at(st, 3);
        double2 v = make_double2(0.0, 0.0);
        if (j <= nyv) v = *rd.at(st, 4);
        const double g3 = rd.at(st, 5)->x;
        if (j - (kStages - 1) >= 1) fillD(j - (kStages - 1));
        cp_commit();
        const size_t o = (size_t)(j - 1) * nc;
        double2 ps = x;  // psi(nyu) = x(nyu)
        if (j < nyu) ps = make_double2(x.x - g3 * psn.x, x.y - g3 * psn.y);
        PS[o] = ps;
        P[o] = make_double2(p.x + ps.x, p.y + ps.y);
        const size_t ou = (size_t)j * nc;
        a = make_double2(a.x - -(kxd * ps.y), a.y - kxd * ps.x);
        c3 = make_double2(c3.x - -(kzd * ps.y), c3.y - kzd * ps.x);
        U1[ou] = a;
        U3[ou] = c3;
        if (j == nyu) {
            U1[ou + nc] = cscale(I.gwbc, a);
            U3[ou + nc] = cscale(I.gwbc, c3);
        }
        if (j == 1) {
            U1[0] = cscale(I.gwbc, a);
            U3[0] = cscale(I.gwbc, c3);
            bad = !isfinite(a.x) || !isfinite(a.y) || !isfinite(ps.x) || !isfinite(ps.y);
        }
        if (j <= nyv) {
            const double mv = dtrk_u2 * I.dthdyv[j];
            v = make_double2(v.x - mv * (psn.x - ps.x), v.y - mv * (psn.y - ps.y));
            U2[ou] = v;
        }
        psn = ps;
    }
    cp_wait<0>();
    U2[0] = make_double2(0.0, 0.0);
    U2[(size_t)(nyv + 1) * nc] = make_double2(0.0, 0.0);
    if (bad) atomicOr(I.err, ERR_NONFINITE);
    if (mean && kRK == 3) {
        // flowrateIm (littleharsh.f90:473-492) via meanflow_ctP (:572-589)
        __threadfence_block();
        double Qu = 0.0;
        for (int j = 1; j <= nyv + 1; j++) Qu = Qu + (I.yv[j] - I.yv[j - 1]) * U1[(size_t)j * nc].x;
        I.sc[SC_QX] = Qu;
        I.sc[SC_ITER] = I.sc[SC_ITER] + 1.0;
    }
}

// ---------------------------------------------------------------------------
// dt at kRK = 1 (FOU3D.f90:290-303).  CFL mode folds the spectral wall plane
// 0 of u1/u3 (which dtc_calc scans as raw coefficients, its explicit-shape
// dummies starting one plane early) into the maxima the plane pipeline
// gathered, then resets the maxima.  The v term 1/(u2max*dthetavi) is +inf
// in the reference because dthetavi is never assigned, so it never wins.
__global__ void k_dt(const Inst *__restrict__ insts, int ninst)
{
    const int q = blockIdx.x;
    if (q >= ninst) return;
    const Inst &I = insts[q];
    __shared__ double r1[32], r3[32];
    double m1 = 0.0, m3 = 0.0;
    if (I.dt_mode == 0) {
        for (int c = threadIdx.x; c < I.nc; c += blockDim.x) {
            double2 a = I.U1[c], b = I.U3[c];
            m1 = fmax(m1, fmax(fabs(a.x), fabs(a.y)));
            m3 = fmax(m3, fmax(fabs(b.x), fabs(b.y)));
        }
        for (int o = 16; o > 0; o >>= 1) {
            m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
            m3 = fmax(m3, __shfl_xor_sync(0xffffffffu, m3, o));
        }
        if ((threadIdx.x & 31) == 0) {
            r1[threadIdx.x >> 5] = m1;
            r3[threadIdx.x >> 5] = m3;
        }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double *sc = I.sc;
    double dt;
    if (I.dt_mode == 0) {
        double a1 = __longlong_as_double((long long)*reinterpret_cast<unsigned long long *>(&sc[SC_U1MAX]));
        double a3 = __longlong_as_double((long long)*reinterpret_cast<unsigned long long *>(&sc[SC_U3MAX]));
        for (int k = 0; k < (int)(blockDim.x + 31) / 32; k++) {
            a1 = fmax(a1, r1[k]);
            a3 = fmax(a3, r3[k]);
        }
        const double ta = 1.0 / (I.alp * (double)(I.Nx / 2) * a1);
        const double tb = 1.0 / (I.bet * (double)(I.Nz / 2) * a3);
        const double dtc = fmin(ta, tb);
        sc[SC_DTC] = dtc;
        dt = fmin(2.5 * I.dtv, I.CFL * dtc);
        sc[SC_U1MAX] = 0.0;
        sc[SC_U3MAX] = 0.0;
    } else {
        dt = I.dt_fixed;
    }
    sc[SC_DT] = dt;
    sc[SC_T] = sc[SC_T] + dt;
}

// ---------------------------------------------------------------------------
// Layout transforms between the reference column layout x(j, column) (j
// fastest) and the plane-major device layout [j][column]: a 32x32 tiled
// transpose of a len x nc complex matrix.
__global__ void k_col_to_plane(const double2 *__restrict__ src, double2 *__restrict__ dst, int len, int nc)
{
    __shared__ double2 tile[32][33];
    const int c0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int c = c0 + r, j = j0 + threadIdx.x;
        if (c < nc && j < len) tile[r][threadIdx.x] = src[(size_t)c * len + j];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int j = j0 + r, c = c0 + threadIdx.x;
        if (c < nc && j < len) dst[(size_t)j * nc + c] = tile[threadIdx.x][r];
    }
}

__global__ void k_plane_to_col(const double2 *__restrict__ src, double2 *__restrict__ dst, int len, int nc)
{
    __shared__ double2 tile[32][33];
    const int c0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int j = j0 + r, c = c0 + threadIdx.x;
        if (c < nc && j < len) tile[r][threadIdx.x] = src[(size_t)j * nc + c];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int c = c0 + r, j = j0 + threadIdx.x;
        if (c < nc && j < len) dst[(size_t)c * len + j] = tile[threadIdx.x][r];
    }
}

// ---------------------------------------------------------------------------
// Stand-alone LUsolU on plane-major columns (unit entry): grid 2 = u/w
// (rows 0..nyu+1), 1 = v (rows 0..nyv+1)
__global__ void k_lusolu(const Inst *__restrict__ insts, int grid, int kRK, double dt, const double2 *rhs,
                         double2 *u, double *fac)
{
    const Inst &I = insts[0];
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= I.nc) return;
    const int nc = I.nc, i = col % I.nxh, kr = col / I.nxh;
    const int ne = grid == 2 ? I.nyu + 1 : I.nyv + 1;
    const double *d = grid == 2 ? I.dyu2i : I.dyv2i;
    const RK rk = rk_coeffs(kRK);
    const double beta = rk.b * dt / I.Re;
    const double k2x = I.k2x[i], k2z = I.k2z[kr];
    double a3p = (grid == 2 ? I.gw1 : 0.0) * 1.0;
    double2 r0 = rhs[col];
    double2 yp = make_double2(r0.x * 1.0, r0.y * 1.0);
    u[col] = yp;
    fac[col] = a3p;
    for (int j = 1; j <= ne; j++) {
        double a1, a2, a3;
        if (j < ne) {
            a1 = -beta * d[3 * j];
            a2 = 1.0 - beta * (d[3 * j + 1] + k2x + k2z);
            a3 = -beta * d[3 * j + 2];
        } else {
            a1 = grid == 2 ? I.gw2 : 0.0;
            a2 = 1.0;
            a3 = 0.0;
        }
        const double inv = 1.0 / (a2 - a1 * a3p);
        const double2 r = rhs[(size_t)j * nc + col];
        yp = make_double2((r.x - a1 * yp.x) * inv, (r.y - a1 * yp.y) * inv);
        a3p = a3 * inv;
        u[(size_t)j * nc + col] = yp;
        fac[(size_t)j * nc + col] = a3p;
    }
    double2 up = yp;
    for (int j = ne - 1; j >= 0; j--) {
        const double2 y = u[(size_t)j * nc + col];
        const double f = fac[(size_t)j * nc + col];
        up = make_double2(y.x - f * up.x, y.y - f * up.y);
        u[(size_t)j * nc + col] = up;
    }
}

// Stand-alone LUsolP on plane-major columns, rows 1..nyu stored from 0
__global__ void k_lusolp(const Inst *__restrict__ insts, double2 *x)
{
    const Inst &I = insts[0];
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= I.nc) return;
    const int nc = I.nc, nyu = I.nyu;
    double2 xp = x[col];
    xp = cscale(I.DG2[col], xp);
    x[col] = xp;
    for (int j = 2; j <= nyu; j++) {
        const size_t o = (size_t)(j - 1) * nc + col;
        const double2 v = x[o];
        xp = make_double2((v.x - I.DG1[j] * xp.x) * I.DG2[o], (v.y - I.DG1[j] * xp.y) * I.DG2[o]);
        x[o] = xp;
    }
    double2 pn = xp;
    for (int j = nyu - 1; j >= 1; j--) {
        const size_t o = (size_t)(j - 1) * nc + col;
        const double2 v = x[o];
        pn = make_double2(v.x - I.DG3[o] * pn.x, v.y - I.DG3[o] * pn.y);
        x[o] = pn;
    }
}

// max |div| over all columns (error(), littleharsh.f90:370-409); div is
// recomputed from the projected state
__global__ void k_divmax(const Inst *__restrict__ insts, double *out)
{
    const Inst &I = insts[0];
    double m = 0.0;
    const int nc = I.nc;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nc * I.nyu; t += gridDim.x * blockDim.x) {
        const int col = t % nc, jp = t / nc + 1;
        const int i = col % I.nxh, kr = col / I.nxh;
        const double kxr = I.kx[i], kzr = I.kz[kr];
        const double2 a = I.U1[(size_t)jp * nc + col], c3 = I.U3[(size_t)jp * nc + col];
        const double2 v0 = I.U2[(size_t)jp * nc + col], vm = I.U2[(size_t)(jp - 1) * nc + col];
        const double mm = I.ddthetavi * I.dthdyu[jp];
        double dr = -(kxr * a.y) + -(kzr * c3.y) + mm * (v0.x - vm.x);
        double di = kxr * a.x + kzr * c3.x + mm * (v0.y - vm.y);
        m = fmax(m, hypot(dr, di));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(reinterpret_cast<unsigned long long *>(out), (unsigned long long)__double_as_longlong(m));
}

}  // namespace lh
