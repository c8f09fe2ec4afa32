// Host set-up of one channel instance (see lh_setup.h).  The formulas follow
// start.f90 line by line so the device operators see the same numbers the
// reference would compute; integer powers use binary powering, which is how
// a Fortran real**integer with a run-time exponent is evaluated.
#include "lh_setup.h"

#include <algorithm>
#include <cmath>
#include <thread>
#include <sstream>

namespace lh {

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

// cffti1-style factorisation (cft_buff.f:141-163): try 3, 4, 2, 5, then odd
// numbers; a factor 2 found after the first is moved to the front.
static bool factor_fftpack(int n, const int try4[4], std::vector<int> &out)
{
    out.clear();
    int nl = n, j = 0, ntry = 0;
    std::vector<int> f;
    while (nl != 1) {
        j++;
        ntry = j <= 4 ? try4[j - 1] : ntry + 2;
        if (ntry > n) return false;
        while (nl % ntry == 0) {
            f.push_back(ntry);
            nl /= ntry;
            if (ntry == 2 && f.size() != 1) {
                f.pop_back();
                f.insert(f.begin(), 2);
            }
            if (nl == 1) break;
        }
    }
    for (int p : f)
        if (p != 2 && p != 3 && p != 4) return false;
    out = f;
    return true;
}

// Radix orders: cffti1 tries 3, 4, 2, 5 (cft_buff.f:144), rffti1 4, 2, 3
// (rft_buff.f:136).
bool cft_radices(int n, std::vector<int> &rad)
{
    static const int t[4] = {3, 4, 2, 5};
    return factor_fftpack(n, t, rad);
}

bool rft_radices(int n, std::vector<int> &rad)
{
    static const int t[4] = {4, 2, 3, 5};
    return factor_fftpack(n, t, rad);
}

// z twiddles with the rotation recurrence of cffti1 (cft_buff.f:166-179)
void cft_table(int n, std::vector<double> &tw)
{
    tw.assign(2 * n, 0.0);
    const double tpi = 8.0 * std::atan(1.0);
    const double arg1 = tpi / (double)(float)n;
    const double dc = std::cos(arg1), ds = std::sin(arg1);
    std::vector<double> wa(2 * n);
    wa[0] = dc;
    wa[1] = ds;
    for (int ii = 4; ii <= 2 * n; ii += 2) {
        wa[ii - 2] = dc * wa[ii - 4] - ds * wa[ii - 3];
        wa[ii - 1] = ds * wa[ii - 4] + dc * wa[ii - 3];
    }
    tw[0] = 1.0;
    tw[1] = 0.0;
    for (int t = 1; t < n; t++) {
        tw[2 * t] = wa[2 * t - 2];
        tw[2 * t + 1] = wa[2 * t - 1];
    }
}

// x twiddles with direct cos/sin as rffti1 computes them
void rft_table(int n, std::vector<double> &tw)
{
    tw.assign(2 * n, 0.0);
    const double tpi = 2.0 * std::atan2(0.0, -1.0);
    const double argh = tpi / (double)(float)n;
    for (int t = 0; t < n; t++) {
        const double arg = (double)t * argh;
        tw[2 * t] = std::cos(arg);
        tw[2 * t + 1] = std::sin(arg);
    }
    tw[0] = 1.0;
    tw[1] = 0.0;
}

double flowrate_host(const HostSetup &s, const double *u1col)
{
    double Qu = 0.0;
    for (int j = 1; j <= s.nyv + 1; j++) Qu = Qu + (s.yv[j] - s.yv[j - 1]) * u1col[2 * j];
    return Qu;
}

std::string build_setup(const lh_grid_desc &d, HostSetup &s)
{
    std::ostringstream err;
    if (d.Nx < 2 || d.Nz < 2 || d.Nx % 2 || d.Nz % 2) return "Nx and Nz must be even and >= 2";
    if (d.ny < 5) return "ny must be >= 5";
    if (!(d.Re > 0)) return "Re must be positive";
    if (d.grid_type != LH_GRID_POLY && d.grid_type != LH_GRID_TANH) return "unknown grid_type";
    if (d.dt_mode != LH_DT_CFL && d.dt_mode != LH_DT_FIXED) return "unknown dt_mode";
    if (d.dt_mode == LH_DT_FIXED && !(d.dt > 0)) return "fixed dt must be positive";
    if (d.flag_ctpress != 0 && d.flag_ctpress != 1) return "flag_ctpress must be 0 or 1";
    s.Nx = d.Nx;
    s.Nz = d.Nz;
    // start.f90:135-136 Nspec = 2 Ngal / 3: only Ngal = 3 Nspec / 2 is exact
    s.Mx = 3 * d.Nx / 2;
    s.Mz = 3 * d.Nz / 2;
    if ((3 * d.Nx) % 2 || (3 * d.Nz) % 2) return "3N/2 must be an integer";
    s.nxh = d.Nx / 2 + 1;
    s.nc = s.nxh * d.Nz;
    s.nyv = d.ny - 2;
    s.nyu = s.nyv + 1;
    if (!cft_radices(s.Mz, s.radz)) {
        err << "Ngal_z = " << s.Mz << " is not 2/3-smooth";
        return err.str();
    }
    if (!rft_radices(s.Mx, s.radx) || s.Mx % 2) {
        err << "Ngal_x = " << s.Mx << " is not 2/3-smooth (rft_buff.f:308-311)";
        return err.str();
    }
    if (s.radz.size() > 12 || s.radx.size() > 12) return "transform too long";

    // ---- ygrid (start.f90:665-806)
    const int nn = s.nyv + 1;
    s.yu.assign(nn + 2, 0.0);
    s.yv.assign(nn + 1, 0.0);
    s.dthdyu.assign(nn + 2, 0.0);
    s.dthdyv.assign(nn + 1, 0.0);
    const double qqq = nn / 2.0;
    if (d.grid_type == LH_GRID_POLY) {
        const int ppp = d.ppp;
        const double dyq = d.dyq;
        if (ppp < 1) return "ppp must be >= 1";
        const double bbb = (dyq - 1.0) / (qqq * (1.0 - powi(qqq, ppp - 1) +
                                                 dyq * ((1.0 - qqq) * powi(qqq, ppp - 1) - powi(1.0 - qqq, ppp))));
        const double aaa = (1.0 - bbb * powi(qqq, ppp)) / qqq;
        s.yu[0] = aaa * (-1.0 + .5 - qqq) + bbb * powi(-1.0 + .5 - qqq, ppp);
        for (int j = 0; j <= nn; j++) {
            s.yv[j] = aaa * (j - qqq) + bbb * powi(j - qqq, ppp);
            s.yu[j + 1] = aaa * (j + .5 - qqq) + bbb * powi(j + .5 - qqq, ppp);
        }
        s.dthdyu[0] = 1.0 / (aaa + ppp * bbb * powi(-1.0 + .5 - qqq, ppp - 1));
        for (int j = 0; j <= nn; j++) {
            s.dthdyv[j] = 1.0 / (aaa + ppp * bbb * powi(j - qqq, ppp - 1));
            s.dthdyu[j + 1] = 1.0 / (aaa + ppp * bbb * powi(j + .5 - qqq, ppp - 1));
        }
    } else {
        // tanh stretching: y(s) = tanh(g s)/tanh(g), s = (j - q)/q, with the
        // analytic dtheta/dy = q tanh(g) / (g (1 - tanh^2(g s)))
        const double g = d.gamma, tg = std::tanh(g);
        if (!(g > 0)) return "gamma must be positive";
        auto Y = [&](double x) { return std::tanh(g * (x - qqq) / qqq) / tg; };
        auto T = [&](double x) {
            const double th = std::tanh(g * (x - qqq) / qqq);
            return 1.0 / (g * (1.0 - th * th) / (qqq * tg));
        };
        s.yu[0] = Y(-1.0 + .5);
        s.dthdyu[0] = T(-1.0 + .5);
        for (int j = 0; j <= nn; j++) {
            s.yv[j] = Y((double)j);
            s.yu[j + 1] = Y(j + .5);
            s.dthdyv[j] = T((double)j);
            s.dthdyu[j + 1] = T(j + .5);
        }
    }
    const std::vector<double> &yu = s.yu, &yv = s.yv;
    s.dyu2i.assign(3 * (nn + 2), 0.0);
    s.dyv2i.assign(3 * (nn + 1), 0.0);
    auto DU = [&](int r, int j) -> double & { return s.dyu2i[(r - 1) + 3 * j]; };
    auto DV = [&](int r, int j) -> double & { return s.dyv2i[(r - 1) + 3 * j]; };
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
    s.ddthetavi = 1.0;

    // ---- def_k (start.f90:842-862)
    s.kx.assign(s.nxh, 0.0);
    s.k2x.assign(s.nxh, 0.0);
    for (int i = 0; i <= d.Nx / 2; i++) {
        s.kx[i] = d.alp * i;
        s.k2x[i] = -((d.alp * i) * (d.alp * i));
    }
    s.kz.assign(d.Nz, 0.0);
    s.k2z.assign(d.Nz, 0.0);
    for (int k = 1; k <= d.Nz / 2; k++) {
        s.kz[k - 1] = d.bet * (k - 1);
        s.k2z[k - 1] = -((d.bet * (k - 1)) * (d.bet * (k - 1)));
    }
    for (int k = d.Nz / 2 + 1; k <= d.Nz; k++) {
        s.kz[k - 1] = -(d.bet * (d.Nz - k + 1));
        s.k2z[k - 1] = -((d.bet * (d.Nz - k + 1)) * (d.bet * (d.Nz - k + 1)));
    }

    // ---- weights and dtv (start.f90:476, 518-537)
    const int nyu = s.nyu, nyv = s.nyv;
    s.gw1 = -(yv[0] - yu[0]) / (yv[0] - yu[1]);
    s.gw2 = (yu[nyu + 1] - yv[nyv + 1]) / (yv[nyv + 1] - yu[nyu]);
    s.gwbc = (yu[0] - yv[0]) / (yu[1] - yv[0]);
    s.gwi1 = (yu[0] - yu[1]) / (yv[0] - yu[1]);
    s.gwi2 = (yu[nyu + 1] - yu[nyu]) / (yv[nyv + 1] - yu[nyu]);
    s.dtv = d.Re / (-s.k2x[d.Nx / 2] - s.k2z[d.Nz / 2 - 1] + 4.0 / ((yv[1] - yv[0]) * (yv[1] - yv[0])));

    // ---- LU_buildP + LU_decP (tridLU_3D.f90:224-297, 366-407)
    const int ns = 1, ne = nyu, len = ne - ns + 1, nc = s.nc;
    std::vector<double> Db(len + 2), Gb(len + 2), Dt(len + 2), Gt(len + 2);
    auto V = [&](std::vector<double> &a, int jj) -> double & { return a[jj - ns + 1]; };
    for (int jj = ns; jj <= ne; jj++) {
        V(Db, jj - 1) = -s.ddthetavi * s.dthdyu[jj];
        V(Gb, jj) = -s.ddthetavi * s.dthdyv[jj];
        V(Dt, jj) = s.ddthetavi * s.dthdyu[jj];
        V(Gt, jj + 1) = s.ddthetavi * s.dthdyv[jj];
    }
    s.DG1.assign(nyu + 1, 0.0);
    for (int jj = ns + 1; jj <= ne; jj++) s.DG1[jj] = V(Db, jj - 1) * V(Gb, jj - 1);
    s.DG2.assign((size_t)len * nc, 0.0);
    s.DG3.assign((size_t)len * nc, 0.0);
    // Row by row over all columns (the recurrence runs along y, columns are
    // independent), so the plane-major DG rows are written contiguously; per
    // element the operations and their order are those of LU_decP.
    std::vector<double> k2x_c(nc), k2z_c(nc), a2p(nc), a3p(nc);
    for (int col = 0; col < nc; col++) {
        k2x_c[col] = s.k2x[col % s.nxh];
        k2z_c[col] = s.k2z[col / s.nxh];
    }
    auto factor_columns = [&](int c0, int c1) {
        {
            const double dg = V(Dt, ns) * V(Gb, ns), a3r = V(Dt, ns) * V(Gt, ns + 1);
            for (int col = c0; col < c1; col++) {
                double a2 = (dg + k2x_c[col]) + k2z_c[col], a3 = a3r;
                if (col == 0) {  // gauge row of the (0,0) mode (tridLU_3D.f90:276-280)
                    a2 = 1.0 / ((yu[1 + 1] - yu[1]) * (yu[1 + 1] - yu[1]));
                    a3 = 0.0;
                }
                a2p[col] = 1.0 / a2;
                a3p[col] = a3;
            }
        }
        for (int jj = ns + 1; jj <= ne; jj++) {
            const double a1 = V(Db, jj - 1) * V(Gb, jj - 1);
            const double b1 = V(Db, jj - 1) * V(Gt, jj);
            const double b2 = jj < ne ? V(Dt, jj) * V(Gb, jj) : 0.0;
            const double a3r = jj < ne ? V(Dt, jj) * V(Gt, jj + 1) : 0.0;
            double *dg2p = &s.DG2[(size_t)(jj - 2) * nc], *dg3p = &s.DG3[(size_t)(jj - 2) * nc];
            for (int col = c0; col < c1; col++) {
                const double a3s = a3p[col] * a2p[col];  // a3(jj-1) scaled by its pivot
                dg2p[col] = a2p[col];
                dg3p[col] = a3s;
                const double raw = jj < ne ? ((b1 + b2) + k2x_c[col]) + k2z_c[col] : (b1 + k2x_c[col]) + k2z_c[col];
                a2p[col] = 1.0 / (raw - a1 * a3s);
                a3p[col] = a3r;
            }
        }
        for (int col = c0; col < c1; col++) {
            s.DG2[(size_t)(ne - 1) * nc + col] = a2p[col];
            s.DG3[(size_t)(ne - 1) * nc + col] = 0.0;
        }
    };
    // large instances: column ranges on several host threads
    const size_t work = (size_t)nc * len;
    int nth = work > (1u << 20) ? (int)std::min<unsigned>(8u, std::max(1u, std::thread::hardware_concurrency())) : 1;
    if (nth > 1) {
        std::vector<std::thread> pool;
        const int per = (nc + nth - 1) / nth;
        for (int t = 0; t < nth; t++) {
            const int c0 = t * per, c1 = std::min(nc, c0 + per);
            if (c0 < c1) pool.emplace_back(factor_columns, c0, c1);
        }
        for (auto &th : pool) th.join();
    } else {
        factor_columns(0, nc);
    }

    cft_table(s.Mz, s.twz);
    rft_table(s.Mx, s.twx);
    return std::string();
}

}  // namespace lh
