// Column pass of one RK3 substep: everything that couples a (kx, kz) mode
// along y.  A CTA owns 32 columns (one per lane) and runs three warps on
// them, one per velocity component (u1, u3, u2), so the three Helmholtz
// chains of a column advance side by side:
//
//   A (up, all warps)   RHS0_u1/u2/u3 (littleharsh.f90:682-856, laplacian_U/V
//            :281-368), the y-flux derivatives and the Nu sum (FOU3D.f90:
//            268-281, 550-590), du += -g Nu (:359-368), the solveU right-hand
//            side (littleharsh.f90:878-890) and the forward elimination of
//            that warp's Helmholtz system.  The LU factors of LU_build/LU_dec
//            (tridLU_3D.f90:163-221, 327-364) are formed on the fly; the u
//            and w warps form the same u-grid factors with the same
//            arithmetic, so they agree bit for bit.
//   B (down, all warps) back substitution (tridLU_3D.f90:80-82).
//   C (up, u1 warp)     flow-rate correction for flag_ctpress = 0 (column 0
//            only, littleharsh.f90:515-548), divergence and the Poisson
//            right-hand side (:645-658), LUsolP forward sweep with the set-up
//            DG factors (tridLU_3D.f90:118-124).
//   D (down, u1 warp)   LUsolP back sweep, p += psi and v_corr with the ghost
//            rows (littleharsh.f90:896-993) in one sweep: row j of psi is
//            final when the sweep reaches it, and u1, u3 need psi(j), u2
//            psi(j) and psi(j+1), so each row of the state is written once.
//
// Block barriers separate the phases; every lane reaches them, columns past
// the instance's last only skip the work.  Intermediate y rows are written
// in place into the state arrays; the scaled upper diagonals go to FACU/FACV
// for the back substitution, the forward sweep of LUsolP to PSI.
#include "lh_kernels.cuh"

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
constexpr int kColThreads = kColumnThreads;
constexpr int kRoles = kColumnBlock / kColumnThreads;
// Row slots (one complex per lane, 512 B per warp) of shared memory each
// warp owns; a phase that loads S slots per row keeps kWarpSlots / S rows in
// flight, and the single-warp Poisson sweeps use all warps' slots.
#ifndef LH_COLUMN_SLOTS
#define LH_COLUMN_SLOTS 40
#endif
constexpr int kWarpSlots = LH_COLUMN_SLOTS;

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp16(double2 *s, const double2 *g)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(s)), "l"(g));
}
__device__ __forceinline__ void cp8(double *s, const double *g)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(s)), "l"(g));
}
// L2 eviction hints (LH_COLUMN_HINTS, compile time; 0 = none): 1 marks the
// forward sweep's read-once rows (Nu_old, the Nu x/z parts, the y fluxes)
// and the Nu and psi rows no later sweep of the launch reads as evict-first;
// 2 also marks the rows the later sweeps read back (eliminated rows, factors,
// the forward Poisson sweep) as evict-last.
#ifndef LH_COLUMN_HINTS
#define LH_COLUMN_HINTS 0
#endif
struct Hints {
    unsigned long long first, last;
    __device__ Hints()
    {
        first = last = 0ull;
#if LH_COLUMN_HINTS >= 1
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(first));
#endif
#if LH_COLUMN_HINTS >= 2
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(last));
#endif
    }
    __device__ __forceinline__ void cp_once(double2 *s, const double2 *g) const
    {
#if LH_COLUMN_HINTS >= 1
        asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;\n" ::"r"(smem_addr(s)), "l"(g),
                     "l"(first));
#else
        cp16(s, g);
#endif
    }
    __device__ __forceinline__ void st_once(double2 *g, double2 v) const
    {
#if LH_COLUMN_HINTS >= 1
        asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(g), "d"(v.x), "d"(v.y), "l"(first)
                     : "memory");
#else
        *g = v;
#endif
    }
    __device__ __forceinline__ void st_back(double2 *g, double2 v) const
    {
#if LH_COLUMN_HINTS >= 2
        asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(g), "d"(v.x), "d"(v.y), "l"(last)
                     : "memory");
#else
        *g = v;
#endif
    }
    __device__ __forceinline__ void st_back(double *g, double v) const
    {
#if LH_COLUMN_HINTS >= 2
        asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(g), "d"(v), "l"(last) : "memory");
#else
        *g = v;
#endif
    }
};
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Ring of D row stages with S complex slots each, laid out
// [stage][slot][lane] so a warp's 32 lanes touch 512 contiguous bytes.
template <int D, int S>
struct Ring {
    static constexpr int kDepth = D;
    double2 *base;
    int lane;
    __device__ double2 *at(int stage, int slot) const { return base + ((stage * S + slot) * kColThreads + lane); }
};

// Doubles of the per-row y metrics staged in shared memory: d2/dy2
// coefficients of both grids, dtheta/dy of both grids, DG1.
__host__ __device__ inline size_t column_metric_doubles(int nyu, int nyv)
{
    return 4 * (size_t)(nyu + 2) + 4 * (size_t)(nyv + 2) + (size_t)(nyu + 1);
}

size_t column_smem_bytes(int max_nyu)
{
    return (size_t)kRoles * kWarpSlots * kColThreads * sizeof(double2) +
           column_metric_doubles(max_nyu, max_nyu - 1) * sizeof(double);
}

// Row streamer over a ring of depth D: rows are visited in order
// r = 0..n-1.  fill(r, stage) issues the copies of row r; load(r, stage)
// reads the landed row (and its shared-memory metrics) into registers;
// use(r, row) consumes it.  Keeps D-1 rows in flight and handles U rows per
// step, all loads first, so the reads of the next rows are not ordered
// behind the global stores of the current one and overlap its recurrence.
template <int D, int U, class Fill, class Load, class Use>
__device__ __forceinline__ void stream_rows(int n, Fill &&fill, Load &&load, Use &&use)
{
    static_assert(U >= 1 && U < D - 1, "unroll must leave rows in flight");
    using Row = decltype(load(0, 0));
    for (int r = 0; r < D - 1; r++) {
        if (r < n) fill(r, r % D);
        cp_commit();
    }
    int r = 0;
    for (; r + U <= n; r += U) {
        cp_wait<D - 1 - U>();  // rows r .. r+U-1 have landed
        Row v[U];
#pragma unroll
        for (int u = 0; u < U; u++) v[u] = load(r + u, (r + u) % D);
#pragma unroll
        for (int u = 0; u < U; u++) use(r + u, v[u]);
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int rn = r + D - 1 + u;  // reuses the stage of row r-1+u
            if (rn < n) fill(rn, rn % D);
            cp_commit();
        }
    }
    for (; r < n; r++) {
        cp_wait<D - 2>();
        const Row v = load(r, r % D);
        use(r, v);
        if (r + D - 1 < n) fill(r + D - 1, (r + D - 1) % D);
        cp_commit();
    }
    cp_wait<0>();
}

struct RowA {
    double2 a, b, c, d, e;
    double m0, m1, m2, m3;
};
struct RowB {
    double2 y;
    double f;
};
struct RowC {
    double2 a, c3, v2c;
    double g2, th, g1;
};
struct RowD {
    double2 x, p, u1, u3, u2;
    double g3, th;
};

// Carried state of a forward-sweep chunk, per (role, column): u1/u3 roles
// um, uc, flp, yp and the factor a3u; the u2 role um, uc, vvc, pc, yp and
// a3v (the factor in .x of the last slot).
constexpr int kCarryFields = 6;
__device__ __forceinline__ double2 *carry_slot(const Inst &I, int role, int f, size_t col)
{
    return I.CARRY + ((size_t)role * kCarryFields + f) * I.nc + col;
}

// MODE 0: the whole pass in one launch (phase A writes the eliminated rows
// in place into the state).  MODE 1: phase A only, for the u rows w.slot ..
// w.blk of the work item (the u2 chain one row behind, since its y-flux
// needs vv_c of the next plane), into the Y arrays, carrying the sweep's
// state between chunks.  MODE 2: phases B-D, the back substitution reading
// the Y arrays.
template <int MODE>
__device__ __forceinline__ void column_body(const Inst *__restrict__ insts, const Work *__restrict__ work, int kRK)
{
    extern __shared__ double2 ring_mem[];
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    const int lane = threadIdx.x % kColThreads, role = threadIdx.x / kColThreads;
    const int col = w.j * kColThreads + lane;
    const bool live = col < I.nc;  // inactive lanes still reach every barrier
    const int nc = I.nc, nxh = I.nxh, nyu = I.nyu, nyv = I.nyv;
    const int i = live ? col % nxh : 0, kr = live ? col / nxh : 0;
    const RK rk = rk_coeffs(kRK);
    const double dt = I.sc[SC_DT];
    const double Re = I.Re;
    const double C1 = rk.a / Re, C2 = -rk.c, G = -rk.g;
    const double kxr = I.kx[i], kzr = I.kz[kr];
    const double k2x = I.k2x[i], k2z = I.k2z[kr];
    const double beta = rk.b * dt / Re;
    const double ddv = I.ddthetavi;
    const bool mean = (col == 0);
    const size_t cc = live ? col : 0;
    double2 *U1 = I.U1 + cc, *U2 = I.U2 + cc, *U3 = I.U3 + cc, *P = I.P + cc;
    double2 *PS = I.PSI + cc;
    double *FU = I.FACU + cc, *FV = I.FACV + cc;
    // per-row y metrics, read by every row of every sweep, staged once
    double *sdu = reinterpret_cast<double *>(ring_mem + (size_t)kRoles * kWarpSlots * kColThreads);
    double *sdv = sdu + 3 * (nyu + 2), *sthu = sdv + 3 * (nyv + 2), *sthv = sthu + (nyu + 2), *sdg1 = sthv + (nyv + 2);
    for (int e = threadIdx.x; e < 3 * (nyu + 2); e += blockDim.x) sdu[e] = I.dyu2i[e];
    for (int e = threadIdx.x; e < 3 * (nyv + 2); e += blockDim.x) sdv[e] = I.dyv2i[e];
    for (int e = threadIdx.x; e < nyu + 2; e += blockDim.x) sthu[e] = I.dthdyu[e];
    for (int e = threadIdx.x; e < nyv + 2; e += blockDim.x) sthv[e] = I.dthdyv[e];
    for (int e = threadIdx.x; e < nyu + 1; e += blockDim.x) sdg1[e] = I.DG1[e];
    __syncthreads();
    const double *du = sdu, *dv = sdv;
    double2 *warp_mem = ring_mem + (size_t)role * kWarpSlots * kColThreads;
    const Hints hint;
    using RingA = Ring<kWarpSlots / 5, 5>;         // phase A: 5 slots per row
    using RingW2 = Ring<kWarpSlots / 2, 2>;        // phase B: 2 slots per row
    using RingC = Ring<kRoles * kWarpSlots / 4, 4>;   // phase C (u1 warp, all slots)
    using RingD = Ring<kRoles * kWarpSlots / 6, 6>;   // phase D (u1 warp, all slots)

    // ---------------- A: right-hand sides and forward elimination --------
    const int ja = MODE == 1 ? w.slot : 1, jb = MODE == 1 ? w.blk : nyu;  // u rows of this launch
    if (MODE != 2 && live && role < 2) {
        // u1 (role 0) or u3 (role 1): RHS0_u1/u3 (littleharsh.f90:682-751,
        // 807-856), Nu sum (FOU3D.f90:268-281), du += -g Nu (:359-364),
        // solveU rhs (littleharsh.f90:878-890), LU_build/LU_dec on the fly;
        // both roles form the same u-grid factors with the same arithmetic.
        double2 *U = role == 0 ? U1 : U3;
        double2 *YD = MODE == 0 ? U : (role == 0 ? I.Y1 : I.Y3) + cc;  // eliminated rows
        double2 *N = (role == 0 ? I.NU1 : I.NU3) + cc;
        const double2 *X = (role == 0 ? I.NXZ1 : I.NXZ3) + cc;
        const double2 *FL = (role == 0 ? I.UVF : I.WVF) + cc;
        // C3 = -dRK*k1F: (-0, -(d k)); C3*p = ((d k) p.im, -((d k) p.re))
        const double dC3 = rk.d * (role == 0 ? kxr : kzr);
        const double C1m = (role == 0 && mean) ? -rk.d * I.sc[SC_MPGX] : 0.0;
        double2 um, uc, flp, yp;
        double a3u;
        if (ja == 1) {
            um = U[0];
            uc = U[(size_t)nc];
            flp = FL[0];
            a3u = I.gw1 * 1.0;
            yp = make_double2(0.0, 0.0);
            YD[0] = yp;
            if (role == 0) FU[0] = a3u;
        } else {
            um = *carry_slot(I, role, 0, cc);
            uc = *carry_slot(I, role, 1, cc);
            flp = *carry_slot(I, role, 2, cc);
            yp = *carry_slot(I, role, 3, cc);
            a3u = carry_slot(I, role, 4, cc)->x;
        }
        const RingA ring{warp_mem, lane};
        stream_rows<RingA::kDepth, 2>(jb - ja + 1,
                    [&](int r, int st) {
                        const int j = r + ja;
                        const size_t o = (size_t)j * nc, on = o - nc;
                        cp16(ring.at(st, 0), U + o + nc);
                        cp16(ring.at(st, 1), P + on);
                        if (kRK != 1) hint.cp_once(ring.at(st, 2), N + on);  // c_1 = 0: Nu_old unused
                        hint.cp_once(ring.at(st, 3), X + on);
                        hint.cp_once(ring.at(st, 4), FL + o);
                    },
                    [&](int r, int st) {
                        const int j = r + ja;
                        return RowA{*ring.at(st, 0), *ring.at(st, 1), *ring.at(st, 2), *ring.at(st, 3), *ring.at(st, 4),
                                    du[3 * j], du[3 * j + 1], du[3 * j + 2], sthu[j]};
                    },
                    [&](int r, const RowA &w) {
                        const int j = r + ja;
                        const size_t o = (size_t)j * nc, on = o - nc;
                        const double2 up = w.a, pj = w.b, x = w.d, fl = w.e;
                        const double2 no = kRK == 1 ? make_double2(0.0, 0.0) : w.c;
                        const double d1 = w.m0, d2 = w.m1, d3 = w.m2;
                        const double cen = k2x + k2z + d2;
                        const double2 L = make_double2(d1 * um.x + cen * uc.x + d3 * up.x, d1 * um.y + cen * uc.y + d3 * up.y);
                        double2 dd = make_double2(C1 * L.x + C2 * no.x + dC3 * pj.y, C1 * L.y + C2 * no.y + -(dC3 * pj.x));
                        if (role == 0 && mean) dd.x = dd.x + C1m;
                        const double m = w.m3;
                        const double2 nu = make_double2(x.x + (fl.x - flp.x) * m * ddv, x.y + (fl.y - flp.y) * m * ddv);
                        hint.st_once(N + on, nu);
                        dd = make_double2(dd.x + G * nu.x, dd.y + G * nu.y);
                        const double2 rh = make_double2(uc.x + dt * dd.x, uc.y + dt * dd.y);
                        const double a1 = -beta * d1;
                        const double a2 = 1.0 - beta * (d2 + k2x + k2z);
                        const double a3 = -beta * d3;
                        const double inv = 1.0 / (a2 - a1 * a3u);
                        const double2 y = make_double2((rh.x - a1 * yp.x) * inv, (rh.y - a1 * yp.y) * inv);
                        a3u = a3 * inv;
                        hint.st_back(YD + o, y);
                        if (role == 0) hint.st_back(FU + o, a3u);
                        yp = y;
                        um = uc;
                        uc = up;
                        flp = fl;
                    });
        if (jb == nyu) {
            // top row: a = [gw2, 1, 0], rhs = 0
            const double inv = 1.0 / (1.0 - I.gw2 * a3u);
            YD[(size_t)(nyu + 1) * nc] = make_double2((0.0 - I.gw2 * yp.x) * inv, (0.0 - I.gw2 * yp.y) * inv);
        } else {
            *carry_slot(I, role, 0, cc) = um;
            *carry_slot(I, role, 1, cc) = uc;
            *carry_slot(I, role, 2, cc) = flp;
            *carry_slot(I, role, 3, cc) = yp;
            *carry_slot(I, role, 4, cc) = make_double2(a3u, 0.0);
        }
    } else if (MODE != 2 && live && role == 2) {
        // u2: RHS0_u2 (littleharsh.f90:753-805) with laplacian_V, Nu2 sum,
        // solveU on the v grid; rows ja2 .. jb2 (one behind the u rows)
        const int ja2 = MODE == 1 ? max(1, ja - 1) : 1, jb2 = MODE == 1 ? jb - 1 : nyv;
        double2 *YD = MODE == 0 ? U2 : I.Y2 + cc;
        double2 *N = I.NU2 + cc;
        const double2 *X = I.NXZ2 + cc;
        const double2 *VV = I.VVC + cc;
        double2 um, uc, vvc, pc, yp;
        double a3v;
        if (ja2 == 1) {
            um = U2[0];
            uc = U2[(size_t)nc];
            vvc = VV[(size_t)nc];
            pc = P[0];
            a3v = 0.0 * 1.0;
            yp = make_double2(0.0, 0.0);
            YD[0] = yp;
            FV[0] = a3v;
        } else {
            um = *carry_slot(I, 2, 0, cc);
            uc = *carry_slot(I, 2, 1, cc);
            vvc = *carry_slot(I, 2, 2, cc);
            pc = *carry_slot(I, 2, 3, cc);
            yp = *carry_slot(I, 2, 4, cc);
            a3v = carry_slot(I, 2, 5, cc)->x;
        }
        const RingA ring{warp_mem, lane};
        stream_rows<RingA::kDepth, 2>(max(0, jb2 - ja2 + 1),
                    [&](int r, int st) {
                        const int j = r + ja2;
                        const size_t o = (size_t)j * nc, on = o - nc;
                        cp16(ring.at(st, 0), U2 + o + nc);
                        cp16(ring.at(st, 1), P + o);  // p(j+1)
                        if (kRK != 1) hint.cp_once(ring.at(st, 2), N + on);  // c_1 = 0: Nu_old unused
                        hint.cp_once(ring.at(st, 3), X + on);
                        hint.cp_once(ring.at(st, 4), VV + o + nc);
                    },
                    [&](int r, int st) {
                        const int j = r + ja2;
                        return RowA{*ring.at(st, 0), *ring.at(st, 1), *ring.at(st, 2), *ring.at(st, 3), *ring.at(st, 4),
                                    dv[3 * j], dv[3 * j + 1], dv[3 * j + 2], sthv[j]};
                    },
                    [&](int r, const RowA &w) {
                        const int j = r + ja2;
                        const size_t o = (size_t)j * nc, on = o - nc;
                        const double2 up = w.a, pn = w.b, x = w.d, vvn = w.e;
                        const double2 no = kRK == 1 ? make_double2(0.0, 0.0) : w.c;
                        const double e1 = w.m0, e2 = w.m1, e3 = w.m2;
                        const double cenv = k2x + k2z + e2;
                        const double2 L = make_double2(e1 * um.x + cenv * uc.x + e3 * up.x, e1 * um.y + cenv * uc.y + e3 * up.y);
                        const double mv = w.m3;
                        const double C3 = -rk.d * ddv * mv;
                        double2 dd = make_double2(C1 * L.x + C2 * no.x + C3 * (pn.x - pc.x), C1 * L.y + C2 * no.y + C3 * (pn.y - pc.y));
                        const double2 nu = make_double2(x.x + (vvn.x - vvc.x) * mv * ddv, x.y + (vvn.y - vvc.y) * mv * ddv);
                        hint.st_once(N + on, nu);
                        dd = make_double2(dd.x + G * nu.x, dd.y + G * nu.y);
                        const double2 rh = make_double2(uc.x + dt * dd.x, uc.y + dt * dd.y);
                        const double b1 = -beta * e1;
                        const double b2 = 1.0 - beta * (e2 + k2x + k2z);
                        const double b3 = -beta * e3;
                        const double inv = 1.0 / (b2 - b1 * a3v);
                        const double2 y = make_double2((rh.x - b1 * yp.x) * inv, (rh.y - b1 * yp.y) * inv);
                        a3v = b3 * inv;
                        hint.st_back(YD + o, y);
                        hint.st_back(FV + o, a3v);
                        yp = y;
                        um = uc;
                        uc = up;
                        vvc = vvn;
                        pc = pn;
                    });
        if (jb2 == nyv) {
            const double inv = 1.0 / (1.0 - 0.0 * a3v);
            YD[(size_t)(nyv + 1) * nc] = make_double2((0.0 - 0.0 * yp.x) * inv, (0.0 - 0.0 * yp.y) * inv);
        } else {
            *carry_slot(I, 2, 0, cc) = um;
            *carry_slot(I, 2, 1, cc) = uc;
            *carry_slot(I, 2, 2, cc) = vvc;
            *carry_slot(I, 2, 3, cc) = pc;
            *carry_slot(I, 2, 4, cc) = yp;
            *carry_slot(I, 2, 5, cc) = make_double2(a3v, 0.0);
        }
    }
    if (MODE == 1) return;
    if (MODE == 0) __syncthreads();

    // ---------------- B: back substitution (tridLU_3D.f90:80-82) ----------
    if (live) {
        double2 *U = role == 0 ? U1 : (role == 1 ? U3 : U2);
        // the eliminated rows: in place (MODE 0) or in the Y arrays (MODE 2)
        const double2 *YS = MODE == 0 ? U : (role == 0 ? I.Y1 : (role == 1 ? I.Y3 : I.Y2)) + cc;
        const double *F = role == 2 ? FV : FU;
        const int top = role == 2 ? nyv + 1 : nyu + 1;
        double2 v = YS[(size_t)top * nc];
        if (MODE == 2) U[(size_t)top * nc] = v;
        const RingW2 ring{warp_mem, lane};
        stream_rows<RingW2::kDepth, 4>(top,
                    [&](int r, int st) {
                        const int j = top - 1 - r;
                        cp16(ring.at(st, 0), YS + (size_t)j * nc);
                        cp8(&ring.at(st, 1)->x, F + (size_t)j * nc);
                    },
                    [&](int r, int st) { return RowB{*ring.at(st, 0), ring.at(st, 1)->x}; },
                    [&](int r, const RowB &w) {
                        const int j = top - 1 - r;
                        const double2 y = w.y;
                        const double f = w.f;
                        v = make_double2(y.x - f * v.x, y.y - f * v.y);
                        U[(size_t)j * nc] = v;
                    });
    }
    __syncthreads();

    const double dtirk = (1.0 / dt) / (rk.a + rk.b);
    if (live && role == 0) {
        if (I.flag_ctpress == 0 && mean) {
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
            __threadfence_block();
        }
        // ---------------- C: divergence and the LUsolP forward sweep -------
        // psi = div/(dt (a+b)) (littleharsh.f90:645-658), gauge psi(1) = 0 on
        // mode (0,0), forward elimination with the DG factors (tridLU_3D.f90:118-124)
        const double *G2 = I.DG2 + cc;
        double2 v2m = U2[0];
        double2 xp = make_double2(0.0, 0.0);
        const RingC ring{ring_mem, lane};
        stream_rows<RingC::kDepth, 4>(nyu,
                    [&](int r, int st) {
                        const int j = r + 1;
                        const size_t o = (size_t)j * nc;
                        cp16(ring.at(st, 0), U1 + o);
                        cp16(ring.at(st, 1), U3 + o);
                        cp16(ring.at(st, 2), U2 + o);
                        cp8(&ring.at(st, 3)->x, G2 + o - nc);
                    },
                    [&](int r, int st) {
                        const int j = r + 1;
                        return RowC{*ring.at(st, 0), *ring.at(st, 1), *ring.at(st, 2), ring.at(st, 3)->x, sthu[j], sdg1[j]};
                    },
                    [&](int r, const RowC &w) {
                        const int j = r + 1;
                        const double2 a = w.a, c3 = w.c3, v2c = w.v2c;
                        const double g2 = w.g2;
                        const double mm = ddv * w.th;
                        const double2 d = make_double2(-(kxr * a.y) + -(kzr * c3.y) + mm * (v2c.x - v2m.x),
                                                       kxr * a.x + kzr * c3.x + mm * (v2c.y - v2m.y));
                        double2 ps = cscale(dtirk, d);
                        if (mean && j == 1) ps = make_double2(0.0, 0.0);
                        if (j == 1) {
                            xp = cscale(g2, ps);
                        } else {
                            const double g1 = w.g1;
                            xp = make_double2((ps.x - g1 * xp.x) * g2, (ps.y - g1 * xp.y) * g2);
                        }
                        hint.st_back(PS + (size_t)(j - 1) * nc, xp);
                        v2m = v2c;
                    });
        // ---------------- D: LUsolP back sweep, p += psi and v_corr ---------
        // One downward sweep of the u1 warp (tridLU_3D.f90:125-127,
        // littleharsh.f90:660-664, v_corr :896-993): psi(j) from the forward
        // sweep's x(j), then row j of p, u1 and u3, and row j of u2 with
        // psi(j+1) of the previous row; psi itself is never stored.
        const double *G3 = I.DG3 + cc;
        const double dtrk = dt * (rk.a + rk.b);
        const double kd1 = dtrk * kxr, kd3 = dtrk * kzr, dtrk_u2 = dtrk * ddv;
        double2 psn = xp;  // psi(nyu) = x(nyu)
        double2 first1 = make_double2(0.0, 0.0), first3 = first1, last1 = first1, last3 = first1, ps1 = first1;
        const RingD ringd{ring_mem, lane};
        stream_rows<RingD::kDepth, 4>(nyu,
                    [&](int r, int st) {
                        const int j = nyu - r;
                        const size_t o = (size_t)(j - 1) * nc, oj = (size_t)j * nc;
                        hint.cp_once(ringd.at(st, 0), PS + o);
                        cp16(ringd.at(st, 1), P + o);
                        if (j < nyu) cp8(&ringd.at(st, 2)->x, G3 + o);
                        cp16(ringd.at(st, 3), U1 + oj);
                        cp16(ringd.at(st, 4), U3 + oj);
                        if (j <= nyv) cp16(ringd.at(st, 5), U2 + oj);
                    },
                    [&](int r, int st) {
                        const int j = nyu - r;
                        return RowD{*ringd.at(st, 0), *ringd.at(st, 1), *ringd.at(st, 3), *ringd.at(st, 4),
                                    *ringd.at(st, 5), j < nyu ? ringd.at(st, 2)->x : 0.0, sthv[j]};
                    },
                    [&](int r, const RowD &w) {
                        const int j = nyu - r;
                        const size_t o = (size_t)(j - 1) * nc, oj = (size_t)j * nc;
                        double2 ps = w.x;
                        if (j < nyu) ps = make_double2(w.x.x - w.g3 * psn.x, w.x.y - w.g3 * psn.y);
                        P[o] = make_double2(w.p.x + ps.x, w.p.y + ps.y);
                        const double2 a1 = make_double2(w.u1.x - -(kd1 * ps.y), w.u1.y - kd1 * ps.x);
                        const double2 a3 = make_double2(w.u3.x - -(kd3 * ps.y), w.u3.y - kd3 * ps.x);
                        U1[oj] = a1;
                        U3[oj] = a3;
                        if (j <= nyv) {
                            const double mv = dtrk_u2 * w.th;
                            U2[oj] = make_double2(w.u2.x - mv * (psn.x - ps.x), w.u2.y - mv * (psn.y - ps.y));
                        }
                        if (j == nyu) {
                            last1 = a1;
                            last3 = a3;
                        }
                        if (j == 1) {
                            first1 = a1;
                            first3 = a3;
                            ps1 = ps;
                        }
                        psn = ps;
                    });
        U1[0] = cscale(I.gwbc, first1);
        U1[(size_t)(nyu + 1) * nc] = cscale(I.gwbc, last1);
        U3[0] = cscale(I.gwbc, first3);
        U3[(size_t)(nyu + 1) * nc] = cscale(I.gwbc, last3);
        U2[0] = make_double2(0.0, 0.0);
        U2[(size_t)(nyv + 1) * nc] = make_double2(0.0, 0.0);
        if (!isfinite(first1.x) || !isfinite(first1.y) || !isfinite(first3.x) || !isfinite(first3.y) ||
            !isfinite(ps1.x) || !isfinite(ps1.y))
            atomicOr(I.err, ERR_NONFINITE);
        if (mean && kRK == 3) {
            // flowrateIm (littleharsh.f90:473-492) via meanflow_ctP (:572-589)
            __threadfence_block();
            double Qu = 0.0;
            for (int j = 1; j <= nyv + 1; j++) Qu = Qu + (I.yv[j] - I.yv[j - 1]) * U1[(size_t)j * nc].x;
            I.sc[SC_QX] = Qu;
            I.sc[SC_ITER] = I.sc[SC_ITER] + 1.0;
        }
    }
}

__global__ void __launch_bounds__(kColThreads *kRoles) k_column(const Inst *__restrict__ insts,
                                                                const Work *__restrict__ work, int kRK)
{
    column_body<0>(insts, work, kRK);
}

__global__ void __launch_bounds__(kColThreads *kRoles) k_column_a(const Inst *__restrict__ insts,
                                                                  const Work *__restrict__ work, int kRK)
{
    column_body<1>(insts, work, kRK);
}

__global__ void __launch_bounds__(kColThreads *kRoles) k_column_bcd(const Inst *__restrict__ insts,
                                                                    const Work *__restrict__ work, int kRK)
{
    column_body<2>(insts, work, kRK);
}

// ---------------------------------------------------------------------------
// Column pass for small mode counts: one CTA per column, the y rows spread
// over the lanes.  With few columns the sequential sweeps of k_column leave
// most SMs idle and the step waits on the per-row latency of 154-row
// recurrences; here every recurrence of the column pass -- the Helmholtz LU
// factors (a continued fraction), the forward and back substitutions and the
// LUsolP sweeps -- is a chain of per-row maps, each lane composes the maps of
// its block of rows, a warp scan (5 shuffle steps) gives every lane the value
// entering its block, and the lane then runs its rows with the reference's
// per-row arithmetic.  Only the values at block boundaries are formed in a
// different order (rounding differences of a few ulp; the per-row operations
// are the sequential ones).  The column's fields stay in shared memory
// between the phases, so besides the state only Nu and p are written.
// x -> (a x + b) / (c x + d), the LU-factor step a3u' = a3 / (a2 - a1 a3u)
struct Mob {
    double a, b, c, d;
};
__device__ __forceinline__ Mob mob_then(const Mob &m, const Mob &n)  // m after n
{
    Mob r{m.a * n.a + m.b * n.c, m.a * n.b + m.b * n.d, m.c * n.a + m.d * n.c, m.c * n.b + m.d * n.d};
    // rescale by a power of two (exact) so long products stay in range
    const double sc = fmax(fmax(fabs(r.a), fabs(r.b)), fmax(fabs(r.c), fabs(r.d)));
    if (sc > 0.0 && isfinite(sc)) {
        int e;
        frexp(sc, &e);
        r.a = ldexp(r.a, -e);
        r.b = ldexp(r.b, -e);
        r.c = ldexp(r.c, -e);
        r.d = ldexp(r.d, -e);
    }
    return r;
}
// y -> A + B y with complex A, real B (forward and back substitutions)
struct Aff {
    double2 A;
    double B;
};
__device__ __forceinline__ Aff aff_then(const Aff &m, const Aff &n)  // m after n
{
    return Aff{make_double2(m.A.x + m.B * n.A.x, m.A.y + m.B * n.A.y), m.B * n.B};
}
__device__ __forceinline__ Mob shfl_mob(const Mob &m, int o, bool up)
{
    Mob r;
    r.a = up ? __shfl_up_sync(0xffffffffu, m.a, o) : __shfl_down_sync(0xffffffffu, m.a, o);
    r.b = up ? __shfl_up_sync(0xffffffffu, m.b, o) : __shfl_down_sync(0xffffffffu, m.b, o);
    r.c = up ? __shfl_up_sync(0xffffffffu, m.c, o) : __shfl_down_sync(0xffffffffu, m.c, o);
    r.d = up ? __shfl_up_sync(0xffffffffu, m.d, o) : __shfl_down_sync(0xffffffffu, m.d, o);
    return r;
}
__device__ __forceinline__ Aff shfl_aff(const Aff &m, int o, bool up)
{
    Aff r;
    r.A.x = up ? __shfl_up_sync(0xffffffffu, m.A.x, o) : __shfl_down_sync(0xffffffffu, m.A.x, o);
    r.A.y = up ? __shfl_up_sync(0xffffffffu, m.A.y, o) : __shfl_down_sync(0xffffffffu, m.A.y, o);
    r.B = up ? __shfl_up_sync(0xffffffffu, m.B, o) : __shfl_down_sync(0xffffffffu, m.B, o);
    return r;
}
// Exclusive scans over the lanes: what enters lane l's block is the
// composition of the blocks before it (ascending rows) or after it
// (descending rows).
__device__ __forceinline__ Mob scan_mob_excl(Mob m, int lane)
{
    for (int o = 1; o < 32; o <<= 1) {
        const Mob other = shfl_mob(m, o, true);
        if (lane >= o) m = mob_then(m, other);
    }
    Mob e = shfl_mob(m, 1, true);
    if (lane == 0) e = Mob{1.0, 0.0, 0.0, 1.0};
    return e;
}
__device__ __forceinline__ Aff scan_aff_excl(Aff m, int lane, bool ascending)
{
    for (int o = 1; o < 32; o <<= 1) {
        const Aff other = shfl_aff(m, o, ascending);
        if (ascending ? lane >= o : lane + o < 32) m = aff_then(m, other);
    }
    Aff e = shfl_aff(m, 1, ascending);
    if (ascending ? lane == 0 : lane == 31) e = Aff{make_double2(0.0, 0.0), 1.0};
    return e;
}

// Helmholtz rows of one grid (solveU's LU_build, tridLU_3D.f90:163-221):
// row 0 [0, 1, w0], rows 1..n [-beta d1, 1 - beta (d2 + k2), -beta d3],
// row n+1 [wt, 1, 0]
struct HRow {
    double a1, a2, a3;
};
__device__ __forceinline__ HRow helm_row(int j, int n, const double *d, double beta, double k2x, double k2z,
                                         double w0, double wt)
{
    if (j == 0) return HRow{0.0, 1.0, w0 * 1.0};
    if (j == n + 1) return HRow{wt, 1.0, 0.0};
    return HRow{-beta * d[3 * j], 1.0 - beta * (d[3 * j + 1] + k2x + k2z), -beta * d[3 * j + 2]};
}

// LU factors of one grid's Helmholtz matrix for rows 0..n+1 into fac
// (a3u, the scaled upper diagonal) and inv (the inverse pivot), one warp.
__device__ void small_factors(int lane, int n, const double *d, double beta, double k2x, double k2z, double w0,
                              double wt, double *fac, double *inv)
{
    const int rows = n + 2, K = (rows + 31) / 32, r0 = lane * K, r1 = min(rows, r0 + K);
    Mob m{1.0, 0.0, 0.0, 1.0};
    for (int j = r0; j < r1; j++) {
        const HRow h = helm_row(j, n, d, beta, k2x, k2z, w0, wt);
        m = mob_then(Mob{0.0, h.a3, -h.a1, h.a2}, m);
    }
    const Mob e = scan_mob_excl(m, lane);
    double x = e.b / e.d;  // a3u entering the block (the block of row 0 ignores it)
    for (int j = r0; j < r1; j++) {
        const HRow h = helm_row(j, n, d, beta, k2x, k2z, w0, wt);
        const double iv = 1.0 / (h.a2 - h.a1 * x);
        x = h.a3 * iv;
        inv[j] = iv;
        fac[j] = x;
    }
}

// Forward and back substitution of one Helmholtz system, one warp: rh holds
// the right-hand side (rows 0 and n+1: zero) and receives the solution.
__device__ void small_solve(int lane, int n, const double *d, double beta, double k2x, double k2z, double w0,
                            double wt, const double *fac, const double *inv, double2 *rh)
{
    const int rows = n + 2, K = (rows + 31) / 32, r0 = lane * K, r1 = min(rows, r0 + K);
    // forward: y_j = (rh_j - a1_j y_{j-1}) inv_j
    Aff m{make_double2(0.0, 0.0), 1.0};
    for (int j = r0; j < r1; j++) {
        const double a1 = helm_row(j, n, d, beta, k2x, k2z, w0, wt).a1, iv = inv[j];
        const double2 r = rh[j];
        m = aff_then(Aff{make_double2(r.x * iv, r.y * iv), -(a1 * iv)}, m);
    }
    Aff e = scan_aff_excl(m, lane, true);
    double2 yp = e.A;
    for (int j = r0; j < r1; j++) {
        const double a1 = helm_row(j, n, d, beta, k2x, k2z, w0, wt).a1, iv = inv[j];
        const double2 r = rh[j];
        yp = make_double2((r.x - a1 * yp.x) * iv, (r.y - a1 * yp.y) * iv);
        rh[j] = yp;
    }
    __syncwarp();
    // back: u_j = y_j - fac_j u_{j+1} (fac of row n+1 is zero)
    m = Aff{make_double2(0.0, 0.0), 1.0};
    for (int j = r1 - 1; j >= r0; j--) m = aff_then(Aff{rh[j], -fac[j]}, m);
    e = scan_aff_excl(m, lane, false);
    double2 v = e.A;
    for (int j = r1 - 1; j >= r0; j--) {
        const double2 y = rh[j];
        const double f = fac[j];
        v = make_double2(y.x - f * v.x, y.y - f * v.y);
        rh[j] = v;
    }
    __syncwarp();
}

size_t column_small_smem_bytes(int max_nyu)
{
    const size_t R = (size_t)max_nyu + 2;
    // double2 rows: old u1 u3 u2, solved u1 u3 u2, psi, p; doubles: the two
    // grids' factors and pivots, DG2, DG3, and the y metrics (d2/dy2 of both
    // grids, dtheta/dy of both grids, DG1)
    return 8 * R * sizeof(double2) + 15 * R * sizeof(double);
}

__global__ void __launch_bounds__(32 * kSmallWarps) k_column_small(const Inst *__restrict__ insts,
                                                                   const Work *__restrict__ work, int kRK)
{
    extern __shared__ double2 sbuf[];
    const Work w = work[blockIdx.x];
    const Inst &I = insts[w.inst];
    const int col = w.j, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nc = I.nc, nxh = I.nxh, nyu = I.nyu, nyv = I.nyv, R = nyu + 2, Rv = nyv + 2;
    const int i = col % nxh, kr = col / nxh;
    const RK rk = rk_coeffs(kRK);
    const double dt = I.sc[SC_DT];
    const double Re = I.Re;
    const double C1 = rk.a / Re, C2 = -rk.c, G = -rk.g;
    const double kxr = I.kx[i], kzr = I.kz[kr];
    const double k2x = I.k2x[i], k2z = I.k2z[kr];
    const double beta = rk.b * dt / Re;
    const double ddv = I.ddthetavi;
    const bool mean = (col == 0);
    double2 *U1 = I.U1 + col, *U2 = I.U2 + col, *U3 = I.U3 + col, *P = I.P + col;
    // shared layout, R = nyu+2 rows per array (the v grid uses Rv = R-1);
    // rows of fields stored from j = 1 sit at index j-1
    double2 *O1 = sbuf, *O3 = O1 + R, *O2 = O3 + R;      // state before the substep
    double2 *S1 = O2 + R, *S3 = S1 + R, *S2 = S3 + R;    // right-hand sides -> solutions
    double2 *PS = S2 + R;                                 // psi, rows 1..nyu
    double2 *SP = PS + R;                                 // p, rows 1..nyu
    double *facu = reinterpret_cast<double *>(SP + R), *invu = facu + R, *facv = invu + R, *invv = facv + R;
    double *SG2 = invv + R, *SG3 = SG2 + R;               // DG2, DG3, rows 1..nyu

    // Stage the column and the y metrics: every load of a row is issued
    // before its stores.  The loads go through the read-only path: a CTA
    // reads only its own column here, before any of its writes.
    double *du = SG3 + R, *dv = du + 3 * R, *thu = dv + 3 * R, *thv = thu + R, *dg1 = thv + R;  // y metrics
    const double2 z2 = make_double2(0.0, 0.0);
    for (int j = threadIdx.x; j < R; j += blockDim.x) {
        const size_t o = (size_t)j * nc + col;
        const bool v = j < Rv, pr = j < nyu;
        const double2 a1 = __ldg(I.U1 + o), a3 = __ldg(I.U3 + o), a2 = v ? __ldg(I.U2 + o) : z2;
        const double2 pp = pr ? __ldg(I.P + o) : z2;
        const double g2 = pr ? __ldg(I.DG2 + o) : 0.0, g3 = pr ? __ldg(I.DG3 + o) : 0.0;
        const double m0 = __ldg(I.dyu2i + 3 * j), m1 = __ldg(I.dyu2i + 3 * j + 1), m2 = __ldg(I.dyu2i + 3 * j + 2);
        const double e0 = v ? __ldg(I.dyv2i + 3 * j) : 0.0, e1 = v ? __ldg(I.dyv2i + 3 * j + 1) : 0.0;
        const double e2 = v ? __ldg(I.dyv2i + 3 * j + 2) : 0.0;
        const double tu = __ldg(I.dthdyu + j), tv = v ? __ldg(I.dthdyv + j) : 0.0;
        const double d1 = j < nyu + 1 ? __ldg(I.DG1 + j) : 0.0;
        O1[j] = a1;
        O3[j] = a3;
        du[3 * j] = m0;
        du[3 * j + 1] = m1;
        du[3 * j + 2] = m2;
        thu[j] = tu;
        if (j < nyu + 1) dg1[j] = d1;
        if (v) {
            O2[j] = a2;
            dv[3 * j] = e0;
            dv[3 * j + 1] = e1;
            dv[3 * j + 2] = e2;
            thv[j] = tv;
        }
        if (pr) {
            SP[j] = pp;
            SG2[j] = g2;
            SG3[j] = g3;
        }
    }
    __syncthreads();
    // LU factors (u grid by warp 0, shared by the u1 and u3 chains, which
    // form identical factors in the reference; v grid by warp 2)
    if (warp == 0) small_factors(lane, nyu, du, beta, k2x, k2z, I.gw1, I.gw2, facu, invu);
    if (warp == 2) small_factors(lane, nyv, dv, beta, k2x, k2z, 0.0, 0.0, facv, invv);
    __syncthreads();

    // ---- right-hand sides (RHS0, Nu sum, du += -g Nu, solveU rhs) --------
    if (warp < 2) {
        const int role = warp;
        const double2 *O = role == 0 ? O1 : O3;
        const double2 *SN = (role == 0 ? I.NU1 : I.NU3) + col, *SX = (role == 0 ? I.NXZ1 : I.NXZ3) + col;
        const double2 *FL = (role == 0 ? I.UVF : I.WVF) + col;
        double2 *S = role == 0 ? S1 : S3;
        double2 *N = (role == 0 ? I.NU1 : I.NU3) + col;
        const double dC3 = rk.d * (role == 0 ? kxr : kzr);
        const double C1m = (role == 0 && mean) ? -rk.d * I.sc[SC_MPGX] : 0.0;
        // rows in batches of kSmallBatch per lane, every global load of a batch
        // issued before its arithmetic (the per-row operations are unchanged)
        for (int jb = lane; jb < R; jb += 32 * kSmallBatch) {
        double2 lno[kSmallBatch], lx[kSmallBatch], lfl[kSmallBatch], lflp[kSmallBatch];
#pragma unroll
        for (int b = 0; b < kSmallBatch; b++) {
            const int j = jb + 32 * b;
            lno[b] = lx[b] = lfl[b] = lflp[b] = z2;
            if (j >= 1 && j <= nyu) {
                const size_t o = (size_t)j * nc, on = o - nc;
                // Nu_old is overwritten below by the same thread: a plain load
                if (kRK != 1) lno[b] = SN[on];  // c_1 = 0: Nu_old unused at kRK = 1
                lx[b] = __ldg(SX + on);
                lfl[b] = __ldg(FL + o);
                lflp[b] = __ldg(FL + on);
            }
        }
#pragma unroll
        for (int b = 0; b < kSmallBatch; b++) {
            const int j = jb + 32 * b;
            if (j >= R) break;
            if (j == 0 || j == nyu + 1) {
                S[j] = make_double2(0.0, 0.0);
                continue;
            }
            const double2 um = O[j - 1], uc = O[j], up = O[j + 1];
            const double2 no = lno[b], x = lx[b], fl = lfl[b], flp = lflp[b];
            const double2 pj = SP[j - 1];
            const double d1 = du[3 * j], d2 = du[3 * j + 1], d3 = du[3 * j + 2];
            const double cen = k2x + k2z + d2;
            const double2 L = make_double2(d1 * um.x + cen * uc.x + d3 * up.x, d1 * um.y + cen * uc.y + d3 * up.y);
            double2 dd = make_double2(C1 * L.x + C2 * no.x + dC3 * pj.y, C1 * L.y + C2 * no.y + -(dC3 * pj.x));
            if (role == 0 && mean) dd.x = dd.x + C1m;
            const double m = thu[j];
            const double2 nu = make_double2(x.x + (fl.x - flp.x) * m * ddv, x.y + (fl.y - flp.y) * m * ddv);
            N[(size_t)(j - 1) * nc] = nu;
            dd = make_double2(dd.x + G * nu.x, dd.y + G * nu.y);
            S[j] = make_double2(uc.x + dt * dd.x, uc.y + dt * dd.y);
        }
        }
        __syncwarp();
        small_solve(lane, nyu, du, beta, k2x, k2z, I.gw1, I.gw2, facu, invu, S);
    } else {
        double2 *N = I.NU2 + col;
        const double2 *SN2 = I.NU2 + col, *SX2 = I.NXZ2 + col, *SVV = I.VVC + col;
        for (int jb = lane; jb < Rv; jb += 32 * kSmallBatch) {
        double2 lno[kSmallBatch], lx[kSmallBatch], lvc[kSmallBatch], lvn[kSmallBatch];
#pragma unroll
        for (int b = 0; b < kSmallBatch; b++) {
            const int j = jb + 32 * b;
            lno[b] = lx[b] = lvc[b] = lvn[b] = z2;
            if (j >= 1 && j <= nyv) {
                const size_t o = (size_t)j * nc, on = o - nc;
                // Nu_old is overwritten below by the same thread: a plain load
                if (kRK != 1) lno[b] = SN2[on];  // c_1 = 0: Nu_old unused at kRK = 1
                lx[b] = __ldg(SX2 + on);
                lvc[b] = __ldg(SVV + o);
                lvn[b] = __ldg(SVV + o + nc);
            }
        }
#pragma unroll
        for (int b = 0; b < kSmallBatch; b++) {
            const int j = jb + 32 * b;
            if (j >= Rv) break;
            if (j == 0 || j == nyv + 1) {
                S2[j] = make_double2(0.0, 0.0);
                continue;
            }
            const double2 um = O2[j - 1], uc = O2[j], up = O2[j + 1];
            const double2 no = lno[b], x = lx[b], vvc = lvc[b], vvn = lvn[b];
            const double2 pc = SP[j - 1], pn = SP[j];
            const double e1 = dv[3 * j], e2 = dv[3 * j + 1], e3 = dv[3 * j + 2];
            const double cenv = k2x + k2z + e2;
            const double2 L = make_double2(e1 * um.x + cenv * uc.x + e3 * up.x, e1 * um.y + cenv * uc.y + e3 * up.y);
            const double mv = thv[j];
            const double C3 = -rk.d * ddv * mv;
            double2 dd = make_double2(C1 * L.x + C2 * no.x + C3 * (pn.x - pc.x), C1 * L.y + C2 * no.y + C3 * (pn.y - pc.y));
            const double2 nu = make_double2(x.x + (vvn.x - vvc.x) * mv * ddv, x.y + (vvn.y - vvc.y) * mv * ddv);
            N[(size_t)(j - 1) * nc] = nu;
            dd = make_double2(dd.x + G * nu.x, dd.y + G * nu.y);
            S2[j] = make_double2(uc.x + dt * dd.x, uc.y + dt * dd.y);
        }
        }
        __syncwarp();
        small_solve(lane, nyv, dv, beta, k2x, k2z, 0.0, 0.0, facv, invv, S2);
    }
    __syncthreads();

    const double dtirk = (1.0 / dt) / (rk.a + rk.b);
    if (I.flag_ctpress == 0 && mean && threadIdx.x == 0) {
        // flowrate_corr (littleharsh.f90:515-548), as in k_column
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
        for (int j = 1; j <= nyv + 1; j++) Qx0 = Qx0 + (I.yv[j] - I.yv[j - 1]) * S1[j].x;
        const double g = (I.sc[SC_QXT] - Qx0) / Qx1;
        I.sc[SC_MPGX] = I.sc[SC_MPGX] + g;
        I.sc[SC_DGX] = g;
        for (int j = 0; j <= ne; j++) S1[j].x = S1[j].x + g * u11[j];
    }
    __syncthreads();

    // ---- divergence and LUsolP (warp 0), p += psi ------------------------
    if (warp == 0) {
        const int K = (nyu + 31) / 32, r0 = 1 + lane * K, r1 = min(nyu + 1, r0 + K);
        // psi = div / (dt (a+b)) into PS; forward x_j = (ps_j - g1_j x_{j-1}) g2_j, x_0 = 0
        Aff m{make_double2(0.0, 0.0), 1.0};
        for (int j = r0; j < r1; j++) {
            const double2 a = S1[j], c3 = S3[j], v2c = S2[j], v2m = S2[j - 1];
            const double mm = ddv * thu[j];
            const double2 d = make_double2(-(kxr * a.y) + -(kzr * c3.y) + mm * (v2c.x - v2m.x),
                                           kxr * a.x + kzr * c3.x + mm * (v2c.y - v2m.y));
            double2 ps = cscale(dtirk, d);
            if (mean && j == 1) ps = make_double2(0.0, 0.0);
            PS[j - 1] = ps;
            const double g2 = SG2[j - 1], g1 = j == 1 ? 0.0 : dg1[j];
            m = aff_then(Aff{make_double2(ps.x * g2, ps.y * g2), -(g1 * g2)}, m);
        }
        Aff e = scan_aff_excl(m, lane, true);
        double2 xp = e.A;
        for (int j = r0; j < r1; j++) {
            const double2 ps = PS[j - 1];
            const double g2 = SG2[j - 1];
            if (j == 1) xp = cscale(g2, ps);
            else {
                const double g1 = dg1[j];
                xp = make_double2((ps.x - g1 * xp.x) * g2, (ps.y - g1 * xp.y) * g2);
            }
            PS[j - 1] = xp;
        }
        __syncwarp();
        // back: psi_j = x_j - g3_j psi_{j+1} (psi_nyu = x_nyu); p += psi
        m = Aff{make_double2(0.0, 0.0), 1.0};
        for (int j = r1 - 1; j >= r0; j--) {
            const double g3 = j < nyu ? SG3[j - 1] : 0.0;
            m = aff_then(Aff{PS[j - 1], -g3}, m);
        }
        e = scan_aff_excl(m, lane, false);
        double2 psn = e.A;
        for (int j = r1 - 1; j >= r0; j--) {
            const double2 x = PS[j - 1];
            double2 ps = x;
            if (j < nyu) {
                const double g3 = SG3[j - 1];
                ps = make_double2(x.x - g3 * psn.x, x.y - g3 * psn.y);
            }
            PS[j - 1] = ps;
            const double2 pv = SP[j - 1];
            P[(size_t)(j - 1) * nc] = make_double2(pv.x + ps.x, pv.y + ps.y);
            psn = ps;
        }
    }
    __syncthreads();

    // ---- v_corr and the ghost rows (littleharsh.f90:896-993) -------------
    const double dtrk = dt * (rk.a + rk.b);
    if (warp < 2) {
        const int role = warp;
        double2 *S = role == 0 ? S1 : S3;
        double2 *U = role == 0 ? U1 : U3;
        const double kd = dtrk * (role == 0 ? kxr : kzr);
        for (int j = 1 + lane; j <= nyu; j += 32) {
            const double2 ps = PS[j - 1];
            double2 a = S[j];
            a = make_double2(a.x - -(kd * ps.y), a.y - kd * ps.x);
            S[j] = a;
            U[(size_t)j * nc] = a;
        }
        __syncwarp();
        if (lane == 0) {
            const double2 first = S[1], last = S[nyu], ps1 = PS[0];
            U[0] = cscale(I.gwbc, first);
            U[(size_t)(nyu + 1) * nc] = cscale(I.gwbc, last);
            if (!isfinite(first.x) || !isfinite(first.y) || !isfinite(ps1.x) || !isfinite(ps1.y))
                atomicOr(I.err, ERR_NONFINITE);
            if (role == 0 && mean && kRK == 3) {
                // flowrateIm (littleharsh.f90:473-492) via meanflow_ctP (:572-589)
                double Qu = 0.0;
                for (int j = 1; j <= nyv + 1; j++) Qu = Qu + (I.yv[j] - I.yv[j - 1]) * S1[j].x;
                I.sc[SC_QX] = Qu;
                I.sc[SC_ITER] = I.sc[SC_ITER] + 1.0;
            }
        }
    } else {
        const double dtrk_u2 = dtrk * ddv;
        for (int j = 1 + lane; j <= nyv; j += 32) {
            const double2 psc = PS[j - 1], psn = PS[j];
            const double mv = dtrk_u2 * thv[j];
            double2 v = S2[j];
            v = make_double2(v.x - mv * (psn.x - psc.x), v.y - mv * (psn.y - psc.y));
            U2[(size_t)j * nc] = v;
        }
        if (lane == 0) {
            U2[0] = make_double2(0.0, 0.0);
            U2[(size_t)(nyv + 1) * nc] = make_double2(0.0, 0.0);
        }
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
