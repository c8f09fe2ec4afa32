// Engine internals: device memory of an instance, the layout transforms at
// the host boundary, work tables and the launch sequence of a substep.
#include "lh_engine.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "lh_kernels.cuh"

namespace lh {

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// A kernel's dynamic shared-memory limit is process-wide and captured graphs
// of other plans may rely on it, so it is only ever raised.
cudaError_t raise_smem_limit(const void *func, size_t bytes)
{
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, func);
    if (e != cudaSuccess) return e;
    if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Plane fields (Mz x nxh complex) of the staging buffer for `chunk` planes:
// the fast path's Sin (chunk + 2 kRoundStreams rows x 3 fields: the rounds in
// flight each hold a share of the chunk plus a halo row on either side) and
// Sprod (chunk x 6); the generic path uses the first 6 * chunk.
size_t staging_units(int chunk) { return (size_t)(chunk + 2 * kRoundStreams) * 3 + (size_t)chunk * kNumProducts; }

// Bytes of plane staging one chunk round may use across all instances of a
// plan, kept well inside the 126 MB L2 (LH_STAGING_MB overrides, for tuning).
size_t staging_budget()
{
    const char *ev = getenv("LH_STAGING_MB");
    const long mb = ev ? atol(ev) : 0;
    return (size_t)(mb > 0 ? mb : 96) << 20;
}

Tiles default_tiles(int Mx, int Mz, int nxh, int nyu)
{
    Tiles t;
    const size_t target = 48 * 1024;
    t.bc_zinv = std::max(1, std::min(nxh, (int)(target / (32 * (size_t)Mz))));
    t.br_x = std::max(1, std::min(Mz, (int)(target / (96 * (size_t)Mx))));
    t.bc_zfwd = std::max(1, std::min(nxh, (int)(target / (192 * (size_t)Mz))));
    t.threads = 256;
    // staging capacity: the fast path holds 9 plane fields per plane plus 6
    // for the halo rows (staging_units), the generic path 6 per plane
    const size_t unit = (size_t)Mz * nxh * sizeof(double2);
    const size_t units = staging_budget() / unit;
    const size_t fixed = 6 * kRoundStreams;
    t.chunk = (int)std::max<size_t>(kRoundStreams, std::min<size_t>((size_t)nyu + kRoundStreams - 1,
                                                                  units > fixed ? (units - fixed) / 9 : kRoundStreams));
    return t;
}

size_t smem_zinv(const Tiles &t, int Mz) { return 2 * (size_t)Mz * t.bc_zinv * sizeof(double2); }
size_t smem_x(const Tiles &t, int Mx) { return 2 * (size_t)Mx * 3 * t.br_x * sizeof(double2); }
size_t smem_zfwd(const Tiles &t, int Mz) { return 2 * (size_t)Mz * kNumProducts * t.bc_zfwd * sizeof(double2); }

namespace {
struct Carver {
    size_t off = 0;
    char *base = nullptr;
    template <class T>
    T *take(size_t n)
    {
        size_t o = off;
        off = align256(off + n * sizeof(T));
        return base ? reinterpret_cast<T *>(base + o) : nullptr;
    }
};

// Lay out every buffer of an instance; with base == nullptr it only sizes.
void carve(const HostSetup &s, int chunk, Carver &c, Inst &I, double2 **stage, size_t *stage_elems)
{
    const size_t nc = s.nc, nu = s.nyu + 2, nv = s.nyv + 2, np = s.nyu;
    I.yu = c.take<double>(nu);
    I.yv = c.take<double>(nv);
    I.dthdyu = c.take<double>(nu);
    I.dthdyv = c.take<double>(nv);
    I.dyu2i = c.take<double>(3 * nu);
    I.dyv2i = c.take<double>(3 * nv);
    I.kx = c.take<double>(s.nxh);
    I.kz = c.take<double>(s.Nz);
    I.k2x = c.take<double>(s.nxh);
    I.k2z = c.take<double>(s.Nz);
    I.DG1 = c.take<double>(s.nyu + 1);
    I.DG2 = c.take<double>(np * nc);
    I.DG3 = c.take<double>(np * nc);
    I.twz = c.take<double2>(s.Mz);
    I.twx = c.take<double2>(s.Mx);
    I.U1 = c.take<double2>(nu * nc);
    I.U2 = c.take<double2>(nv * nc);
    I.U3 = c.take<double2>(nu * nc);
    I.P = c.take<double2>(np * nc);
    I.NU1 = c.take<double2>(np * nc);
    I.NU2 = c.take<double2>(np * nc);
    I.NU3 = c.take<double2>(np * nc);
    I.NXZ1 = c.take<double2>(np * nc);
    I.NXZ2 = c.take<double2>(np * nc);
    I.NXZ3 = c.take<double2>(np * nc);
    I.UVF = c.take<double2>((np + 1) * nc);
    I.WVF = c.take<double2>((np + 1) * nc);
    I.VVC = c.take<double2>(nu * nc);
    I.FACU = c.take<double>(nu * nc);
    I.FACV = c.take<double>(nv * nc);
    I.PSI = c.take<double2>(np * nc);
    I.Y1 = c.take<double2>(nu * nc);
    I.Y2 = c.take<double2>(nv * nc);
    I.Y3 = c.take<double2>(nu * nc);
    I.CARRY = c.take<double2>(18 * nc);
    I.U11 = c.take<double>(nu);
    I.F11 = c.take<double>(nu);
    I.S = c.take<double2>(staging_units(chunk) * s.Mz * s.nxh);
    I.sc = c.take<double>(SC_COUNT);
    I.err = c.take<int>(8);
    *stage_elems = nu * nc;
    *stage = c.take<double2>(*stage_elems);
}
}  // namespace

size_t instance_bytes(const HostSetup &hs, int chunk)
{
    Carver c;
    Inst I{};
    double2 *st;
    size_t se;
    carve(hs, chunk, c, I, &st, &se);
    return c.off;
}

cudaError_t instance_alloc(DevInstance &d, int chunk, cudaStream_t st, void *reuse, size_t reuse_bytes)
{
    const HostSetup &s = d.hs;
    Carver c;
    Inst &I = d.inst;
    memset(&I, 0, sizeof(I));
    carve(s, chunk, c, I, &d.stage, &d.stage_elems);
    d.bytes = c.off;
    cudaError_t e = cudaSuccess;
    if (reuse && reuse_bytes >= d.bytes) {
        d.block = reuse;
        d.alloc_bytes = reuse_bytes;
    } else {
        e = cudaMalloc(&d.block, d.bytes);
        if (e != cudaSuccess) {
            d.block = nullptr;
            return e;
        }
        d.alloc_bytes = d.bytes;
    }
    c = Carver();
    c.base = (char *)d.block;
    carve(s, chunk, c, I, &d.stage, &d.stage_elems);
    e = cudaMemsetAsync(d.block, 0, d.bytes, st);
    if (e != cudaSuccess) return e;
    auto up = [&](const void *dst, const void *src, size_t bytes) {
        if (e == cudaSuccess) e = cudaMemcpyAsync(const_cast<void *>(dst), src, bytes, cudaMemcpyHostToDevice, st);
    };
    up(I.yu, s.yu.data(), s.yu.size() * 8);
    up(I.yv, s.yv.data(), s.yv.size() * 8);
    up(I.dthdyu, s.dthdyu.data(), s.dthdyu.size() * 8);
    up(I.dthdyv, s.dthdyv.data(), s.dthdyv.size() * 8);
    up(I.dyu2i, s.dyu2i.data(), s.dyu2i.size() * 8);
    up(I.dyv2i, s.dyv2i.data(), s.dyv2i.size() * 8);
    up(I.kx, s.kx.data(), s.kx.size() * 8);
    up(I.kz, s.kz.data(), s.kz.size() * 8);
    up(I.k2x, s.k2x.data(), s.k2x.size() * 8);
    up(I.k2z, s.k2z.data(), s.k2z.size() * 8);
    up(I.DG1, s.DG1.data(), s.DG1.size() * 8);
    up(I.DG2, s.DG2.data(), s.DG2.size() * 8);
    up(I.DG3, s.DG3.data(), s.DG3.size() * 8);
    up(I.twz, s.twz.data(), s.twz.size() * 8);
    up(I.twx, s.twx.data(), s.twx.size() * 8);
    if (e != cudaSuccess) return e;
    I.Nx = s.Nx;
    I.Nz = s.Nz;
    I.Mx = s.Mx;
    I.Mz = s.Mz;
    I.nxh = s.nxh;
    I.nc = s.nc;
    I.nyu = s.nyu;
    I.nyv = s.nyv;
    I.dt_mode = d.desc.dt_mode;
    I.flag_ctpress = d.desc.flag_ctpress;
    I.nradz = (int)s.radz.size();
    I.nradx = (int)s.radx.size();
    for (int k = 0; k < I.nradz; k++) I.radz[k] = s.radz[k];
    for (int k = 0; k < I.nradx; k++) I.radx[k] = s.radx[k];
    I.Re = d.desc.Re;
    I.alp = d.desc.alp;
    I.bet = d.desc.bet;
    I.CFL = d.desc.CFL;
    I.dtv = s.dtv;
    I.dt_fixed = d.desc.dt;
    I.gw1 = s.gw1;
    I.gw2 = s.gw2;
    I.gwbc = s.gwbc;
    I.gwi1 = s.gwi1;
    I.gwi2 = s.gwi2;
    I.ddthetavi = s.ddthetavi;
    I.chunk = chunk;
    return cudaStreamSynchronize(st);
}

void instance_free(DevInstance &d)
{
    if (d.block) cudaFree(d.block);
    d.block = nullptr;
}

static cudaError_t upload_field(DevInstance &d, const double *src, double2 *dst, int len, cudaStream_t st)
{
    const int nc = d.hs.nc;
    if (!src) return cudaMemsetAsync(dst, 0, (size_t)len * nc * sizeof(double2), st);
    cudaError_t e = cudaMemcpyAsync(d.stage, src, (size_t)len * nc * sizeof(double2), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    dim3 grid((nc + 31) / 32, (len + 31) / 32), block(32, 8);
    k_col_to_plane<<<grid, block, 0, st>>>(d.stage, dst, len, nc);
    return cudaGetLastError();
}

cudaError_t download_field(const DevInstance &d, const double2 *src, int len, double *dst, cudaStream_t st)
{
    const int nc = d.hs.nc;
    dim3 grid((nc + 31) / 32, (len + 31) / 32), block(32, 8);
    k_plane_to_col<<<grid, block, 0, st>>>(src, d.stage, len, nc);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(dst, d.stage, (size_t)len * nc * sizeof(double2), cudaMemcpyDeviceToHost, st);
}

// The fields but p, the Nu reset and the scalars of an upload (getini).
static cudaError_t upload_without_p(DevInstance &d, const double *u1, const double *u2, const double *u3,
                                    cudaStream_t st)
{
    const HostSetup &s = d.hs;
    Inst &I = d.inst;
    cudaError_t e;
    if ((e = upload_field(d, u1, I.U1, s.nyu + 2, st)) != cudaSuccess) return e;
    if ((e = upload_field(d, u2, I.U2, s.nyv + 2, st)) != cudaSuccess) return e;
    if ((e = upload_field(d, u3, I.U3, s.nyu + 2, st)) != cudaSuccess) return e;
    const size_t npc = (size_t)s.nyu * s.nc * sizeof(double2);
    // Nu = 0 before the first step (littleharsh.f90:127-129)
    if ((e = cudaMemsetAsync(I.NU1, 0, npc, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(I.NU2, 0, npc, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(I.NU3, 0, npc, st)) != cudaSuccess) return e;
    double sc[SC_COUNT] = {0};
    sc[SC_T] = 0.0;
    sc[SC_DT] = d.desc.dt_mode == LH_DT_FIXED ? d.desc.dt : 0.0;
    sc[SC_MPGX] = d.desc.mpgx;
    const double q = u1 ? flowrate_host(s, u1) : 0.0;
    sc[SC_QX] = q;
    sc[SC_QXT] = q;  // getini: QxT = Qx for the constant flow-rate mode
    if ((e = cudaMemcpyAsync(I.sc, sc, sizeof(sc), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    return cudaMemsetAsync(I.err, 0, sizeof(int), st);
}

cudaError_t instance_upload(DevInstance &d, const double *u1, const double *u2, const double *u3, const double *p,
                            cudaStream_t st)
{
    cudaError_t e = upload_without_p(d, u1, u2, u3, st);
    if (e == cudaSuccess) e = upload_field(d, p, d.inst.P, d.hs.nyu, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

cudaError_t instance_upload_p_last(DevInstance &d, const double *u1, const double *u2, const double *u3,
                                   const double *p, cudaStream_t st, cudaEvent_t ev_u)
{
    cudaError_t e = upload_without_p(d, u1, u2, u3, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev_u, st);
    if (e == cudaSuccess) e = upload_field(d, p, d.inst.P, d.hs.nyu, st);
    return e;
}

cudaError_t instance_download(DevInstance &d, double *u1, double *u2, double *u3, double *p, cudaStream_t st)
{
    const HostSetup &s = d.hs;
    const Inst &I = d.inst;
    cudaError_t e = cudaSuccess;
    if (u1 && (e = download_field(d, I.U1, s.nyu + 2, u1, st)) != cudaSuccess) return e;
    if (u2 && (e = download_field(d, I.U2, s.nyv + 2, u2, st)) != cudaSuccess) return e;
    if (u3 && (e = download_field(d, I.U3, s.nyu + 2, u3, st)) != cudaSuccess) return e;
    if (p && (e = download_field(d, I.P, s.nyu, p, st)) != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

// Whether the sequential column pass is split into forward-sweep chunks
// beside the plane rounds (LH_COLUMN_SPLIT=0/1 overrides).
constexpr bool kColumnSplitDefault = false;

// Plans with at most this many columns in all use the one-CTA-per-column
// column pass (LH_SMALL_COLUMNS overrides).
constexpr long kSmallColumnsDefault = 1536;

// ---------------------------------------------------------------------------
namespace {
struct ClassTiles {
    bool fast;
    int cbz, rbx, cbf;
    int tz, tx, tf;
    size_t smz, smx, smf;
};

// Fast-path launch shapes from upper bounds on the x modes per z-inverse
// CTA, the z rows per x CTA and the x modes per z-forward CTA; every bound is
// lowered until the block fits the kernel's launch bounds and 110 KB of
// shared memory, and the x-mode blocks are balanced.
ClassTiles fast_tiles(const HostSetup &s, int cbz_max, int rb, int cbf_max)
{
    ClassTiles c{};
    c.fast = true;
    const size_t smax = 110 * 1024;
    auto fits = [&](int stage, int M, int vectors, int per) {
        return fast_threads(M, vectors) <= fast_max_threads(stage) && (size_t)M * per * 16 <= smax;
    };
    cbz_max = std::max(1, std::min(cbz_max, s.nxh));
    while (cbz_max > 1 && !fits(0, s.Mz, cbz_max, cbz_max)) cbz_max--;
    int nb = (s.nxh + cbz_max - 1) / cbz_max;
    c.cbz = (s.nxh + nb - 1) / nb;
    c.tz = fast_threads(s.Mz, c.cbz);
    c.smz = zinv_smem(s.Mz, c.cbz);
    rb = std::max(1, std::min(rb, s.Mz));
    // the x stage's vectors sit at an odd row stride (3 rb rounded up to odd)
    while (rb > 1 && !(xprod_threads(s.Mx, rb) <= xprod_max_threads(s.Mx) && xprod_smem(s.Mx, rb) <= smax)) rb--;
    c.rbx = rb;
    c.tx = xprod_threads(s.Mx, rb);
    c.smx = xprod_smem(s.Mx, rb);
    cbf_max = std::max(1, std::min(cbf_max, s.nxh));
    // z forward: one half of the six products (3 vectors per x mode) per CTA
    while (cbf_max > 1 && !(zfwd_threads(s.Mz, cbf_max) <= fast_max_threads(2) && zfwd_smem(s.Mz, cbf_max) <= smax))
        cbf_max--;
    nb = (s.nxh + cbf_max - 1) / cbf_max;
    c.cbf = (s.nxh + nb - 1) / nb;
    c.tf = zfwd_threads(s.Mz, c.cbf);
    c.smf = zfwd_smem(s.Mz, c.cbf);
    return c;
}

// Default tile bounds of a fast size: measured on B200 at 128^2 (16 threads
// per vector): 16 x modes per z-inverse CTA, 4 z rows per x CTA, up to 4 x
// modes per z-forward CTA; sizes with fewer threads per vector take
// proportionally more, the x stage at 18 and more one z row.  The z-forward bound is 80/vz, one less at Mz = 96
// and 192 (ny = 153 sweeps: one x mode fewer was faster there, slower at
// Mz = 288 and 384, even at 48).
void default_bounds(const HostSetup &s, int &cbz, int &rbx, int &cbf)
{
    const int vz = std::max(1, fast_vector_threads(s.Mz)), vx = std::max(1, fast_vector_threads(s.Mx));
    cbz = 256 / vz;
    // the multi-plane x stage holds seven vectors per z row: one row group;
    // the block-synchronous stage at 18 and 24 threads per vector (Ngal 288,
    // 384) is fastest with one z row per CTA (autotuner on B200: 192^2 x 257
    // 5.43 -> 5.07 ms per step, 256^2 x 257 10.11 -> 9.76)
    rbx = vx >= 18 && !xprod_warp(s.Mx) ? 1 : std::max(1, (xprod_multi(s.Mx) ? 32 : 64) / vx);
    cbf = std::max(1, 80 / vz - ((s.Mz == 96 || s.Mz == 192) ? 1 : 0));
}

// Tile bounds of a class: the autotuner's candidate, else the environment
// override LH_TILES=cbz,rbx,cbf, else the tuned table, else the defaults.
ClassTiles class_tiles(const HostSetup &s, bool force_generic, const TuneParams *force)
{
    ClassTiles c{};
    c.fast = !force_generic && fast_size(s.Mz) && fast_size(s.Mx);
    if (c.fast) {
        int a = 0, b = 0, d = 0;
        default_bounds(s, a, b, d);
        TuneParams tp;
        const char *ov = getenv("LH_TILES");
        int oa = 0, ob = 0, od = 0;
        if (force && force->cbz > 0) {
            a = force->cbz;
            b = force->rbx;
            d = force->cbf;
        } else if (ov && sscanf(ov, "%d,%d,%d", &oa, &ob, &od) == 3 && oa > 0 && ob > 0 && od > 0) {
            a = oa;
            b = ob;
            d = od;
        } else if (tune_lookup(s.Mz, s.Mx, s.nyu, tp) && tp.cbz > 0) {
            a = tp.cbz;
            b = tp.rbx;
            d = tp.cbf;
        }
        c = fast_tiles(s, a, b, d);
    } else {
        Tiles t = default_tiles(s.Mx, s.Mz, s.nxh, s.nyu);
        c.cbz = t.bc_zinv;
        c.rbx = t.br_x;
        c.cbf = t.bc_zfwd;
        c.tz = c.tx = c.tf = t.threads;
        c.smz = smem_zinv(t, s.Mz);
        c.smx = smem_x(t, s.Mx);
        c.smf = smem_zfwd(t, s.Mz);
    }
    return c;
}
}  // namespace

TuneParams default_params(const HostSetup &s)
{
    TuneParams t;
    if (fast_size(s.Mz) && fast_size(s.Mx)) default_bounds(s, t.cbz, t.rbx, t.cbf);
    t.staging_mb = (int)(staging_budget() >> 20);
    t.col_waves = 1;
    return t;
}

cudaError_t plan_build(Plan &p, const std::vector<const DevInstance *> &insts, bool force_generic,
                       const TuneParams *force)
{
    // the work buffer, side stream and events survive a rebuild
    p.rounds.clear();
    p.column.clear();
    p.force_generic = force_generic;
    p.ninst = (int)insts.size();
    // size classes in order of first appearance
    std::vector<std::pair<int, int>> classes;
    std::vector<int> cls_of(insts.size());
    int rounds = 0;
    for (size_t q = 0; q < insts.size(); q++) {
        const HostSetup &s = insts[q]->hs;
        std::pair<int, int> key(s.Mz, s.Mx);
        auto it = std::find(classes.begin(), classes.end(), key);
        if (it == classes.end()) {
            classes.push_back(key);
            it = classes.end() - 1;
        }
        cls_of[q] = (int)(it - classes.begin());
    }
    // Planes per round: the staging of one round, summed over every instance
    // of the plan, stays inside the L2 budget so staging never reaches HBM.
    const size_t ncls = classes.size();
    std::vector<ClassTiles> tiles(ncls);
    std::vector<const HostSetup *> rep(ncls, nullptr);
    for (size_t q = 0; q < insts.size(); q++)
        if (!rep[cls_of[q]]) rep[cls_of[q]] = &insts[q]->hs;
    for (size_t c = 0; c < ncls; c++) tiles[c] = class_tiles(*rep[c], force_generic, force);
    // staging budget and column-pass launches: the candidate, else the
    // environment, else the tuned entry of a single-class plan, else defaults
    TuneParams tuned;
    const bool have_tuned = ncls == 1 && tune_lookup(rep[0]->Mz, rep[0]->Mx, rep[0]->nyu, tuned);
    size_t l2_budget = staging_budget();
    if (force && force->staging_mb > 0) l2_budget = (size_t)force->staging_mb << 20;
    else if (!getenv("LH_STAGING_MB") && have_tuned && tuned.staging_mb > 0) l2_budget = (size_t)tuned.staging_mb << 20;
    std::vector<int> chunk_eff(insts.size());
    for (size_t q = 0; q < insts.size(); q++) {
        const HostSetup &s = insts[q]->hs;
        const bool fast = tiles[cls_of[q]].fast;
        const size_t unit = (size_t)s.Mz * s.nxh * sizeof(double2);
        const size_t units = l2_budget / (unit * insts.size());
        // kRoundStreams rounds are in flight (round r on stream r %
        // kRoundStreams), each with its share of the staging.  The L2 share
        // shrinks with the number of instances; below nyu/8 planes per round
        // the launch count costs more than staging spilling to HBM, so that
        // is the floor (within the allocated capacity).
        const size_t fixed = 6 * kRoundStreams;
        size_t c = fast ? (units > fixed ? (units - fixed) / 9 : kRoundStreams) : units / kNumProducts;
        c = std::max<size_t>(c / kRoundStreams, (size_t)(s.nyu + 7) / 8);
        c = std::max<size_t>(1, std::min<size_t>(c, (size_t)insts[q]->inst.chunk / kRoundStreams));
        // the multi-plane x stage's groups start at absolute planes 1 + kXGroup g,
        // so rounds hold whole groups
        if (fast && xprod_multi(s.Mx) && c >= (size_t)kXGroup) c -= c % kXGroup;
        chunk_eff[q] = (int)c;
        rounds = std::max(rounds, (s.nyu + chunk_eff[q] - 1) / chunk_eff[q]);
    }
    // The column pass: with few columns in the plan, one CTA per column with
    // the rows spread over its lanes (k_column_small); otherwise 32 columns
    // per CTA, one lane each (k_column).
    size_t total_cols = 0;
    for (const DevInstance *d : insts) total_cols += (size_t)d->hs.nc;
    const char *sc = getenv("LH_SMALL_COLUMNS");
    const long small_max = sc ? atol(sc) : kSmallColumnsDefault;
    p.col_small = (long)total_cols <= small_max;
    // Column blocks split over this many back-to-back launches (LH_COLUMN_WAVES):
    // fewer columns in flight keep the pass's intermediates in L2.
    const char *cw = getenv("LH_COLUMN_WAVES");
    p.col_waves = force && force->col_waves > 0 ? force->col_waves
                  : cw ? std::max(1, atoi(cw))
                  : (have_tuned && tuned.col_waves > 0 ? tuned.col_waves : 1);
    // work lists [round][stage][class]
    std::vector<std::vector<std::vector<std::vector<Work>>>> lists(
        rounds, std::vector<std::vector<std::vector<Work>>>(3, std::vector<std::vector<Work>>(ncls)));
    p.column.clear();
    for (int q = 0; q < (int)insts.size(); q++) {
        const HostSetup &s = insts[q]->hs;
        const ClassTiles &ct = tiles[cls_of[q]];
        const int chunk = chunk_eff[q];
        const int nbz = (s.nxh + ct.cbz - 1) / ct.cbz;
        const int nbx = (s.Mz + ct.rbx - 1) / ct.rbx;
        const int nbf = (s.nxh + ct.cbf - 1) / ct.cbf;
        if (ct.fast) {
            // round r: planes j0..j1 in staging half r%2; Sin slot sb+p holds
            // y row j0-1+p (u1/u3 on rows j0..j1+1, u2 on rows j0-1..j1),
            // Sprod slot pb+j-j0 plane j
            for (int j0 = 1, r = 0; j0 <= s.nyu; j0 += chunk, r++) {
                const int j1 = std::min(s.nyu, j0 + chunk - 1);
                const int sb = (r % kRoundStreams) * (chunk + 2), pb = (r % kRoundStreams) * chunk;
                auto &L = lists[r];
                for (int jp = j0 - 1; jp <= j1 + 1; jp++)
                    for (int f = 0; f < 3; f++) {
                        if (f < 2 ? jp < j0 : jp > j1) continue;
                        for (int b = 0; b < nbz; b++)
                            L[0][cls_of[q]].push_back({q, jp, sb + jp - j0 + 1, f * nbz + b, 0});
                    }
                if (xprod_multi(s.Mx))
                    for (int j = j0; j <= j1; j += kXGroup) {
                        const int np = std::min(kXGroup, j1 - j + 1);
                        for (int b = 0; b < nbx; b++)
                            L[1][cls_of[q]].push_back({q, j, pb + j - j0, b | (np << 16), sb + j - j0});
                    }
                for (int j = j0; j <= j1; j++) {
                    if (!xprod_multi(s.Mx))
                        for (int b = 0; b < nbx; b++) L[1][cls_of[q]].push_back({q, j, pb + j - j0, b, sb + j - j0});
                    for (int b = 0; b < nbf; b++)
                        for (int h = 0; h < 2; h++) L[2][cls_of[q]].push_back({q, j, pb + j - j0, 2 * b + h, 0});
                }
            }
        } else {
            for (int j = 1; j <= s.nyu; j++) {
                const int r = (j - 1) / chunk, slot = (r % kRoundStreams) * chunk + (j - 1) % chunk;
                auto &L = lists[r];
                for (int f = 0; f < kNumProducts; f++)
                    for (int b = 0; b < nbz; b++) L[0][cls_of[q]].push_back({q, j, slot, f * nbz + b, 0});
                for (int b = 0; b < nbx; b++) L[1][cls_of[q]].push_back({q, j, slot, b, 0});
                for (int b = 0; b < nbf; b++) L[2][cls_of[q]].push_back({q, j, slot, b, 0});
            }
        }
        if (p.col_small)
            for (int c = 0; c < s.nc; c++) p.column.push_back({q, c, 0, 0, 0});
        else
            for (int b = 0; b < (s.nc + kColumnThreads - 1) / kColumnThreads; b++) p.column.push_back({q, b, 0, 0, 0});
    }
    std::vector<Work> all;
    p.rounds.assign(rounds, {});
    for (int r = 0; r < rounds; r++)
        for (int stg = 0; stg < 3; stg++)
            for (size_t c = 0; c < ncls; c++) {
                const auto &v = lists[r][stg][c];
                if (v.empty()) continue;
                Group g;
                g.stage = stg;
                g.fast = tiles[c].fast;
                g.Mz = classes[c].first;
                g.Mx = classes[c].second;
                g.off = all.size();
                g.count = v.size();
                g.threads = stg == 0 ? tiles[c].tz : stg == 1 ? tiles[c].tx : tiles[c].tf;
                g.smem = stg == 0 ? tiles[c].smz : stg == 1 ? tiles[c].smx : tiles[c].smf;
                g.param = stg == 0 ? tiles[c].cbz : stg == 1 ? tiles[c].rbx : tiles[c].cbf;
                g.grid = (unsigned)g.count;
                all.insert(all.end(), v.begin(), v.end());
                p.rounds[r].push_back(g);
            }
    p.off_column = all.size();
    all.insert(all.end(), p.column.begin(), p.column.end());
    // split column pass: per round, every instance's rows of that round x its
    // column blocks; plus one chunk of all rows
    const char *cs = getenv("LH_COLUMN_SPLIT");
    p.col_split = !p.col_small && (cs ? cs[0] == '1' : kColumnSplitDefault);
    p.col_a.assign(rounds, {0, 0});
    p.off_col_full = p.n_col_full = 0;
    if (p.col_split) {
        for (int r = 0; r < rounds; r++) {
            p.col_a[r].first = all.size();
            for (int q = 0; q < (int)insts.size(); q++) {
                const HostSetup &s = insts[q]->hs;
                const int j0 = 1 + r * chunk_eff[q];
                if (j0 > s.nyu) continue;
                const int j1 = std::min(s.nyu, j0 + chunk_eff[q] - 1);
                for (int b = 0; b < (s.nc + kColumnThreads - 1) / kColumnThreads; b++) all.push_back({q, b, j0, j1, 0});
            }
            p.col_a[r].second = all.size() - p.col_a[r].first;
        }
        p.off_col_full = all.size();
        for (int q = 0; q < (int)insts.size(); q++) {
            const HostSetup &s = insts[q]->hs;
            for (int b = 0; b < (s.nc + kColumnThreads - 1) / kColumnThreads; b++) all.push_back({q, b, 1, s.nyu, 0});
        }
        p.n_col_full = all.size() - p.off_col_full;
    }
    cudaError_t e = cudaSuccess;
    if (p.col_split) {
        if (!p.side_a) e = cudaStreamCreateWithFlags(&p.side_a, cudaStreamNonBlocking);
        if (e == cudaSuccess && !p.ev_a) e = cudaEventCreateWithFlags(&p.ev_a, cudaEventDisableTiming);
        while (e == cudaSuccess && p.ev_round.size() < (size_t)rounds) {
            cudaEvent_t ev = nullptr;
            e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (e == cudaSuccess) p.ev_round.push_back(ev);
        }
        if (e != cudaSuccess) return e;
    }
    if (!p.ev_fork) e = cudaEventCreateWithFlags(&p.ev_fork, cudaEventDisableTiming);
    for (int k = 0; k < kRoundStreams - 1 && e == cudaSuccess; k++) {
        if (!p.side[k]) e = cudaStreamCreateWithFlags(&p.side[k], cudaStreamNonBlocking);
        if (e == cudaSuccess && !p.ev_join[k]) e = cudaEventCreateWithFlags(&p.ev_join[k], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return e;
    if (all.size() > p.work_cap) {
        if (p.d_work) cudaFree(p.d_work);
        p.d_work = nullptr;
        p.work_cap = 0;
        e = cudaMalloc(&p.d_work, all.size() * sizeof(Work));
        if (e != cudaSuccess) {
            p.d_work = nullptr;
            return e;
        }
        p.work_cap = all.size();
    }
    e = cudaMemcpy(p.d_work, all.data(), all.size() * sizeof(Work), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    // dynamic shared-memory limits for every kernel this plan launches
    size_t gz = 0, gx = 0, gf = 0;
    for (size_t c = 0; c < ncls; c++) {
        if (tiles[c].fast) {
            if ((e = fast_set_attributes(classes[c].first, classes[c].second, tiles[c].smz, tiles[c].smx,
                                         tiles[c].smf)) != cudaSuccess)
                return e;
        } else {
            gz = std::max(gz, tiles[c].smz);
            gx = std::max(gx, tiles[c].smx);
            gf = std::max(gf, tiles[c].smf);
        }
    }
    if (gz && (e = raise_smem_limit((const void *)k_zinv, gz)) != cudaSuccess) return e;
    if (gx && (e = raise_smem_limit((const void *)k_xprod, gx)) != cudaSuccess) return e;
    if (gf && (e = raise_smem_limit((const void *)k_zfwd, gf)) != cudaSuccess) return e;
    int max_nyu = 1;
    for (const DevInstance *d : insts) max_nyu = std::max(max_nyu, d->hs.nyu);
    if (p.col_small) {
        p.sm_col = column_small_smem_bytes(max_nyu);
        return raise_smem_limit((const void *)k_column_small, p.sm_col);
    }
    p.sm_col = column_smem_bytes(max_nyu);
    if ((e = raise_smem_limit((const void *)k_column_a, p.sm_col)) != cudaSuccess) return e;
    if ((e = raise_smem_limit((const void *)k_column_bcd, p.sm_col)) != cudaSuccess) return e;
    return raise_smem_limit((const void *)k_column, p.sm_col);
}

void plan_free(Plan &p)
{
    if (p.d_work) cudaFree(p.d_work);
    p.d_work = nullptr;
    p.work_cap = 0;
    if (p.ev_fork) cudaEventDestroy(p.ev_fork);
    p.ev_fork = nullptr;
    for (int k = 0; k < kRoundStreams - 1; k++) {
        if (p.ev_join[k]) cudaEventDestroy(p.ev_join[k]);
        if (p.side[k]) cudaStreamDestroy(p.side[k]);
        p.ev_join[k] = nullptr;
        p.side[k] = nullptr;
    }
    p.rounds.clear();
    for (cudaEvent_t ev : p.ev_round) cudaEventDestroy(ev);
    p.ev_round.clear();
    if (p.ev_a) cudaEventDestroy(p.ev_a);
    p.ev_a = nullptr;
    if (p.side_a) cudaStreamDestroy(p.side_a);
    p.side_a = nullptr;
}

static void time_begin(LaunchTimer *t, cudaStream_t st)
{
    if (t) cudaEventRecord(t->ev[0], st);
}

static cudaError_t time_end(LaunchTimer *t, int cls, cudaStream_t st)
{
    if (!t) return cudaSuccess;
    cudaEventRecord(t->ev[1], st);
    cudaError_t e = cudaEventSynchronize(t->ev[1]);
    float f = 0.f;
    cudaEventElapsedTime(&f, t->ev[0], t->ev[1]);
    t->ms[cls] += f;
    t->n[cls] += 1;
    return e;
}

cudaError_t launch_substep(const Plan &p, const Inst *d_insts, int kRK, bool cfl_any, cudaStream_t st,
                           LaunchTimer *timer, cudaEvent_t before_column)
{
    const int want_max = (kRK == 1 && cfl_any) ? 1 : 0;
    cudaError_t e = cudaSuccess;
    // a split column pass reads p in the forward-sweep chunks beside the
    // plane rounds: there the whole substep waits for before_column
    if (before_column && p.col_split) {
        if ((e = cudaStreamWaitEvent(st, before_column, cudaEventWaitExternal)) != cudaSuccess) return e;
        before_column = nullptr;
    }
    // round r on stream r % kRoundStreams (0 = st; their staging shares are
    // disjoint), forked from st after the work the plane pass depends on and
    // joined back before the work that consumes it; timed profiles keep one
    // stream
    const int nstreams = (timer == nullptr && p.side[0] != nullptr)
                             ? (int)std::min<size_t>(kRoundStreams, p.rounds.size()) : 1;
    if (nstreams > 1) {
        if ((e = cudaEventRecord(p.ev_fork, st)) != cudaSuccess) return e;
        for (int k = 0; k < nstreams - 1; k++)
            if ((e = cudaStreamWaitEvent(p.side[k], p.ev_fork, 0)) != cudaSuccess) return e;
    }
    // forward-sweep chunks beside the plane rounds (split column pass; not
    // when dt is only known after the plane pass, nor in timed profiles)
    const bool a_beside = p.col_split && !(kRK == 1 && cfl_any);
    const bool a_stream = a_beside && timer == nullptr && p.side_a != nullptr;
    if (a_stream) {
        if (nstreams <= 1 && (e = cudaEventRecord(p.ev_fork, st)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(p.side_a, p.ev_fork, 0)) != cudaSuccess) return e;
    }
    for (size_t ri = 0; ri < p.rounds.size(); ri++) {
        for (const Group &g : p.rounds[ri]) {
            const Work *w = p.d_work + g.off;
            const unsigned n = (unsigned)g.count;
            const int si = (int)(ri % kRoundStreams);
            cudaStream_t st0 = st;
            cudaStream_t st = (nstreams > 1 && si > 0) ? p.side[si - 1] : st0;
            time_begin(timer, st);
            if (g.fast) {
                const int cnt = (int)g.count;
                if (g.stage == 0) fast_launch_zinv(g.Mz, g.grid, g.threads, g.smem, st, d_insts, w, cnt, g.param);
                else if (g.stage == 1)
                    fast_launch_xprod(g.Mx, g.grid, g.threads, g.smem, st, d_insts, w, cnt, g.param, want_max);
                else fast_launch_zfwd(g.Mz, g.grid, g.threads, g.smem, st, d_insts, w, cnt, g.param);
            } else {
                if (g.stage == 0) k_zinv<<<n, g.threads, g.smem, st>>>(d_insts, w, g.param);
                else if (g.stage == 1) k_xprod<<<n, g.threads, g.smem, st>>>(d_insts, w, g.param, want_max);
                else k_zfwd<<<n, g.threads, g.smem, st>>>(d_insts, w, g.param);
            }
            if ((e = time_end(timer, g.stage, st)) != cudaSuccess) return e;
        }
        if (a_beside && p.col_a[ri].second) {
            const int si = (int)(ri % kRoundStreams);
            cudaStream_t rs = (nstreams > 1 && si > 0) ? p.side[si - 1] : st;
            cudaStream_t as = rs;
            if (a_stream) {
                if ((e = cudaEventRecord(p.ev_round[ri], rs)) != cudaSuccess) return e;
                if ((e = cudaStreamWaitEvent(p.side_a, p.ev_round[ri], 0)) != cudaSuccess) return e;
                as = p.side_a;
            }
            time_begin(timer, as);
            k_column_a<<<(unsigned)p.col_a[ri].second, kColumnBlock, p.sm_col, as>>>(
                d_insts, p.d_work + p.col_a[ri].first, kRK);
            if ((e = time_end(timer, 4, as)) != cudaSuccess) return e;
        }
    }
    if (a_stream) {
        if ((e = cudaEventRecord(p.ev_a, p.side_a)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(st, p.ev_a, 0)) != cudaSuccess) return e;
    }
    for (int k = 0; k < nstreams - 1; k++) {
        if ((e = cudaEventRecord(p.ev_join[k], p.side[k])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(st, p.ev_join[k], 0)) != cudaSuccess) return e;
    }
    if (kRK == 1) {
        time_begin(timer, st);
        k_dt<<<p.ninst, 256, 0, st>>>(d_insts, p.ninst);
        if ((e = time_end(timer, 3, st)) != cudaSuccess) return e;
    }
    if (before_column && (e = cudaStreamWaitEvent(st, before_column, cudaEventWaitExternal)) != cudaSuccess) return e;
    time_begin(timer, st);
    if (p.col_split) {
        if (!a_beside)
            k_column_a<<<(unsigned)p.n_col_full, kColumnBlock, p.sm_col, st>>>(d_insts, p.d_work + p.off_col_full, kRK);
        k_column_bcd<<<(unsigned)p.column.size(), kColumnBlock, p.sm_col, st>>>(d_insts, p.d_work + p.off_column, kRK);
    } else if (p.col_small)
        k_column_small<<<(unsigned)p.column.size(), 32 * kSmallWarps, p.sm_col, st>>>(d_insts, p.d_work + p.off_column,
                                                                                      kRK);
    else {
        const size_t nb = p.column.size(), per = (nb + p.col_waves - 1) / p.col_waves;
        for (size_t b0 = 0; b0 < nb; b0 += per)
            k_column<<<(unsigned)std::min(per, nb - b0), kColumnBlock, p.sm_col, st>>>(
                d_insts, p.d_work + p.off_column + b0, kRK);
    }
    if ((e = time_end(timer, 4, st)) != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace lh
