// Batched engine: many independent channel instances of uneven size advance
// together.  Every substep issues the same kernels as a single instance, but
// each launch's work table spans all live instances (instance, plane, block),
// so a batch of N instances costs one launch per kernel class and chunk
// round rather than N.  Each instance owns its device allocation; admission
// is checked against an HBM budget.  One RK3 step of the current membership
// is captured once in a CUDA graph and replayed until membership changes.
//
// Instances of at least kIsolateModes Fourier modes (Nx*Nz) keep the GPU
// busy on their own; sharing launches with others only shrinks their L2
// staging share and splits their rounds, so each gets its own launch plan
// (its chunk rounds sized as if alone), while the smaller instances share
// one plan.  The plans' launches follow one another on the batch stream
// inside the same captured step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "lh_engine.h"
#include "lh_gpu.h"
#include "lh_kernels.cuh"

using namespace lh;

struct lh_batch {
    size_t budget = 0, used = 0;
    std::vector<std::unique_ptr<DevInstance>> slots;  // nullptr = free slot
    std::vector<int> live;                            // slot ids in launch order
    std::vector<Plan> plans;                          // plan groups (see above)
    std::vector<int> plan_off;                        // first instance of each group in d_insts
    std::vector<bool> plan_cfl;                       // a CFL-mode instance in the group
    Inst *d_insts = nullptr;
    size_t d_insts_cap = 0;
    cudaStream_t st = nullptr;
    cudaStream_t st_up = nullptr;  // admissions upload here while steps run on st
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool dirty = true;
    bool any_cfl = false;
    std::string err;
    // device blocks of retired instances, reused by later admissions so a
    // request stream does not pay cudaMalloc/cudaFree (a device-wide
    // synchronisation) per request
    struct Block {
        void *ptr;
        size_t bytes;
    };
    std::vector<Block> pool;
    size_t pooled = 0;
};

static constexpr size_t kPoolBlocks = 16;
static constexpr long kIsolateModes = 128 * 128;  // LH_BATCH_ISOLATE overrides

static void pool_release(lh_batch *b, size_t keep_bytes)
{
    while (!b->pool.empty() && b->pooled > keep_bytes) {
        cudaFree(b->pool.front().ptr);
        b->pooled -= b->pool.front().bytes;
        b->pool.erase(b->pool.begin());
    }
}

static int bfail(lh_batch *b, int code, const std::string &m)
{
    if (b) b->err = m;
    return code;
}

static int bcuda(lh_batch *b, cudaError_t e, const char *where)
{
    return bfail(b, e == cudaErrorMemoryAllocation ? LH_ENOMEM : LH_ECUDA,
                 std::string(where) + ": " + cudaGetErrorString(e));
}

#define BCK(call, where)                                        \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return bcuda(b, e_, where);      \
    } while (0)

static void drop_graph(lh_batch *b)
{
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
}

extern "C" int lh_batch_create(size_t budget, lh_batch **out)
{
    if (!out) return LH_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return LH_ECUDA;
    lh_batch *b = new (std::nothrow) lh_batch();
    if (!b) return LH_ENOMEM;
    b->budget = budget;
    if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return LH_ECUDA;
    }
    if (cudaStreamCreateWithFlags(&b->st_up, cudaStreamNonBlocking) != cudaSuccess) {
        cudaStreamDestroy(b->st);
        delete b;
        return LH_ECUDA;
    }
    *out = b;
    return LH_OK;
}

extern "C" int lh_batch_destroy(lh_batch *b)
{
    if (!b) return LH_OK;
    if (b->st) cudaStreamSynchronize(b->st);
    drop_graph(b);
    for (Plan &p : b->plans) plan_free(p);
    if (b->d_insts) cudaFree(b->d_insts);
    for (auto &s : b->slots)
        if (s) instance_free(*s);
    pool_release(b, 0);
    if (b->st_up) cudaStreamDestroy(b->st_up);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
    return LH_OK;
}

extern "C" const char *lh_batch_last_error(const lh_batch *b) { return b ? b->err.c_str() : "null batch"; }

extern "C" size_t lh_instance_bytes(const lh_grid_desc *desc)
{
    if (!desc) return 0;
    HostSetup hs;
    if (!build_setup(*desc, hs).empty()) return 0;
    Tiles t = default_tiles(hs.Mx, hs.Mz, hs.nxh, hs.nyu);
    return instance_bytes(hs, t.chunk);
}

extern "C" int lh_batch_add(lh_batch *b, const lh_grid_desc *desc, const double *u1, const double *u2,
                            const double *u3, const double *p, int *slot)
{
    if (!b || !desc || !u1 || !u2 || !u3 || !slot) return bfail(b, LH_EINVAL, "bad arguments");
    auto d = std::unique_ptr<DevInstance>(new (std::nothrow) DevInstance());
    if (!d) return bfail(b, LH_ENOMEM, "host allocation");
    d->desc = *desc;
    std::string why = build_setup(*desc, d->hs);
    if (!why.empty()) return bfail(b, LH_EINVAL, why);
    Tiles t = default_tiles(d->hs.Mx, d->hs.Mz, d->hs.nxh, d->hs.nyu);
    const size_t need = instance_bytes(d->hs, t.chunk);
    if (b->budget && b->used + need > b->budget)
        return bfail(b, LH_ENOMEM, "HBM budget exhausted");
    // The new instance is allocated and uploaded on the admission stream
    // while steps already queued on the batch stream keep running: its memory
    // is fresh or a pooled block of an instance retired after a
    // synchronisation (lh_batch_remove), so no queued step touches it, and the
    // next lh_batch_step synchronises before it rebuilds the step graph.
    // smallest pooled block that fits; else make room under the budget and allocate
    int pick = -1;
    for (size_t k = 0; k < b->pool.size(); k++)
        if (b->pool[k].bytes >= need && (pick < 0 || b->pool[k].bytes < b->pool[pick].bytes)) pick = (int)k;
    void *reuse = nullptr;
    size_t reuse_bytes = 0;
    if (pick >= 0) {
        reuse = b->pool[pick].ptr;
        reuse_bytes = b->pool[pick].bytes;
        b->pooled -= reuse_bytes;
        b->pool.erase(b->pool.begin() + pick);
    } else if (b->budget) {
        pool_release(b, b->budget > b->used + need ? b->budget - b->used - need : 0);
    }
    cudaError_t e = instance_alloc(*d, t.chunk, b->st_up, reuse, reuse_bytes);
    if (e == cudaErrorMemoryAllocation && !reuse && !b->pool.empty()) {
        cudaGetLastError();
        pool_release(b, 0);
        e = instance_alloc(*d, t.chunk, b->st_up);
    }
    if (e == cudaSuccess) e = instance_upload(*d, u1, u2, u3, p, b->st_up);
    if (e != cudaSuccess) {
        instance_free(*d);
        return bcuda(b, e, "admit");
    }
    b->used += d->bytes;
    int id = -1;
    for (size_t k = 0; k < b->slots.size(); k++)
        if (!b->slots[k]) {
            id = (int)k;
            break;
        }
    if (id < 0) {
        id = (int)b->slots.size();
        b->slots.emplace_back();
    }
    b->slots[id] = std::move(d);
    b->dirty = true;
    *slot = id;
    return LH_OK;
}

extern "C" int lh_batch_remove(lh_batch *b, int slot)
{
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot]) return bfail(b, LH_EINVAL, "bad slot");
    BCK(cudaStreamSynchronize(b->st), "synchronize");
    b->used -= b->slots[slot]->bytes;
    DevInstance &d = *b->slots[slot];
    b->pool.push_back({d.block, d.alloc_bytes});
    b->pooled += d.alloc_bytes;
    d.block = nullptr;
    if (b->pool.size() > kPoolBlocks) {
        cudaFree(b->pool.front().ptr);
        b->pooled -= b->pool.front().bytes;
        b->pool.erase(b->pool.begin());
    }
    b->slots[slot].reset();
    b->dirty = true;
    return LH_OK;
}

static int rebuild(lh_batch *b)
{
    if (!b->dirty) return LH_OK;
    // queued steps still read the work tables and the instance table that
    // are rewritten below
    BCK(cudaStreamSynchronize(b->st), "synchronize");
    drop_graph(b);
    b->live.clear();
    b->any_cfl = false;
    const char *iso = getenv("LH_BATCH_ISOLATE");
    const long isolate = iso ? atol(iso) : kIsolateModes;
    // groups: the shared group of the smaller instances first, then one group
    // per isolated instance; d_insts holds the instances in that order
    std::vector<std::vector<int>> groups(1);
    for (size_t k = 0; k < b->slots.size(); k++)
        if (b->slots[k]) {
            const HostSetup &hs = b->slots[k]->hs;
            if ((long)hs.Nx * hs.Nz >= isolate) groups.push_back({(int)k});
            else groups[0].push_back((int)k);
        }
    if (groups[0].empty()) groups.erase(groups.begin());
    std::vector<Inst> hi;
    b->plan_off.clear();
    b->plan_cfl.clear();
    for (const auto &g : groups) {
        b->plan_off.push_back((int)hi.size());
        bool cfl = false;
        for (int k : g) {
            b->live.push_back(k);
            hi.push_back(b->slots[k]->inst);
            cfl |= b->slots[k]->desc.dt_mode == LH_DT_CFL;
        }
        b->plan_cfl.push_back(cfl);
        b->any_cfl |= cfl;
    }
    if (hi.empty()) {
        b->dirty = false;
        return LH_OK;
    }
    if (hi.size() > b->d_insts_cap) {
        if (b->d_insts) cudaFree(b->d_insts);
        b->d_insts = nullptr;
        BCK(cudaMalloc(&b->d_insts, hi.size() * sizeof(Inst)), "alloc instance table");
        b->d_insts_cap = hi.size();
    }
    BCK(cudaMemcpy(b->d_insts, hi.data(), hi.size() * sizeof(Inst), cudaMemcpyHostToDevice), "instance table");
    // plans (their work buffers, streams and events) are kept and rebuilt in place
    while (b->plans.size() > groups.size()) {
        plan_free(b->plans.back());
        b->plans.pop_back();
    }
    b->plans.resize(groups.size());
    for (size_t g = 0; g < groups.size(); g++) {
        std::vector<const DevInstance *> v;
        for (int k : groups[g]) v.push_back(b->slots[k].get());
        BCK(plan_build(b->plans[g], v), "plan");
    }
    BCK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal), "capture");
    cudaError_t el = cudaSuccess;
    for (int k = 1; k <= 3 && el == cudaSuccess; k++)
        for (size_t g = 0; g < b->plans.size() && el == cudaSuccess; g++)
            el = launch_substep(b->plans[g], b->d_insts + b->plan_off[g], k, b->plan_cfl[g], b->st);
    cudaGraph_t gr = nullptr;
    cudaError_t ee = cudaStreamEndCapture(b->st, &gr);
    if (el != cudaSuccess) return bcuda(b, el, "capture launch");
    if (ee != cudaSuccess) return bcuda(b, ee, "capture end");
    b->graph = gr;
    BCK(cudaGraphInstantiate(&b->gexec, gr, 0), "instantiate");
    b->dirty = false;
    return LH_OK;
}

extern "C" int lh_batch_step(lh_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return bfail(b, LH_EINVAL, "bad arguments");
    int rc = rebuild(b);
    if (rc) return rc;
    if (b->live.empty()) return LH_OK;
    for (int s = 0; s < nsteps; s++) BCK(cudaGraphLaunch(b->gexec, b->st), "graph launch");
    return LH_OK;
}

extern "C" int lh_batch_download(lh_batch *b, int slot, double *u1, double *u2, double *u3, double *p)
{
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot]) return bfail(b, LH_EINVAL, "bad slot");
    BCK(instance_download(*b->slots[slot], u1, u2, u3, p, b->st), "download");
    return LH_OK;
}

extern "C" int lh_batch_scalars(lh_batch *b, int slot, double *t, double *dt, int *iter)
{
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot]) return bfail(b, LH_EINVAL, "bad slot");
    double sc[SC_COUNT];
    int err = 0;
    const Inst &I = b->slots[slot]->inst;
    BCK(cudaMemcpyAsync(sc, I.sc, sizeof(sc), cudaMemcpyDeviceToHost, b->st), "scalars");
    BCK(cudaMemcpyAsync(&err, I.err, sizeof(int), cudaMemcpyDeviceToHost, b->st), "scalars");
    BCK(cudaStreamSynchronize(b->st), "scalars");
    if (t) *t = sc[SC_T];
    if (dt) *dt = sc[SC_DT];
    if (iter) *iter = (int)sc[SC_ITER];
    if (err & ERR_NONFINITE) return bfail(b, LH_EDEVICE, "instance state became non-finite");
    return LH_OK;
}

extern "C" int lh_batch_set_scalars(lh_batch *b, int slot, double t, int iter, double mpgx)
{
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot] || iter < 0)
        return bfail(b, LH_EINVAL, "bad arguments");
    const Inst &I = b->slots[slot]->inst;
    const double v[3] = {t, mpgx, (double)iter};
    // queued steps may still advance this instance: ordered after them
    BCK(cudaMemcpyAsync(I.sc + SC_T, &v[0], sizeof(double), cudaMemcpyHostToDevice, b->st), "set scalars");
    BCK(cudaMemcpyAsync(I.sc + SC_MPGX, &v[1], sizeof(double), cudaMemcpyHostToDevice, b->st), "set scalars");
    BCK(cudaMemcpyAsync(I.sc + SC_ITER, &v[2], sizeof(double), cudaMemcpyHostToDevice, b->st), "set scalars");
    BCK(cudaStreamSynchronize(b->st), "set scalars");
    return LH_OK;
}

extern "C" int lh_batch_count(const lh_batch *b)
{
    if (!b) return 0;
    int n = 0;
    for (auto &s : b->slots) n += s ? 1 : 0;
    return n;
}

extern "C" int lh_batch_synchronize(lh_batch *b)
{
    if (!b) return LH_EINVAL;
    BCK(cudaStreamSynchronize(b->st), "synchronize");
    return LH_OK;
}
