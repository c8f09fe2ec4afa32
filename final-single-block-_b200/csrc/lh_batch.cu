// Batched engine: many independent channel instances of uneven size advance
// together.  Every substep issues the same kernels as a single instance, but
// each launch's work table spans all instances of a launch group (instance,
// plane, block), so a group of N instances costs one launch per kernel
// class and chunk round rather than N.  Each instance owns its device
// allocation; admission is checked against an HBM budget.
//
// Instances of at least kIsolateModes Fourier modes (Nx*Nz) keep the GPU
// busy on their own; sharing launches with others only shrinks their L2
// staging share and splits their rounds, so each forms a launch group of its
// own (its chunk rounds sized as if alone), while the smaller instances
// share one group.  Every group keeps its own plan, instance table and CUDA
// graph of one RK3 step; a batch step replays the groups' graphs one after
// another on the batch stream (LH_BATCH_STREAMS = 2..4 replays them on that
// many forked streams at once instead: measured slower on B200, the groups'
// plane staging then competes for L2).  When membership changes, only the groups
// whose members changed are planned and captured again -- an admission or a
// retirement of a large instance leaves every other group's graph as it was.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
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
    std::vector<uint64_t> serial;                     // admission number of each slot's instance
    uint64_t next_serial = 1;
    // one launch group: its members (admission numbers, launch order), plan,
    // device instance table and captured RK3 step
    struct Group {
        std::vector<uint64_t> key;
        Plan plan;
        Inst *d_inst = nullptr;
        bool cfl = false;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t gexec = nullptr;
    };
    std::vector<std::unique_ptr<Group>> groups;
    cudaStream_t st = nullptr;
    cudaStream_t st_up = nullptr;  // admissions upload here while steps run on st
    // streams for replaying launch groups concurrently (LH_BATCH_STREAMS),
    // forked from st and joined back at every step (disjoint instances)
    static constexpr int kGroupStreams = 4;
    cudaStream_t gst[kGroupStreams] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kGroupStreams] = {};
    bool dirty = true;
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

static void free_group(lh_batch::Group &g)
{
    if (g.gexec) cudaGraphExecDestroy(g.gexec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g.gexec = nullptr;
    g.graph = nullptr;
    plan_free(g.plan);
    if (g.d_inst) cudaFree(g.d_inst);
    g.d_inst = nullptr;
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
    bool ok = cudaStreamCreateWithFlags(&b->st_up, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess;
    for (int k = 0; k < lh_batch::kGroupStreams && ok; k++)
        ok = cudaStreamCreateWithFlags(&b->gst[k], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&b->ev_join[k], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        lh_batch_destroy(b);
        return LH_ECUDA;
    }
    *out = b;
    return LH_OK;
}

extern "C" int lh_batch_destroy(lh_batch *b)
{
    if (!b) return LH_OK;
    if (b->st) cudaStreamSynchronize(b->st);
    for (auto &g : b->groups) free_group(*g);
    b->groups.clear();
    for (auto &s : b->slots)
        if (s) instance_free(*s);
    pool_release(b, 0);
    for (int k = 0; k < lh_batch::kGroupStreams; k++) {
        if (b->gst[k]) cudaStreamSynchronize(b->gst[k]);
        if (b->gst[k]) cudaStreamDestroy(b->gst[k]);
        if (b->ev_join[k]) cudaEventDestroy(b->ev_join[k]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
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
    if (b->serial.size() < b->slots.size()) b->serial.resize(b->slots.size(), 0);
    b->serial[id] = b->next_serial++;
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
    const char *iso = getenv("LH_BATCH_ISOLATE");
    const long isolate = iso ? atol(iso) : kIsolateModes;
    // groups: the shared group of the smaller instances first, then one group
    // per isolated instance
    std::vector<std::vector<int>> members(1);
    for (size_t k = 0; k < b->slots.size(); k++)
        if (b->slots[k]) {
            const HostSetup &hs = b->slots[k]->hs;
            if ((long)hs.Nx * hs.Nz >= isolate) members.push_back({(int)k});
            else members[0].push_back((int)k);
        }
    if (members[0].empty()) members.erase(members.begin());
    std::vector<std::unique_ptr<lh_batch::Group>> next;
    for (const auto &m : members) {
        std::vector<uint64_t> key;
        for (int k : m) key.push_back(b->serial[k]);
        // a group with the same instances keeps its plan and graph
        auto it = std::find_if(b->groups.begin(), b->groups.end(),
                               [&](const std::unique_ptr<lh_batch::Group> &g) { return g && g->key == key; });
        if (it != b->groups.end()) {
            next.push_back(std::move(*it));
            continue;
        }
        auto g = std::unique_ptr<lh_batch::Group>(new (std::nothrow) lh_batch::Group());
        if (!g) return bfail(b, LH_ENOMEM, "host allocation");
        g->key = key;
        std::vector<Inst> hi;
        std::vector<const DevInstance *> v;
        for (int k : m) {
            hi.push_back(b->slots[k]->inst);
            v.push_back(b->slots[k].get());
            g->cfl |= b->slots[k]->desc.dt_mode == LH_DT_CFL;
        }
        cudaError_t e = cudaMalloc(&g->d_inst, hi.size() * sizeof(Inst));
        if (e == cudaSuccess) e = cudaMemcpy(g->d_inst, hi.data(), hi.size() * sizeof(Inst), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = plan_build(g->plan, v);
        // captured on the admission stream: the batch stream may still be
        // running queued steps of the other groups
        if (e == cudaSuccess) e = cudaStreamBeginCapture(b->st_up, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t el = cudaSuccess;
            for (int kk = 1; kk <= 3 && el == cudaSuccess; kk++)
                el = launch_substep(g->plan, g->d_inst, kk, g->cfl, b->st_up);
            cudaError_t ee = cudaStreamEndCapture(b->st_up, &g->graph);
            e = el != cudaSuccess ? el : ee;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&g->gexec, g->graph, 0);
        if (e != cudaSuccess) {
            free_group(*g);
            return bcuda(b, e, "group plan");
        }
        next.push_back(std::move(g));
    }
    // groups left without a match are freed; queued steps may still read
    // their plans and instance tables, so only then wait for them (an
    // admission that only adds groups keeps the device busy meanwhile)
    bool stale = false;
    for (auto &g : b->groups) stale |= (bool)g;
    if (stale) BCK(cudaStreamSynchronize(b->st), "synchronize");
    for (auto &g : b->groups)
        if (g) free_group(*g);
    b->groups = std::move(next);
    b->dirty = false;
    return LH_OK;
}

extern "C" int lh_batch_step(lh_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return bfail(b, LH_EINVAL, "bad arguments");
    int rc = rebuild(b);
    if (rc) return rc;
    const int ng = (int)b->groups.size();
    if (ng == 1) {
        for (int s = 0; s < nsteps; s++) BCK(cudaGraphLaunch(b->groups[0]->gexec, b->st), "graph launch");
        return LH_OK;
    }
    // group g on stream g % kGroupStreams, each stream's groups in order;
    // every step forks from and joins back to the batch stream, so the
    // batch stream orders steps, downloads and rebuilds as before
    const char *gs = getenv("LH_BATCH_STREAMS");
    const int ns = std::min(ng, std::max(1, std::min(gs ? atoi(gs) : 1, (int)lh_batch::kGroupStreams)));
    if (ns == 1) {
        for (int s = 0; s < nsteps; s++)
            for (auto &g : b->groups) BCK(cudaGraphLaunch(g->gexec, b->st), "graph launch");
        return LH_OK;
    }
    for (int s = 0; s < nsteps; s++) {
        BCK(cudaEventRecord(b->ev_fork, b->st), "fork");
        for (int k = 0; k < ns; k++) BCK(cudaStreamWaitEvent(b->gst[k], b->ev_fork, 0), "fork");
        for (int g = 0; g < ng; g++) BCK(cudaGraphLaunch(b->groups[g]->gexec, b->gst[g % ns]), "graph launch");
        for (int k = 0; k < ns; k++) {
            BCK(cudaEventRecord(b->ev_join[k], b->gst[k]), "join");
            BCK(cudaStreamWaitEvent(b->st, b->ev_join[k], 0), "join");
        }
    }
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
