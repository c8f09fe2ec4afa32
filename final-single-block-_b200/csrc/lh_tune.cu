// Autotuner of the launch shapes of a size class.
//
// The plane pipeline's tile bounds (x modes per z-inverse CTA, z rows per
// x-products CTA, x modes per z-forward CTA), the plane-staging budget and
// the number of column-pass launches are chosen per (Mz, Mx, nyu) by timing
// complete RK3 steps of a scratch instance of that size with CUDA events.
// The search is coordinate descent from the built-in defaults: each
// parameter in turn takes the best of a few candidates with the others held,
// a candidate replacing the incumbent only when it is 2 % faster.
// Nothing it varies changes any arithmetic -- every transform vector and
// every column is computed by the same code whatever the tiling -- so a
// tuned plan gives bit-identical states.
//
// Results live in a process-wide table (plan_build consults it for every
// size class, single instances and batches alike) and in a text cache file,
// one line per entry keyed by the GPU's name and the sizes:
//   <gpu name>|<Mz>|<Mx>|<nyu> <cbz> <rbx> <cbf> <staging_mb> <col_waves> <ms per step>
// The file is LH_TUNE_CACHE, else lh_tune_cache.txt beside the library.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "lh_engine.h"
#include "lh_gpu.h"
#include "lh_kernels.cuh"

using namespace lh;

#include "lh_ctx_internal.h"

namespace lh {
namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, TuneParams> g_tune;
}  // namespace

bool tune_lookup(int Mz, int Mx, int nyu, TuneParams &out)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(std::make_tuple(Mz, Mx, nyu));
    if (it == g_tune.end()) return false;
    out = it->second;
    return true;
}

void tune_store(int Mz, int Mx, int nyu, const TuneParams &t)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[std::make_tuple(Mz, Mx, nyu)] = t;
}
}  // namespace lh

namespace {

std::string cache_path()
{
    const char *ev = getenv("LH_TUNE_CACHE");
    if (ev && *ev) return ev;
    Dl_info info;
    if (dladdr((const void *)&cache_path, &info) && info.dli_fname) {
        std::string so = info.dli_fname;
        const size_t k = so.rfind('/');
        return (k == std::string::npos ? std::string(".") : so.substr(0, k)) + "/lh_tune_cache.txt";
    }
    return "lh_tune_cache.txt";
}

std::string gpu_name()
{
    int dev = 0;
    cudaDeviceProp pr;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&pr, dev) != cudaSuccess) return "unknown";
    std::string n = pr.name;
    std::replace(n.begin(), n.end(), '|', '/');
    std::replace(n.begin(), n.end(), ' ', '_');
    return n;
}

std::string cache_key(const HostSetup &s)
{
    char b[128];
    snprintf(b, sizeof b, "|%d|%d|%d", s.Mz, s.Mx, s.nyu);
    return gpu_name() + b;
}

bool cache_read(const std::string &key, TuneParams &t)
{
    FILE *f = fopen(cache_path().c_str(), "r");
    if (!f) return false;
    char line[512], k[256];
    bool found = false;
    while (fgets(line, sizeof line, f)) {
        TuneParams q;
        double ms = 0;
        if (sscanf(line, "%255s %d %d %d %d %d %lf", k, &q.cbz, &q.rbx, &q.cbf, &q.staging_mb, &q.col_waves, &ms) == 7 &&
            key == k) {
            t = q;  // the last entry of a key wins
            found = true;
        }
    }
    fclose(f);
    return found;
}

void cache_append(const std::string &key, const TuneParams &t, double ms)
{
    FILE *f = fopen(cache_path().c_str(), "a");
    if (!f) return;  // an unwritable cache only costs a re-measurement
    fprintf(f, "%s %d %d %d %d %d %.6f\n", key.c_str(), t.cbz, t.rbx, t.cbf, t.staging_mb, t.col_waves, ms);
    fclose(f);
}

// ms per RK3 step of a plan on the scratch instance: one warm step, then
// enough steps for at least ~8 ms of device time.
cudaError_t time_plan(const Plan &p, const Inst *d_inst, bool cfl, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1,
                      double &ms)
{
    cudaError_t e = cudaSuccess;
    for (int k = 1; k <= 3 && e == cudaSuccess; k++) e = launch_substep(p, d_inst, k, cfl, st);
    if (e != cudaSuccess) return e;
    int reps = 2;
    for (;;) {
        if ((e = cudaEventRecord(e0, st)) != cudaSuccess) return e;
        for (int r = 0; r < reps && e == cudaSuccess; r++)
            for (int k = 1; k <= 3 && e == cudaSuccess; k++) e = launch_substep(p, d_inst, k, cfl, st);
        if (e != cudaSuccess) return e;
        if ((e = cudaEventRecord(e1, st)) != cudaSuccess) return e;
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) return e;
        float f = 0.f;
        cudaEventElapsedTime(&f, e0, e1);
        if (f >= 8.0f || reps >= 256) {
            ms = f / reps;
            return cudaSuccess;
        }
        reps *= 2;
    }
}

}  // namespace

extern "C" int lh_autotune(lh_ctx *c, int force, int *params)
{
    if (!c) return LH_EINVAL;
    const HostSetup &s = c->dev.hs;
    const std::string key = cache_key(s);
    TuneParams best = default_params(s);
    int source = 0;
    if (!force && cache_read(key, best)) {
        source = 2;
    } else {
        // scratch instance of the same size: the caller's state is never touched
        DevInstance scr;
        scr.desc = c->dev.desc;
        scr.hs = s;
        Inst *d_scr = nullptr;
        Plan plan;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        const bool cfl = c->dev.desc.dt_mode == LH_DT_CFL;
        cudaError_t e = instance_alloc(scr, c->dev.inst.chunk, c->st);
        if (e == cudaSuccess && c->have_state) {
            // the current state, so the CFL time step is the run's
            const size_t nc = s.nc;
            e = cudaMemcpyAsync(scr.inst.U1, c->dev.inst.U1, (s.nyu + 2) * nc * sizeof(double2), cudaMemcpyDeviceToDevice, c->st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(scr.inst.U2, c->dev.inst.U2, (s.nyv + 2) * nc * sizeof(double2), cudaMemcpyDeviceToDevice, c->st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(scr.inst.U3, c->dev.inst.U3, (s.nyu + 2) * nc * sizeof(double2), cudaMemcpyDeviceToDevice, c->st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(scr.inst.sc, c->dev.inst.sc, SC_COUNT * sizeof(double), cudaMemcpyDeviceToDevice, c->st);
        }
        if (e == cudaSuccess) e = cudaMalloc(&d_scr, sizeof(Inst));
        if (e == cudaSuccess) e = cudaMemcpy(d_scr, &scr.inst, sizeof(Inst), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaEventCreate(&e0);
        if (e == cudaSuccess) e = cudaEventCreate(&e1);
        double best_ms = 0.0;
        auto trial = [&](const TuneParams &t, double &ms) {
            cudaError_t r = plan_build(plan, {&scr}, false, &t);
            if (r == cudaSuccess) r = time_plan(plan, d_scr, cfl, c->st, e0, e1, ms);
            return r;
        };
        if (e == cudaSuccess) e = trial(best, best_ms);
        // candidate values per parameter, around the defaults
        const bool fast = best.cbz > 0;
        const TuneParams d0 = best;
        std::vector<std::pair<int TuneParams::*, std::vector<int>>> axes;
        if (fast) {
            axes.push_back({&TuneParams::cbz, {std::max(1, d0.cbz / 2), d0.cbz * 2}});
            axes.push_back({&TuneParams::rbx, {std::max(1, d0.rbx / 2), d0.rbx * 2}});
            axes.push_back({&TuneParams::cbf, {std::max(1, d0.cbf - 2), std::max(1, d0.cbf - 1), d0.cbf + 1}});
        }
        axes.push_back({&TuneParams::staging_mb, {48, 64}});
        axes.push_back({&TuneParams::col_waves, {2, 3, 4}});
        for (auto &ax : axes) {
            for (int v : ax.second) {
                if (e != cudaSuccess) break;
                TuneParams t = best;
                if (t.*(ax.first) == v) continue;
                t.*(ax.first) = v;
                double ms = 0.0;
                e = trial(t, ms);
                // a candidate must beat the incumbent by 2 %: run-to-run noise of
                // a step is about 1-2 %, and an unchanged default is the safer pick
                if (e == cudaSuccess && ms < 0.98 * best_ms) {
                    best_ms = ms;
                    best = t;
                }
            }
        }
        cudaStreamSynchronize(c->st);
        plan_free(plan);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (d_scr) cudaFree(d_scr);
        instance_free(scr);
        if (e != cudaSuccess) {
            c->err = std::string("autotune: ") + cudaGetErrorString(e);
            return e == cudaErrorMemoryAllocation ? LH_ENOMEM : LH_ECUDA;
        }
        cache_append(key, best, best_ms);
        source = 1;
    }
    tune_store(s.Mz, s.Mx, s.nyu, best);
    // the context's own plan picks the tuned parameters up; its step graph is
    // captured again on the next lh_step
    ctx_drop_graphs(c);
    const char *gen = getenv("LH_GENERIC_FFT");
    cudaError_t e = plan_build(c->plan, {&c->dev}, gen && gen[0] == '1');
    if (e != cudaSuccess) {
        c->err = std::string("autotune plan: ") + cudaGetErrorString(e);
        return LH_ECUDA;
    }
    if (params) {
        params[0] = best.cbz;
        params[1] = best.rbx;
        params[2] = best.cbf;
        params[3] = best.staging_mb;
        params[4] = best.col_waves;
        params[5] = source;
    }
    return LH_OK;
}
