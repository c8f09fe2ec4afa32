// Engine internals shared by the single-instance context and the batch:
// device memory of one instance and the launch plan of a substep.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "lh_core.cuh"
#include "lh_setup.h"

namespace lh {

// Launch shapes of the plane pipeline and the column pass.
struct Tiles {
    int bc_zinv = 8;   // x modes per z-inverse CTA
    int br_x = 2;      // z rows per x-transform CTA
    int bc_zfwd = 1;   // x modes per z-forward CTA
    int threads = 256; // threads per plane CTA
    int chunk = 32;    // planes per staging chunk
};

Tiles default_tiles(int Mx, int Mz, int nxh, int nyu);
size_t smem_zinv(const Tiles &t, int Mz);
size_t smem_x(const Tiles &t, int Mx);
size_t smem_zfwd(const Tiles &t, int Mz);

// Device memory of one instance.  All buffers come from one allocation.
struct DevInstance {
    HostSetup hs;
    lh_grid_desc desc{};
    Inst inst{};           // host copy with device pointers
    void *block = nullptr; // the allocation
    size_t bytes = 0;      // bytes the instance uses
    size_t alloc_bytes = 0;  // size of the allocation (>= bytes when a pooled block is reused)
    double2 *stage = nullptr;  // layout-transform staging (one field)
    size_t stage_elems = 0;
};

// Plane fields of staging an instance allocates for `chunk` planes.
size_t staging_units(int chunk);
// Bytes one instance needs for a staging chunk of `chunk` planes.
size_t instance_bytes(const HostSetup &hs, int chunk);
// Allocate and fill the device arrays of an instance (synchronous).
// With `reuse` (a device block of reuse_bytes from an earlier instance) the
// instance is carved from it when it is large enough, instead of cudaMalloc.
cudaError_t instance_alloc(DevInstance &d, int chunk, cudaStream_t st, void *reuse = nullptr, size_t reuse_bytes = 0);
void instance_free(DevInstance &d);
// Upload / download the four state fields in the reference column layout.
cudaError_t instance_upload(DevInstance &d, const double *u1, const double *u2, const double *u3, const double *p,
                            cudaStream_t st);
// The same upload with p last: everything the plane pass and the column pass
// read except p is enqueued on st, then ev_u is recorded on st, then p is
// enqueued; nothing waits on the host.
cudaError_t instance_upload_p_last(DevInstance &d, const double *u1, const double *u2, const double *u3,
                                   const double *p, cudaStream_t st, cudaEvent_t ev_u);
cudaError_t instance_download(DevInstance &d, double *u1, double *u2, double *u3, double *p, cudaStream_t st);
cudaError_t download_field(const DevInstance &d, const double2 *src, int len, double *dst, cudaStream_t st);

// Device resources of the diagnostics (lh_diag.cu): the pressure snapshot the
// stats read, and the transform scratch of omega_x, allocated on first use.
struct StatsScratch {
    double *planes = nullptr;  // omega_x transform scratch
    size_t bytes = 0;
    int chunk_n = 0;           // omega_x planes per pass (Nspec-sized)
    Inst *d_inst_n = nullptr;  // instance record with the Nspec transform sizes and tables
    double2 *tw_n = nullptr;   // its twiddles: z (Nz), then x (Nx)
    double2 *pp = nullptr;     // pressure snapshot (rows 1..nyu), from the first snapshot on
};
cudaError_t stats_prepare(const DevInstance &d, StatsScratch &s);
void stats_release(StatsScratch &s);
size_t stats_doubles(int nyu);
// Adds the current state's stats into acc[13][nyu+2]; pp (the pressure
// snapshot) may be null.
cudaError_t launch_stats_accumulate(const Inst *d_inst, const HostSetup &hs, const double2 *pp, double *acc,
                                    cudaStream_t st);
// omega_x of the current state into host out[(nyu+2)][Nz][Nx+2] (synchronous).
cudaError_t omega_x_planes(const Inst *d_inst, const HostSetup &hs, const StatsScratch &s, double *out,
                           cudaStream_t st);

// One kernel launch of the plane pipeline: all work items of one stage for
// the instances of one size class in one chunk round.
struct Group {
    int stage = 0;        // 0 z inverse, 1 x products, 2 z forward
    bool fast = false;    // compile-time-sized kernels
    int Mz = 0, Mx = 0;
    size_t off = 0, count = 0;
    int threads = 256;
    size_t smem = 0;
    int param = 1;        // cb (z stages) or rb (x stage)
    unsigned grid = 0;    // CTAs launched, one per work item
};

// Work tables for a set of instances sharing launches.
struct Plan {
    std::vector<std::vector<Group>> rounds;  // launch order within a round
    std::vector<Work> column;
    Work *d_work = nullptr;  // all tables back to back
    size_t work_cap = 0;     // Work entries d_work holds (reused across rebuilds)
    size_t off_column = 0;
    size_t sm_col = 0;
    bool col_small = false;  // column pass by k_column_small (one CTA per column)
    int col_waves = 1;       // column-pass launches the column blocks are split over
    // Split column pass (LH_COLUMN_SPLIT): its forward sweeps run in row
    // chunks, one per plane round, on a stream of their own as soon as the
    // round's z-forward is done, while later rounds still run; phases B-D
    // follow in one launch.  Per round (offset, count) of the k_column_a work
    // items, and a one-chunk list for substeps whose dt is only known after
    // the plane pass (CFL mode, kRK = 1).
    bool col_split = false;
    std::vector<std::pair<size_t, size_t>> col_a;
    size_t off_col_full = 0, n_col_full = 0;
    cudaStream_t side_a = nullptr;
    std::vector<cudaEvent_t> ev_round;
    cudaEvent_t ev_a = nullptr;
    int ninst = 0;
    bool force_generic = false;
    cudaStream_t side[kRoundStreams - 1] = {};  // rounds r % kRoundStreams != 0
    cudaEvent_t ev_fork = nullptr, ev_join[kRoundStreams - 1] = {};
};

// Optional per-launch timing (kernel classes 0 z inverse, 1 x products,
// 2 z forward, 3 dt, 4 column).
struct LaunchTimer {
    cudaEvent_t ev[2];
    double ms[5] = {0, 0, 0, 0, 0};
    int n[5] = {0, 0, 0, 0, 0};
};

// Launch-shape parameters of a size class that the autotuner (lh_tune.cu)
// chooses: x modes per z-inverse CTA, z rows per x-products CTA, x modes per
// z-forward CTA (upper bounds, clamped to each kernel's launch bounds and
// shared memory), the plane-staging budget in MB and the number of
// column-pass launches.  0 = the built-in default (or its environment
// override).  None of them changes any arithmetic.
struct TuneParams {
    int cbz = 0, rbx = 0, cbf = 0, staging_mb = 0, col_waves = 0;
};
// The built-in defaults of a size, as numbers.
TuneParams default_params(const HostSetup &s);
// Process-wide table of tuned parameters keyed by (Mz, Mx, nyu); plan_build
// consults it for every size class it has no environment override for.
bool tune_lookup(int Mz, int Mx, int nyu, TuneParams &out);
void tune_store(int Mz, int Mx, int nyu, const TuneParams &t);

// `force` (the autotuner's candidate) takes precedence over the table and
// the environment.
cudaError_t plan_build(Plan &p, const std::vector<const DevInstance *> &insts, bool force_generic = false,
                       const TuneParams *force = nullptr);
void plan_free(Plan &p);
// Enqueue one substep of every instance of the plan.  With before_column the
// column pass first waits for that event (an external event node when
// captured): the plane pass does not read p, so p may still be uploading
// (with a split column pass, whose chunks read p, the substep waits first).
cudaError_t launch_substep(const Plan &p, const Inst *d_insts, int kRK, bool cfl_any, cudaStream_t st,
                           LaunchTimer *timer = nullptr, cudaEvent_t before_column = nullptr);

}  // namespace lh
