// Kernel declarations (definitions in lh_plane.cu and lh_column.cu).
#pragma once

#include "lh_core.cuh"

namespace lh {

constexpr int kColumnThreads = 32;       // columns per column-pass CTA (one lane each)
constexpr int kColumnBlock = 3 * kColumnThreads;  // three warps: the u1, u3 and u2 chains
size_t column_smem_bytes(int max_nyu);  // ring + staged y metrics
// column pass for small mode counts: one CTA of kSmallWarps warps (the u1,
// u3, u2 chains) per column, rows spread over the lanes
constexpr int kSmallWarps = 3;
// rows per lane whose global loads the right-hand-side phase issues together
constexpr int kSmallBatch = 4;
size_t column_small_smem_bytes(int max_nyu);

__global__ void k_zinv(const Inst *__restrict__ insts, const Work *__restrict__ work, int bc);
__global__ void k_xprod(const Inst *__restrict__ insts, const Work *__restrict__ work, int br, int want_max);
__global__ void k_zfwd(const Inst *__restrict__ insts, const Work *__restrict__ work, int bc);
__global__ void k_plane_z_inv(const Inst *__restrict__ insts, double *planes, int bc, int zero_row);
__global__ void k_plane_z_fwd(const Inst *__restrict__ insts, double *planes, int bc);
__global__ void k_plane_x_inv(const Inst *__restrict__ insts, double *planes, int br);
__global__ void k_plane_x_fwd(const Inst *__restrict__ insts, double *planes, int br);
__global__ void k_plane_zero_row(const Inst *__restrict__ insts, double *planes);

__global__ void k_column(const Inst *__restrict__ insts, const Work *__restrict__ work, int kRK);
// the column pass split: forward sweeps in row chunks, then phases B-D
__global__ void k_column_a(const Inst *__restrict__ insts, const Work *__restrict__ work, int kRK);
__global__ void k_column_bcd(const Inst *__restrict__ insts, const Work *__restrict__ work, int kRK);
__global__ void k_dt(const Inst *__restrict__ insts, int ninst);
__global__ void k_col_to_plane(const double2 *__restrict__ src, double2 *__restrict__ dst, int len, int nc);
__global__ void k_plane_to_col(const double2 *__restrict__ src, double2 *__restrict__ dst, int len, int nc);
__global__ void k_column_small(const Inst *__restrict__ insts, const Work *__restrict__ work, int kRK);
__global__ void k_lusolu(const Inst *__restrict__ insts, int grid, int kRK, double dt, const double2 *rhs,
                         double2 *u, double *fac);
__global__ void k_lusolp(const Inst *__restrict__ insts, double2 *x);
__global__ void k_divmax(const Inst *__restrict__ insts, double *out);

// on-device spectra of flagged steps (lh_diag.cu): accumulator doubles and launch;
// the plane stats are declared in lh_engine.h
size_t spectra_doubles(int nyu, int nyv, int nc);
void launch_spectra_accumulate(const Inst *d_inst, double *sp, int nyu, int nc, cudaStream_t st);

// raise (never lower) a kernel's dynamic shared-memory limit (lh_engine.cu)
cudaError_t raise_smem_limit(const void *func, size_t bytes);

// compile-time-sized fast path (lh_plane_fast.cu)
bool fast_size(int n);
int fast_threads(int n, int vectors);
int fast_max_threads(int stage);  // launch-bounds block size of a fast stage
int fast_vector_threads(int n);   // threads per vector of a fast length
size_t zinv_smem(int n, int cb);  // shared memory of a z-inverse CTA of cb vectors
bool xprod_warp(int n);            // the x stage of length n runs a warp-local kernel
bool xprod_multi(int n);           // the x stage of length n runs the multi-plane kernel
int xprod_max_threads(int n);      // launch-bounds block size of that x-stage kernel
int xprod_threads(int n, int rb);  // threads of an x-stage CTA of rb z rows
size_t xprod_smem(int n, int rb);  // shared memory of an x-stage CTA of rb z rows
int zfwd_threads(int n, int cb);   // threads of a z-forward CTA of cb x modes
size_t zfwd_smem(int n, int cb);   // shared memory of a z-forward CTA of cb x modes
cudaError_t fast_set_attributes(int Mz, int Mx, size_t smz, size_t smx, size_t smf);
void fast_launch_zinv(int Mz, unsigned grid, int threads, size_t smem, cudaStream_t st, const Inst *insts,
                      const Work *work, int count, int cb);
void fast_launch_xprod(int Mx, unsigned grid, int threads, size_t smem, cudaStream_t st, const Inst *insts,
                       const Work *work, int count, int rb, int want_max);
void fast_launch_zfwd(int Mz, unsigned grid, int threads, size_t smem, cudaStream_t st, const Inst *insts,
                      const Work *work, int count, int cb);

}  // namespace lh
