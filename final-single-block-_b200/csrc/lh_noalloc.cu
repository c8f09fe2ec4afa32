// Allocation-free variant of the LUsolU solve (tridLU_3D.f90:38-94).
//
// lh_lusolu() allocates device buffers on every call, which some callers
// cannot do: a solver loop being captured into a CUDA graph (cudaMalloc is
// not capturable), a real-time or serving loop that must not trigger the
// implicit device synchronisation of cudaMalloc/cudaFree, or a host program
// whose device memory is owned by another allocator.  lh_lusolu_noalloc()
// takes the right-hand side and the solution as device arrays the caller
// already owns and keeps its only scratch -- one scaled upper diagonal per
// row and column -- in the file-scope array below.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "lh_ctx_internal.h"
#include "lh_gpu.h"
#include "lh_kernels.cuh"

namespace {

// 2^21 doubles = 16 MiB, allocated when the library's device code is loaded
// and held on every GPU that loads it until the process exits.  It bounds
// rows x columns of one solve (e.g. 154 x 8320 for 128x128 modes, ny=153).
constexpr size_t kScratchDoubles = size_t(1) << 21;
__device__ __align__(256) double g_lusolu_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device, looked up once
// per device.  In host code the array's name is only a host-side stand-in,
// so kernels must receive the address returned here.
cudaError_t scratch_on_current_device(double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        double *p = nullptr;
        e = cudaGetSymbolAddress((void **)&p, g_lusolu_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" int lh_lusolu_noalloc(lh_ctx *c, int grid, int kRK, double dt, const double *rhs_dev, double *u_dev)
{
    if (!c) return LH_EINVAL;
    if (!rhs_dev || !u_dev || (grid != 1 && grid != 2) || kRK < 1 || kRK > 3) {
        c->err = "lh_lusolu_noalloc: bad arguments";
        return LH_EINVAL;
    }
    const lh::HostSetup &s = c->dev.hs;
    const size_t len = grid == 2 ? (size_t)s.nyu + 2 : (size_t)s.nyv + 2;
    const size_t need = len * (size_t)s.nc;
    if (need > kScratchDoubles) {
        c->err = "lh_lusolu_noalloc: " + std::to_string(len) + " rows x " + std::to_string(s.nc) +
                 " columns exceed the fixed scratch of " + std::to_string(kScratchDoubles) + " entries";
        return LH_EINVAL;
    }
    // the scratch address is per device: the context's device must be current
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess && dev != c->device) {
        c->err = "lh_lusolu_noalloc: device " + std::to_string(dev) + " is current, the context was created on device " +
                 std::to_string(c->device);
        return LH_EINVAL;
    }
    double *scratch = nullptr;
    if (e == cudaSuccess) e = scratch_on_current_device(&scratch);
    if (e != cudaSuccess) {
        c->err = std::string("lh_lusolu_noalloc: scratch lookup: ") + cudaGetErrorString(e);
        return LH_ECUDA;
    }
    // an error left by earlier work on this thread is reported as such, not
    // as this launch's
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        c->err = std::string("lh_lusolu_noalloc: earlier error on this thread: ") + cudaGetErrorString(e);
        return LH_ECUDA;
    }
    lh::k_lusolu<<<(s.nc + 127) / 128, 128, 0, c->st>>>(c->d_inst, grid, kRK, dt,
                                                       reinterpret_cast<const double2 *>(rhs_dev),
                                                       reinterpret_cast<double2 *>(u_dev), scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        c->err = std::string("lh_lusolu_noalloc: launch: ") + cudaGetErrorString(e);
        return LH_ECUDA;
    }
    return LH_OK;
}
