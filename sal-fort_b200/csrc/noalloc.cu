// Allocation-free variant of the FP64 direct sum.
//
// sal_direct_sum keeps its per-chunk partial sums in a device buffer it grows
// with cudaMalloc.  Some callers cannot allow that: a host thread that runs
// while another framework's caching allocator already owns the device memory
// (cudaMalloc then fails), or a caller that cannot accept the implicit
// device-wide synchronisation cudaMalloc and cudaFree may perform.  This entry
// point takes its scratch from a fixed array in the library's own device
// memory instead, and allocates nothing.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/salgpu.h"
#include "kernels.cuh"

namespace sal {
int set_error(int code, const std::string &msg);
}

// 2 MiB of partial sums (SAL_NOALLOC_SCRATCH_DOUBLES doubles).  Every GPU that
// loads the library holds it until the process exits.  All calls share it and
// it keeps the last call's contents; the direct-sum kernel writes every slot it
// later reads, so nothing needs clearing between calls.
static __device__ __align__(256) double g_noalloc_scratch[SAL_NOALLOC_SCRATCH_DOUBLES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_scratch_ptr[kMaxDevices] = {nullptr};
}  // namespace

// Device address of the scratch array on the current device.  In host code
// g_noalloc_scratch names a host-side stand-in, so the address is looked up
// once per device (with that device current) and cached for the rest of the
// process.  A cudaDeviceReset would recreate the device's context and leave
// the cached address stale; the header tells callers not to reset a device
// between calls.
static int scratch_address(int dev, double **out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return sal::set_error(SAL_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_ptr[dev];
    return SAL_OK;
}

extern "C" int sal_direct_sum_noalloc(const double *xs, const double *ys, const double *zs, const double *w,
                                      int32_t n, const int32_t *targets, int32_t nt, double *out_x, double *out_y,
                                      void *stream) {
    if (!xs || !ys || !zs || !w || !targets || !out_x || !out_y) return sal::set_error(SAL_EINVAL, "null argument");
    if (n < 0 || nt < 0) return sal::set_error(SAL_EINVAL, "negative size");
    if ((int64_t)nt * 2 > (int64_t)SAL_NOALLOC_SCRATCH_DOUBLES)
        return sal::set_error(SAL_EINVAL, "sal_direct_sum_noalloc: nt = " + std::to_string(nt) +
                                              " exceeds the scratch limit of " +
                                              std::to_string(SAL_NOALLOC_SCRATCH_DOUBLES / 2) + " targets");
    if (nt == 0) return SAL_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return sal::set_error(SAL_ENODEV, "no CUDA device is available");
    if (dev >= kMaxDevices) return sal::set_error(SAL_EINVAL, "device ordinal >= 64");
    double *scratch = nullptr;
    int rc = scratch_address(dev, &scratch);
    if (rc) return rc;
    // as many source chunks as the scratch holds for nt targets, at most the
    // count the allocating entry point uses
    const int cap = (int)((int64_t)SAL_NOALLOC_SCRATCH_DOUBLES / (2 * (int64_t)nt));
    int nch = sal::dev::direct_chunks(n);
    if (nch > cap) nch = cap;
    sal::dev::launch_direct(xs, ys, zs, w, n, targets, nt, out_x, out_y, scratch, nch, (cudaStream_t)stream);
    e = cudaGetLastError();
    if (e != cudaSuccess) return sal::set_error(SAL_ECUDA, cudaGetErrorString(e));
    return SAL_OK;
}
