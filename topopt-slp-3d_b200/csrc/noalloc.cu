// KelemProd without any device allocation: tosp_kelem_prod_noalloc.
//
// Some callers cannot allocate device memory at the time they need the
// product.  A host whose GPU memory is handed out by its own pooling
// allocator (a MATLAB session holding gpuArray data) owns the device's free
// memory, so a cudaMalloc from a MEX file competes with that pool and can
// fail.  Pipelines that keep work in flight on several streams cannot take a
// cudaMalloc or cudaFree, which may synchronise the whole device.  Services
// that fix their device footprint at start-up allow no allocation after it.
// For them this entry point takes its only scratch - the two zero-extended
// full-length vectors of KelemProd - from a fixed array in device memory that
// is part of the loaded library.
//
// The call runs at once: its work is queued on the handle's own stream and it
// returns after y is written.  x must therefore be complete before the call
// (synchronise the stream that produced it first).
//
// Limits and rules:
//  * the array holds 2 x TOSP_NOALLOC_MAX_DOFS doubles (16 MiB); every GPU
//    that loads the library keeps it until the process exits, and problems
//    with more than TOSP_NOALLOC_MAX_DOFS dofs (3 * nnodes) are rejected;
//  * all calls share the array and it keeps the last call's contents, so
//    calls whose GPU work overlaps (two host threads, two handles on the same
//    device) race and must be serialised by the caller;
//  * the first call on a device resolves the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current); make
//    that first call before any stream capture;
//  * device ordinals up to kMaxDevices - 1 (64 GPUs per process) are served.
#include <mutex>
#include <string>

#include "tosp_internal.h"

#define TOSP_NOALLOC_MAX_DOFS (1LL << 20)

static __device__ __align__(256) double g_noalloc_scratch[2 * TOSP_NOALLOC_MAX_DOFS];

namespace {
constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// Device address of the scratch array on `dev` (0 <= dev < kMaxDevices; the
// host-side symbol is only a stand-in and must never reach a kernel).
// Resolved once per device with that device current.
cudaError_t scratch_for_device(int dev, double **out) {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}
}  // namespace

extern "C" int tosp_kelem_prod_noalloc(tosp_handle *h, const double *x, double *y, int64_t nfree) {
    if (!h || !x || !y) return TOSP_ERR_BAD_ARG;
    const int dev = tosp::handle_device(h);
    if (dev < 0 || dev >= kMaxDevices) {
        tosp::set_handle_error(h, "tosp_kelem_prod_noalloc: device " + std::to_string(dev) +
                                      " is beyond the " + std::to_string(kMaxDevices) +
                                      " devices whose scratch addresses this entry point keeps (use tosp_kelem_prod)");
        return TOSP_ERR_UNSUPPORTED;
    }
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) {
        tosp::set_handle_error(h, std::string("cudaSetDevice failed: ") + cudaGetErrorString(e));
        return TOSP_ERR_CUDA;
    }
    const int64_t ndof = tosp::handle_ndof(h);
    if (ndof > TOSP_NOALLOC_MAX_DOFS) {
        tosp::set_handle_error(h, "tosp_kelem_prod_noalloc: problem has " + std::to_string(ndof) +
                                      " dofs, more than the fixed scratch limit of " +
                                      std::to_string((long long)TOSP_NOALLOC_MAX_DOFS) + " (use tosp_kelem_prod)");
        return TOSP_ERR_BAD_ARG;
    }
    double *scratch = nullptr;
    e = scratch_for_device(dev, &scratch);
    if (e != cudaSuccess) {
        tosp::set_handle_error(h, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        return TOSP_ERR_CUDA;
    }
    return tosp::kelem_prod_with_scratch(h, x, y, nfree, scratch, scratch + TOSP_NOALLOC_MAX_DOFS);
}
