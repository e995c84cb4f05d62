// pf_batch_device_noalloc: the device-resident batch entry point without any allocation.
//
// Who needs it.  Some callers of this library cannot let it call cudaMalloc:
//   * code that runs while a CUDA stream is being captured into a graph -- a device
//     allocation during capture is not recorded into the graph and, with the default
//     capture mode, invalidates the capture;
//   * hosts that give every library a fixed device-memory budget through their own
//     allocator (a serving process that has pre-partitioned the GPU) and fail any
//     allocation made behind their back;
//   * plugin hosts whose contract forbids a plugin from allocating device memory on the
//     calls that do the work.
// For them this entry point runs the same Newton-Raphson kernel as pf_batch_device, but
// takes its per-CTA working memory (the slabs holding voltages, currents, mismatches and,
// when the factor does not fit in shared memory, the LU values) and its job counter from a
// file-scope device array instead of the plan's buffers.  A mixed-precision plan re-solves an
// instance that fails in FP32 in FP64 inside the launch, as pf_batch_device does, so the two
// entry points give the same results; its slabs then also hold an FP64 LU.
//
// Limits and rules.
//   * The array is kNoAllocScratchBytes (32 MiB) and exists on every GPU that loads this
//     library, until the process exits.  A plan whose CTA slab does not fit is rejected
//     with an error; otherwise the launch uses as many CTAs as there are slabs in the array
//     (at most the plan's own grid), so large grids may run on fewer CTAs than
//     pf_batch_device would use (the 2,848-bus mixed plan, whose slab carries room for the
//     FP64 fallback's LU, runs on about 50 CTAs).
//   * The current device must be the plan's device (checked before anything else).
//   * The first call on a device looks the array's device address up (cudaGetSymbolAddress
//     with that device current) and caches it; make that first call before any stream
//     capture begins.  Later calls do no set-up.
//   * Every call shares the one array, and the array keeps what the previous call left in
//     it: the job counter is cleared (cudaMemsetAsync on the caller's stream) before each
//     launch, and every slab value is written before it is read.  Calls whose kernels can
//     overlap on the GPU (different streams, different threads) race on the array: issue
//     them on one stream, or serialise them.
//   * The plan must exist (pf_plan_create allocates the plan's structure once); inputs and
//     outputs are the caller's device pointers, as for pf_batch_device.
#include <mutex>
#include <string>

#include "../../include/lightsim2grid_b200.h"
#include "pf_capi_internal.hpp"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

// working memory of pf_batch_device_noalloc (per device, for the life of the process)
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {};

}  // namespace

extern "C" int pf_batch_device_noalloc(pf_plan *plan, const pf_device_batch *batch, void *stream) {
    if (!plan || !batch) {
        l2g::set_last_error("pf_batch_device_noalloc: null argument");
        return -1;
    }
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        l2g::set_last_error(std::string("pf_batch_device_noalloc: no usable current device: ") +
                            cudaGetErrorString(e));
        return -2;
    }
    if (dev != l2g::plan_device(plan)) {
        // the array's address is per device: a launch with another device's address would mix
        // two GPUs' memory
        l2g::set_last_error("pf_batch_device_noalloc: the plan was built on device " +
                            std::to_string(l2g::plan_device(plan)) + " but device " + std::to_string(dev) +
                            " is current");
        return -1;
    }
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        scratch = g_scratch_addr[dev];
        if (scratch == nullptr) {
            // host code must not use g_noalloc_scratch itself: its host-side name is a stand-in,
            // not a device address; look the device address up once per device
            e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
            if (e != cudaSuccess || scratch == nullptr) {
                l2g::set_last_error(std::string("pf_batch_device_noalloc: cudaGetSymbolAddress failed: ") +
                                    cudaGetErrorString(e));
                return -2;
            }
            g_scratch_addr[dev] = scratch;
        }
    }
    const size_t need = l2g::plan_fallback_slab_bytes(plan) + 256;
    if (need > kNoAllocScratchBytes) {
        l2g::set_last_error("pf_batch_device_noalloc: one CTA of this plan needs " + std::to_string(need) +
                            " bytes of working memory, more than the " + std::to_string(kNoAllocScratchBytes) +
                            "-byte static scratch array; use pf_batch_device");
        return -1;
    }
    return l2g::batch_device_with_scratch(plan, batch, stream, scratch, kNoAllocScratchBytes, true);
}
