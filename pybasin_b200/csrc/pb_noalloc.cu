// Allocation-free entry point: pb_solve_batch with its scratch in a fixed
// device array of this library instead of caller-allocated memory.
//
// Some callers cannot allocate device memory on demand: a host application that
// hands the GPU to plug-ins under a fixed memory budget and owns every device
// allocation through its own pool, or a latency-critical loop in which a
// cudaMalloc (which may synchronise the device and take unbounded time) is not
// allowed.  Those callers still own the inputs and outputs; only the integrator's
// internal scratch (queue counter, step records, per-trajectory tails, median
// windows) lives here.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "pb_scratch.cuh"
#include "pybasin_b200.h"

namespace {

// Every GPU that loads this library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[PB_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
struct DeviceSlot {
    CUcontext ctx;  // the context the address was looked up in
    void* addr;
};
DeviceSlot g_slot[kMaxDevices] = {};

using FnCtxGetCurrent = CUresult (*)(CUcontext*);

// cuCtxGetCurrent through the runtime's driver entry points (the library does not
// link libcuda); nullptr if the driver does not provide it
FnCtxGetCurrent ctx_get_current()
{
    static FnCtxGetCurrent fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<FnCtxGetCurrent>(p);
    });
    return fn;
}

// Device address of the array on the current device.  The name g_noalloc_scratch
// is only a host-side handle; the address the kernels use comes from
// cudaGetSymbolAddress with that device current.  It is looked up on the first
// call on a device and again whenever the device's context has changed since
// (after cudaDeviceReset the module, and with it the array, lives in a new
// context at a possibly different address).
cudaError_t device_scratch(void** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    const FnCtxGetCurrent get = ctx_get_current();
    if (!get) return cudaErrorNotSupported;
    CUcontext ctx = nullptr;  // stays null until the runtime has made a context current
    if (get(&ctx) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSlot& s = g_slot[dev];
    if (!s.addr || !ctx || s.ctx != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // initialises the primary context if needed
        if (e != cudaSuccess) return e;
        if (!ctx && (get(&ctx) != CUDA_SUCCESS || !ctx)) return cudaErrorDeviceUninitialized;
        s.addr = p;
        s.ctx = ctx;
    }
    *out = s.addr;
    return cudaSuccess;
}

}  // namespace

extern "C" int pb_solve_batch_noalloc(const pb_solve_args* args, void* stream)
{
    if (!args) return PB_EINVAL;
    if (args->n_traj < 0 || args->n_save < 1 || args->win_begin < 0 || args->win_begin >= args->n_save)
        return PB_EINVAL;
    // the scratch size walks the feature arrays up to n_features: bound it first
    // (pb_solve_batch validates everything else before it launches)
    if (args->n_features < 0 || args->n_features > PB_MAX_FEATURES) return PB_EINVAL;
    // scratch of pb_solve_batch followed by the work-queue counter (256-byte aligned)
    const int64_t need = pb_solve_scratch_bytes(args);
    if (need < 0) return PB_EINVAL;
    const int64_t total = need + 256;
    if (total > static_cast<int64_t>(PB_NOALLOC_SCRATCH_BYTES)) return PB_ESCRATCH_LIMIT;
    void* base = nullptr;
    cudaError_t e = device_scratch(&base);
    if (e != cudaSuccess) return PB_ECUDA;
    pb_solve_args a = *args;
    a.scratch = need > 0 ? base : nullptr;
    a.queue_counter = reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(base) + need);
    // pb_solve_batch zeroes the queue counter on `stream` itself; records, tails and
    // median windows are written before they are read, so nothing else needs clearing.
    return pb_solve_batch(&a, stream);
}
