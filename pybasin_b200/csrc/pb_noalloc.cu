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
#include <cuda_runtime.h>

#include <mutex>

#include "pb_scratch.cuh"
#include "pybasin_b200.h"

namespace {

// Every GPU that loads this library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[PB_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the array on the current device, looked up once per device.
// The name g_noalloc_scratch is only a host-side handle; the address the kernels
// use must come from cudaGetSymbolAddress with that device current.
cudaError_t device_scratch(void** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" int pb_solve_batch_noalloc(const pb_solve_args* args, void* stream)
{
    if (!args) return PB_EINVAL;
    if (args->n_traj < 0 || args->n_save < 1 || args->win_begin < 0 || args->win_begin >= args->n_save)
        return PB_EINVAL;
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
