// Host-side kernel handles shared by the built-in dispatch (pb_api.cu) and the
// runtime-compiled right-hand sides (pb_rtc.cu).  A handle is either a kernel
// of this library (a runtime-API symbol) or a function loaded from an NVRTC
// cubin (a driver-API CUfunction); the solve passes launch either the same way.
#pragma once
#include <cuda_runtime.h>

#include "pybasin_b200.h"

namespace pb {

struct KFn {
    const void* rt = nullptr;  // kernel symbol of this library
    void* drv = nullptr;       // CUfunction of a runtime-compiled module
    bool ok() const { return rt != nullptr || drv != nullptr; }
};

struct KernelSel {
    KFn plain;         // inline dense output, one thread per trajectory
    KFn plain_defer;   // deferred pass 1
    KFn queue;         // inline dense output, persistent warps (also the redo pass)
    KFn queue_defer;   // deferred pass 1, persistent warps
    KFn queue_probe;   // deferred pass 1, probed schedule: probe phase
    KFn queue_main;    // deferred pass 1, probed schedule: main phase
    KFn queue_main_s1; // ... with the sampling of 1 (2) feature states drained into it
    KFn queue_main_s2;
    int smem_per_thread = 0;  // inline kernels: per-thread statistics slot
};

// the argument checks and the solve passes of pb_solve_batch, for any kernel set
int validate_args(const pb_solve_args* a, bool user_system);
int solve_with(const KernelSel& k, const pb_solve_args& a, cudaStream_t st);

// driver-API calls on a CUfunction (pb_rtc.cu)
cudaError_t drv_launch(void* fn, unsigned grid, unsigned block, unsigned smem, cudaStream_t st, void** argv);
cudaError_t drv_occupancy(void* fn, int block, int smem, int* blocks_per_sm);
cudaError_t drv_set_max_smem(void* fn, int bytes);

}  // namespace pb
