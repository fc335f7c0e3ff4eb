// Shared device helpers for the cat-surface B200 kernels.
//
// Everything here is plain CUDA C++ for sm_100a: cache-hinted loads/stores,
// a bounded grid barrier for persistent cooperative kernels, and the status
// word every persistent kernel reports through.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/catsurf_b200.h"

namespace csg {

// Status word layout inside a kernel's control block (first 256 bytes of its
// scratch).  word 0: barrier arrival counter; word 1: status (CSG_OK or a
// negative CSG_ERR_*); word 2: index of the barrier/step that failed.
struct Control {
    unsigned int arrivals;
    int status;
    int where;
    int pad[61];
};
static_assert(sizeof(Control) == 256, "control block is 256 bytes");

__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_relaxed_gpu(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release_gpu_add(unsigned int* p, unsigned int v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier for a cooperatively launched (all CTAs co-resident)
// kernel.  `phase` counts the arrivals expected so far and must be advanced
// identically by every CTA.  Waits are bounded by `timeout_ns`; on timeout or
// when another CTA has already reported an error the barrier returns true
// and the caller must leave the kernel.  No trap, no unbounded spin.
__device__ __forceinline__ bool grid_barrier(Control* ctl, unsigned int& phase, unsigned long long timeout_ns,
                                             int where) {
    __shared__ int s_abort;
    __syncthreads();
    phase += gridDim.x;
    if (threadIdx.x == 0) {
        __threadfence();
        red_release_gpu_add(&ctl->arrivals, 1u);
        int abort = 0;
        unsigned long long start = global_timer_ns();
        unsigned int polls = 0;
        while (true) {
            unsigned int seen = ld_acquire_gpu(&ctl->arrivals);
            if (static_cast<int>(seen - phase) >= 0) break;
            if (((++polls) & 31u) == 0u) {
                if (ld_relaxed_gpu(&ctl->status) != CSG_OK) { abort = 1; break; }
                if (global_timer_ns() - start > timeout_ns) {
                    if (atomicCAS(&ctl->status, CSG_OK, CSG_ERR_TIMEOUT) == CSG_OK) ctl->where = where;
                    abort = 1;
                    break;
                }
            }
        }
        s_abort = abort;
    }
    __syncthreads();
    return s_abort != 0;
}

}  // namespace csg
