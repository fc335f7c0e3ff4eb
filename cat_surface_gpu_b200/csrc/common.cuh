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

// Correctly rounded x / 3 for finite binary64 x with |x| >= 2^-1000 (far from
// the subnormal range, where RN(x zl) loses the needed bits) with two
// multiplies (Brisebarre, Muller and Raina, "Accelerating correctly rounded
// floating-point division when the divisor is known in advance", IEEE TC
// 53(8), 2004): q = RN(x zh + RN(x zl)) with zh = RN(1/3) and
// zl = RN(1/3 - zh) = zh * 2^-54.  Why it is exact for the divisor 3: the
// exact quotient x/3 = M 2^e / 3 sits at a multiple of a third of a unit in
// the last place, so it is never closer than 1/6 ulp to a rounding midpoint,
// while x zh + RN(x zl) is within ~2^-105 relative of x/3.  Equal to
// __ddiv_rn(x, 3.0) bit for bit (csg_selftest_div3 and the sweep and
// preprocess tests, which compare against the oracle's plain division).
__device__ __forceinline__ double div3_rn(double x) {
    const double zh = 0x1.5555555555555p-2;
    const double zl = 0x1.5555555555555p-56;
    return __fma_rn(x, zh, __dmul_rn(x, zl));
}

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
// Ordering: __syncthreads orders the CTA's writes before thread 0's arrival,
// a release at gpu scope (cumulative, so it covers what thread 0 has
// observed through the CTA barrier); the acquire poll and the closing
// __syncthreads order the other CTAs' writes before this CTA's next reads.
__device__ __forceinline__ bool grid_barrier(Control* ctl, unsigned int& phase, unsigned long long timeout_ns,
                                             int where) {
    __shared__ int s_abort;
    __syncthreads();
    phase += gridDim.x;
    if (threadIdx.x == 0) {
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

// Versioned words of the dataflow kernels: a float32 value and the number of
// updates it belongs to in one 8-byte word.  Aligned 8-byte accesses are
// single-copy atomic, so a relaxed load returns a value together with its own
// version and needs no acquire ordering.
__device__ __forceinline__ unsigned long long ld_word(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_word(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long make_word(float x, unsigned int version) {
    return (static_cast<unsigned long long>(version) << 32) | __float_as_uint(x);
}
__device__ __forceinline__ float word_value(unsigned long long w) { return __uint_as_float(static_cast<unsigned>(w)); }
__device__ __forceinline__ unsigned int word_version(unsigned long long w) { return static_cast<unsigned>(w >> 32); }

// Work distribution of a dataflow kernel with few items per step (the
// coloured SOR): the items of successive wavefront steps are dealt to a CTA's
// groups round-robin without restarting at group 0 each step: item k of a
// step goes to group (rot + k) mod groups, rot = items dealt in earlier steps
// mod groups.  Each group still takes its items in step order (progress is
// guaranteed as in the step-by-step form), and groups without an item in this
// step take the next steps' items, so several steps are in flight in a CTA.
// Returns the first item index of this warp's first group (<= 0); the warp's
// groups then take k = first + g + j * groups, valid while 0 <= k < count.
__device__ __forceinline__ int dealt_first(int rot, int warp_first_group, int groups) {
    return -(((rot - warp_first_group) % groups + groups) % groups);
}

// Bounded wait of one warp in a dataflow kernel: lane 0 checks the clock and
// the status word every 64 polls; true (the same in every lane) means give up
// -- the status is CSG_ERR_TIMEOUT (recorded here) or another CTA's error.
__device__ __forceinline__ bool warp_wait_expired(Control* ctl, unsigned long long timeout_ns, unsigned int& polls,
                                                  unsigned long long& start) {
    int expired = 0;
    if ((threadIdx.x & 31) == 0 && ((++polls) & 63u) == 0u) {
        const unsigned long long now = global_timer_ns();
        if (start == 0) start = now;
        if (ld_relaxed_gpu(&ctl->status) != CSG_OK) {
            expired = 1;
        } else if (now - start > timeout_ns) {
            if (atomicCAS(&ctl->status, CSG_OK, CSG_ERR_TIMEOUT) == CSG_OK) ctl->where = -2;
            expired = 1;
        }
    }
    return __shfl_sync(0xffffffffu, expired, 0) != 0;
}

}  // namespace csg
