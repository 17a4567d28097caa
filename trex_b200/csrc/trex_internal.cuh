// Internal declarations shared by the CUDA translation units of libtrex_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/trex_b200.h"

namespace trex {

// ---- error plumbing -------------------------------------------------------
// The library never exits the process: every CUDA failure becomes a return
// code. The last CUDA error string is kept per thread for trex_last_error().
void set_last_error(const char *where, cudaError_t err);
void set_last_error_msg(const char *msg);

#define TREX_CUDA(call)                                              \
    do {                                                             \
        cudaError_t _e = (call);                                     \
        if (_e != cudaSuccess) {                                     \
            ::trex::set_last_error(#call, _e);                       \
            return TREX_ERR_CUDA;                                    \
        }                                                            \
    } while (0)

#define TREX_CHECK_LAUNCH()                                          \
    do {                                                             \
        cudaError_t _e = cudaGetLastError();                         \
        if (_e != cudaSuccess) {                                     \
            ::trex::set_last_error("kernel launch", _e);             \
            return TREX_ERR_CUDA;                                    \
        }                                                            \
    } while (0)

// ---- device helpers ---------------------------------------------------------
// Streaming 16-byte load: non-coherent, no L1 allocation, L2 fetches 256 B.
__device__ __forceinline__ uint4 ld_stream16(const void *p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::256B.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
    return v;
}

// Streaming 32-byte load (two halves returned as uint4).
__device__ __forceinline__ void ld_stream32(const void *p, uint4 &lo, uint4 &hi) {
    asm volatile("ld.global.nc.L1::no_allocate.L2::256B.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(lo.x), "=r"(lo.y), "=r"(lo.z), "=r"(lo.w),
                   "=r"(hi.x), "=r"(hi.y), "=r"(hi.z), "=r"(hi.w)
                 : "l"(p));
}

__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" :: "l"(p));
}

__device__ __forceinline__ void st_stream16(void *p, uint4 v) {
    asm volatile("st.global.L1::no_allocate.v4.u32 [%0], {%1,%2,%3,%4};"
                 :: "l"(p), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w) : "memory");
}

// Streaming 32-byte store (two halves), 32-byte aligned.
__device__ __forceinline__ void st_stream32(void *p, uint4 lo, uint4 hi) {
    asm volatile("st.global.L1::no_allocate.v8.u32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
                 :: "l"(p), "r"(lo.x), "r"(lo.y), "r"(lo.z), "r"(lo.w), "r"(hi.x), "r"(hi.y), "r"(hi.z),
                    "r"(hi.w) : "memory");
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t *p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t lane_id() {
    uint32_t l;
    asm("mov.u32 %0, %%laneid;" : "=r"(l));
    return l;
}

// ---- sizes --------------------------------------------------------------------
constexpr int kMaxDfasPerSet = 64;     // resident automata in one set
constexpr int kSmallDfaStates = 16;    // replicated-table fast path
constexpr int kMaxPlainStates = 256;   // plain-table path (uint8 states)

// Byte counts of the per-lane replicated transition tables held in shared
// memory by the batch kernels (N <= 8 and N <= 16 layouts).
constexpr int kRepTableBytes8 = 256 * 256;    // 64 KiB
constexpr int kRepTableBytes16 = 256 * 512;   // 128 KiB

int sm_count();

// Limits of the kernels' bounded waits: polls of one look-back step of the
// per-position scan, and clock cycles of one mbarrier hand-off of the
// tensor-core NFA kernel. Process-wide; trex_set_wait_limits changes them (for
// tests of the give-up paths), 0 restores the defaults.
constexpr uint32_t kDefaultScanPolls = 1u << 24;
constexpr long long kDefaultMbarCycles = 4000000000ll;   // about 2 s
uint32_t scan_poll_limit();
long long mbar_wait_cycles();

// Launch profiler hooks (no-ops unless trex_profile_begin was called).
void profile_kernel_begin(cudaStream_t s);
void profile_kernel_end(cudaStream_t s);

}  // namespace trex
