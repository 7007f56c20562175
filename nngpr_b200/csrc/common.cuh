// Shared device/host helpers of libnngp_b200 (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/nngp_b200.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "libnngp_b200 is built for sm_100a only"
#endif

namespace nngp {

constexpr int kNumSMsB200 = 148;
// A bounded wait gives up after this many nanoseconds of %globaltimer (well above any
// legitimate wait: the longest single copy here is a few KB).
constexpr uint64_t kWaitLimitNs = 2000000000ull;

// ---------------------------------------------------------------------------------------
// Host-side error state
// ---------------------------------------------------------------------------------------
void set_error(const std::string &msg);
nngp_status fail(nngp_status st, const std::string &msg);
nngp_status cuda_fail(cudaError_t e, const char *what);

#define NNGP_CUDA_TRY(call)                                          \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return ::nngp::cuda_fail(e_, #call);  \
    } while (0)

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Raise a kernel's dynamic shared-memory limit (and, carveout >= 0, its preferred carveout) once
// per process and device: later calls, including calls made while a stream is being captured
// into a CUDA graph, find the setting cached and make no CUDA call.  Defined in abi.cu.
cudaError_t ensure_smem_limit(const void *fn, int bytes, int carveout = -1);

// ---------------------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void flag_or(int32_t *flags, int32_t bits) {
    if (flags) atomicOr(flags, bits);
}

// One rounding per operation (never contracted into FMA): the exact-distance arithmetic
// that the CPU restatement reproduces bit for bit.
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

template <typename T> __device__ __forceinline__ T pos_inf();
template <> __device__ __forceinline__ float pos_inf<float>() { return __int_as_float(0x7f800000); }
template <> __device__ __forceinline__ double pos_inf<double>() { return __longlong_as_double(0x7ff0000000000000ll); }
template <typename T> __device__ __forceinline__ T neg_inf();
template <> __device__ __forceinline__ float neg_inf<float>() { return __int_as_float(0xff800000); }
template <> __device__ __forceinline__ double neg_inf<double>() { return __longlong_as_double(0xfff0000000000000ll); }

// ---- mbarrier + TMA bulk copy (cp.async.bulk, no multicast) ----------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase: false after limit_ns without completion.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint64_t limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_timer_ns() - t0 > limit_ns) return false;
    }
}

// Limit of the bounded waits in the search's main loop (a kernel argument; kWaitLimitNs unless
// nngp_set_wait_limit_ns changed it to exercise the failure path).  The waits that drain a
// CTA's own copies and MMAs before it frees TMEM always use kWaitLimitNs.  Defined in abi.cu.
uint64_t wait_limit_ns();

// Global -> shared bulk copy completing on `bar` (16-byte aligned addresses, bytes % 16 == 0).
__device__ __forceinline__ void tma_bulk_g2s(void *dst_smem, const void *src_gmem, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// ---- warp helpers ----------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace nngp
