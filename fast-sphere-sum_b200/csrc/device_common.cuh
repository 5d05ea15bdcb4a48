// device_common.cuh -- sm_100a device helpers: mbarrier + bulk-copy (TMA)
// wrappers with bounded waits, fast reciprocal / log2, vector types.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "fss_internal.h"

namespace fss {

template <typename T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double4; };

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Make barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Raise the transaction count of the current phase without arriving.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
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

// Wait for phase `parity` of `bar` to complete; false after limit_ns.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_timer_ns() - t0 > limit_ns) return false;
    }
}

// Bulk (non-tensor) TMA copy global -> this CTA's shared memory, completing
// `bytes` transactions on `bar`.  Source and destination 16-byte aligned,
// bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ float rcp_fast(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float lg2_fast(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// FP64 reciprocal: hardware approximation refined by two Newton-Raphson
// steps y <- y + y (1 - x y) (quadratic convergence from the approximation's
// ~2^-20 relative error to below FP64 rounding).
__device__ __forceinline__ double rcp_fast(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    return y;
}

__device__ __forceinline__ double lg2_fast(double x) { return log2(x); }

// Packed FP32 pairs (sm_100 f32x2 arithmetic): two floats in one 64-bit
// register pair, one instruction for both lanes.
typedef unsigned long long f2;
__device__ __forceinline__ f2 f2_pack(float a, float b) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_unpack(f2 r, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) {
    f2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
    f2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// FP64 tensor-core multiply-accumulate of one warp (m8n8k4, A row-major 8x4,
// B column-major 4x8): lane = 4 g + t holds A[g][t], B[t][g] and the
// accumulators D[g][2t], D[g][2t + 1].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Order this thread's generic-proxy shared-memory writes before later
// async-proxy (TMA) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void set_error(int* err, int code) {
    if (err) atomicCAS(err, 0, code);
}

// A block's one-shot bulk staging: thread 0 initialises `bar` and copies
// `bytes` (a multiple of 16; both addresses 16-byte aligned) of global memory
// into shared memory; after a __syncthreads every thread calls stage_wait.
// hold (test hook): the bytes are expected but no copy is issued, so the
// wait runs out with nothing in flight.
__device__ __forceinline__ void stage_issue(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                            bool hold = false) {
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init_fence();
        mbar_arrive_expect_tx(bar, bytes);
        if (!hold) bulk_g2s(dst, src, bytes, bar);
    }
}

// Waits (bounded) for the staged copy; false in every thread of the block
// when it did not land in time, after a second bounded wait, so that no copy
// is left in flight when the block returns.
__device__ __forceinline__ bool stage_wait(uint64_t* bar, uint64_t limit_ns) {
    const bool ok = __syncthreads_and(mbar_wait_bounded(bar, 0, limit_ns)) != 0;
    if (!ok) mbar_wait_bounded(bar, 0, limit_ns);
    return ok;
}

}  // namespace fss
