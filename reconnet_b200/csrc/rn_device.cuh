// Device helpers: mbarrier + bulk (TMA, non-tensor) copies for sm_100a, and
// small numeric utilities.  Every wait is bounded (rn::kSpinLimit).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rn_internal.h"

namespace rn {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

// Returns true when the phase with the given parity has completed, false if
// the bounded spin (`limit` polls) ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit = kSpinLimit) {
    uint32_t addr = smem_u32(bar);
    for (long long it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Bulk global -> shared copy completing on an mbarrier (cp.async.bulk, no
// multicast).  dst/src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// floor(x) and frac(x) for 0 <= x < 2^22 on the FMA/ALU pipes: the integer
// part comes from rounding (x - 0.5) with a 1.5 * 2^23 bias.  At exact
// integers it may return (n-1, 1.0) instead of (n, 0.0); both evaluate the
// same prefix value because entry n-1 plus one full pixel is entry n.
__device__ __forceinline__ int floor_frac(float x, float& frac) {
    const float kBias = 12582912.0f;  // 1.5 * 2^23
    float y = (x - 0.5f) + kBias;
    int k = __float_as_int(y) - 0x4B400000;
    frac = x - (y - kBias);
    return k;
}

// Error-free split of a double into hi + lo floats.
__device__ __forceinline__ float2 split_double(double v) {
    float hi = __double2float_rn(v);
    float lo = __double2float_rn(v - (double)hi);
    return make_float2(hi, lo);
}

// Inclusive prefix sum over the 32 lanes of a warp (all lanes participate).
__device__ __forceinline__ double warp_incl_scan(double v) {
    const unsigned full = 0xffffffffu;
    int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double t = __shfl_up_sync(full, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

}  // namespace rn
