// ct_device.cuh — device-side helpers for sm_100a: mbarriers, TMA 2D tile
// loads (no multicast), bounded waits, packed u16x2 integer ops.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace ct {
namespace dev {

// Upper bound on mbarrier polls. A TMA tile load completes in microseconds;
// if a phase has not completed after this many polls (each try_wait may
// suspend the thread for a while), the wait gives up and the kernel reports
// CT_ETIMEOUT through its status word instead of hanging the GPU.
constexpr uint32_t kWaitLimit = 1u << 20;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of `bar`: at most `limit` polls. Returns
// false if it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit = kWaitLimit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 2D tiled TMA load global -> shared, completion signalled on `bar`.
// x is the innermost coordinate in elements; x * elem_bytes must be a
// multiple of 16 (callers keep x even for 8-byte and a multiple of 16 for
// 1-byte elements). Out-of-range coordinates read zeros.
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, int32_t x, int32_t y,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// 4D tiled TMA load (coordinates innermost first; the innermost one stays 0
// in this library, so its 16-byte alignment rule always holds).
__device__ __forceinline__ void tma_load_4d(void* smem_dst, const CUtensorMap* map, int32_t c0, int32_t c1,
                                            int32_t c2, int32_t c3, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// 3D tiled TMA load (coordinates innermost first). The innermost coordinate
// times the element size must be a multiple of 16 bytes; callers pass a
// multiple of 4 for 4-byte elements.
__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, int32_t c0, int32_t c1,
                                            int32_t c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Packed unsigned 16-bit lane helpers.
__device__ __forceinline__ uint32_t min3_u16x2(uint32_t a, uint32_t b, uint32_t c) {
    return __vimin3_u16x2(a, b, c);
}
__device__ __forceinline__ uint32_t min_u16x2(uint32_t a, uint32_t b) { return __vminu2(a, b); }

// Records an error code in the status word (first writer wins).
__device__ __forceinline__ void report(int32_t* status, int32_t code) {
    if (status) atomicCAS(status, 0, code);
}

}  // namespace dev
}  // namespace ct
