// Tensor-memory-access (TMA) copies and shared-memory transaction barriers for sm_100a, as inline
// PTX, plus the host-side encoder of tensor maps (fetched from the driver at run time, so the
// library does not link libcuda).
//
// Rules kept by every user of this file:
//   * no multicast form of any copy is used (every copy is CTA-local);
//   * every wait on a barrier is bounded in time (`wait`): a wait that runs out sets a fault bit the
//     host reads with prc_device_fault_flags(), and the kernel drains its own copies (again with a
//     bound) and returns instead of spinning;
//   * tiled copies start at an innermost coordinate whose byte offset is a multiple of 16, from
//     16-byte aligned global memory with 16-byte multiple strides, into 128-byte aligned shared
//     memory (checked on the host when the map is encoded and on the device before the first copy).
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace prc {
namespace tma {

// Bit set in the device fault word when a bounded wait gave up.
constexpr unsigned FAULT_WAIT_TIMEOUT = 1u;
constexpr unsigned FAULT_SMEM_ALIGN = 2u;
// Longest wait for one copy before the kernel gives up (ns of %globaltimer).
constexpr uint64_t WAIT_LIMIT_NS = 200ull * 1000 * 1000;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void barrier_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the copy engine.
__device__ __forceinline__ void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders this CTA's earlier shared-memory accesses (made visible to the issuing thread by a CTA
// barrier) before the copy engine's next accesses.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// One arrival (release at CTA scope) on a barrier counting threads, not bytes.
__device__ __forceinline__ void arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase of `parity` to complete; false if it has not after `limit_ns`.
__device__ __forceinline__ bool wait_for(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    if (try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    while (!try_wait(bar, parity))
        if (globaltimer() - t0 > limit_ns) return false;
    return true;
}

// Waits for the phase of `parity` to complete; false if it has not after WAIT_LIMIT_NS.
__device__ __forceinline__ bool wait(uint64_t* bar, uint32_t parity) { return wait_for(bar, parity, WAIT_LIMIT_NS); }

__device__ __forceinline__ void barrier_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Tiled 3D copy global -> shared (this CTA), completion counted in bytes on `bar`.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_addr(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
        : "memory");
}

// Contiguous copy global -> shared (this CTA): addresses and size multiples of 16 bytes.
__device__ __forceinline__ void load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

// Up to six tensor maps passed by value as one __grid_constant__ kernel parameter.
struct Maps {
    CUtensorMap m[6];
};

}  // namespace tma
}  // namespace prc
