// One-dimensional bulk copies from this GPU's global memory into the
// calling CTA's shared memory (cp.async.bulk, the TMA engine's untiled form),
// completed through a shared-memory mbarrier. No multicast: every copy lands
// in the issuing CTA only.
//
// A bulk copy needs a 16-byte aligned source and destination and a size that
// is a multiple of 16 bytes; callers check both. Waits are bounded: after
// kBulkWaitLimit polls the waiter gives up and reports it, so a copy that
// never completes cannot hang the kernel.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace pcg {
namespace {

constexpr uint32_t kBulkWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// one arrival expected per phase (the issuing thread's arrive.expect_tx)
__device__ __forceinline__ void bulk_bar_init(uint64_t* bar) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

// makes the initialised barriers visible to the copy engine; the CTA
// synchronises after it
__device__ __forceinline__ void bulk_bar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// the issuing thread: announce `bytes` for the barrier's current phase and
// start the copy of [src, src + bytes) into dst
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)), "l"(src),
	             "r"(bytes), "r"(smem_u32(bar))
	             : "memory");
}

// waits for the phase with the given parity to complete; false when the
// bounded number of polls ran out first
__device__ __forceinline__ bool bulk_wait(uint64_t* bar, uint32_t parity) {
	for (uint32_t i = 0; i < kBulkWaitLimit; i++) {
		uint32_t done;
		asm volatile(
		    "{\n\t.reg .pred p;\n\t"
		    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		    "selp.u32 %0, 1, 0, p;\n\t}"
		    : "=r"(done)
		    : "r"(smem_u32(bar)), "r"(parity)
		    : "memory");
		if (done) return true;
	}
	return false;
}

}  // namespace
}  // namespace pcg
