// Warp and block helpers shared by the sampler and sort units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "dev.h"

namespace pcg {
namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ uint32_t lanemask_lt() {
	uint32_t m;
	asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
	return m;
}

constexpr int kWarpsPerBlock = 4;            // warp-per-node kernels: warps per CTA
constexpr int kBigThreads = 512;             // CTA-per-node kernels
constexpr int kBigWarps = kBigThreads / 32;

struct BlockScratch {
	unsigned long long warp_sums[kBigWarps];
	int64_t first_true;
	int64_t bracket;
};

// exclusive scan of a packed (hi:lo) 64-bit count over the CTA
__device__ unsigned long long block_scan_u64(unsigned long long v, unsigned long long& total, BlockScratch& sh) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	unsigned long long x = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		unsigned long long y = __shfl_up_sync(FULL, x, o);
		if (lane >= o) x += y;
	}
	if (lane == 31) sh.warp_sums[warp] = x;
	__syncthreads();
	if (warp == 0) {
		unsigned long long w = lane < kBigWarps ? sh.warp_sums[lane] : 0ull;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			unsigned long long y = __shfl_up_sync(FULL, w, o);
			if (lane >= o) w += y;
		}
		if (lane < kBigWarps) sh.warp_sums[lane] = w;
	}
	__syncthreads();
	unsigned long long before = warp > 0 ? sh.warp_sums[warp - 1] : 0ull;
	total = sh.warp_sums[kBigWarps - 1];
	__syncthreads();
	return before + x - v;
}

// multiprocessors of the current device
inline int sm_count() {
	int dev = 0, sms = 0;
	PCG_CUDA(cudaGetDevice(&dev));
	PCG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
	return sms;
}

}  // namespace
}  // namespace pcg
