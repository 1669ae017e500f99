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

// The LAS record's coordinates requantized to the octree's integer grid:
// laszip_get_coordinates (laszip_dll.cpp:1137-1139), then the chunker's
// quantization (chunker_countsort_laszip.cpp:228-230, 781-783). Every kernel
// that needs the integer coordinates of a record uses this one expression.
__device__ __forceinline__ void quantize_record(const DecodeParams& p, const uint8_t* r, double& x, double& y, double& z, int32_t& X,
                                                int32_t& Y, int32_t& Z) {
	int32_t Xi, Yi, Zi;
	memcpy(&Xi, r, 4);
	memcpy(&Yi, r + 4, 4);
	memcpy(&Zi, r + 8, 4);
	x = p.in_scale[0] * (double)Xi + p.in_offset[0];
	y = p.in_scale[1] * (double)Yi + p.in_offset[1];
	z = p.in_scale[2] * (double)Zi + p.in_offset[2];
	X = (int32_t)((x - p.pos_offset[0]) / p.pos_scale[0]);
	Y = (int32_t)((y - p.pos_offset[1]) / p.pos_scale[1]);
	Z = (int32_t)((z - p.pos_offset[2]) / p.pos_scale[2]);
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
