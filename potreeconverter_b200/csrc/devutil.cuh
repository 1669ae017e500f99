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
// laszip_get_coordinates with the record's own source scale and offset
// (laszip_dll.cpp:1137-1139), then the chunker's quantization with the
// job's scale and offset (chunker_countsort_laszip.cpp:228-230, 781-783).
// Every kernel that needs the integer coordinates of a record uses this one
// expression.
__device__ __forceinline__ void quantize_record(const DecodeParams& p, const SourceDesc& sd, const uint8_t* r, double& x, double& y,
                                                double& z, int32_t& X, int32_t& Y, int32_t& Z) {
	int32_t Xi, Yi, Zi;
	memcpy(&Xi, r, 4);
	memcpy(&Yi, r + 4, 4);
	memcpy(&Zi, r + 8, 4);
	x = sd.in_scale[0] * (double)Xi + sd.in_offset[0];
	y = sd.in_scale[1] * (double)Yi + sd.in_offset[1];
	z = sd.in_scale[2] * (double)Zi + sd.in_offset[2];
	X = (int32_t)((x - p.pos_offset[0]) / p.pos_scale[0]);
	Y = (int32_t)((y - p.pos_offset[1]) / p.pos_scale[1]);
	Z = (int32_t)((z - p.pos_offset[2]) / p.pos_scale[2]);
}

// Source of job point i: the last source whose first point is at or before
// i (empty sources share their first index with the next one and are
// skipped). first[0] == 0.
__device__ __forceinline__ int find_source(const int64_t* __restrict__ first, int nsrc, int64_t i) {
	int lo = 0, hi = nsrc - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (__ldg(first + mid) <= i) lo = mid;
		else hi = mid - 1;
	}
	return lo;
}

// Calls f(source descriptor) for job point i: the kernel's own parameter for
// one-source jobs, the device table otherwise.
template <bool kMulti, class F>
__device__ __forceinline__ void with_source(const DecodeParams& p, int64_t i, F&& f) {
	if constexpr (kMulti) f(p.srcs[find_source(p.src_first, p.nsrc, i)]);
	else f(p.src0);
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
