// Generic device primitives: stable LSD radix sort of uint32 key/value pairs
// and exclusive prefix sums. Used by the chunk scatter (stable partition of
// points by chunk, chunker_countsort_laszip.cpp:837-904) and by the per-chunk
// counting sort of the octree build (indexer.cpp:874-909).
//
// Radix sort layout: 8-bit digits, tiles of 4096 pairs per 256-thread CTA.
// Within a tile each warp ranks 512 consecutive pairs in 16 striped steps of
// 32 (coalesced loads); ranks come from __match_any_sync peer masks, so the
// order of equal digits is the input order (stable), and warps are combined
// in warp order. Tile offsets per digit come from one exclusive scan over the
// digit-major [256][tiles] count matrix.

#include "dev.h"

namespace pcg {

thread_local int64_t g_launch_count = 0;

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kItemsPerWarpStep = 32;
constexpr int kSteps = 16;
constexpr int kTile = kSortThreads * kSteps;  // 4096
constexpr int kDigits = 256;

__global__ void __launch_bounds__(kSortThreads) radix_upsweep(const uint32_t* __restrict__ keys, int64_t n, int shift,
                                                              uint32_t* __restrict__ counts, int num_tiles) {
	__shared__ uint32_t hist[kDigits];
	for (int i = threadIdx.x; i < kDigits; i += kSortThreads) hist[i] = 0;
	__syncthreads();
	int64_t base = (int64_t)blockIdx.x * kTile;
	for (int k = 0; k < kSteps; k++) {
		int64_t i = base + (int64_t)k * kSortThreads + threadIdx.x;
		if (i < n) atomicAdd(&hist[(keys[i] >> shift) & 0xff], 1u);
	}
	__syncthreads();
	for (int d = threadIdx.x; d < kDigits; d += kSortThreads) counts[(int64_t)d * num_tiles + blockIdx.x] = hist[d];
}

__global__ void __launch_bounds__(kSortThreads) radix_downsweep(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                                                                uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                                                int64_t n, int shift, const uint32_t* __restrict__ offsets, int num_tiles) {
	__shared__ uint32_t warp_hist[kSortWarps][kDigits];
	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;
	for (int i = threadIdx.x; i < kSortWarps * kDigits; i += kSortThreads) (&warp_hist[0][0])[i] = 0;
	__syncthreads();
	const int64_t base = (int64_t)blockIdx.x * kTile + (int64_t)warp * (kSteps * kItemsPerWarpStep);
	uint32_t k_reg[kSteps], v_reg[kSteps], r_reg[kSteps];
	const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
	for (int s = 0; s < kSteps; s++) {
		int64_t i = base + s * kItemsPerWarpStep + lane;
		uint32_t key = 0, val = 0;
		int digit = kDigits;  // sentinel for out-of-range items
		if (i < n) {
			key = keys_in[i];
			val = vals_in[i];
			digit = (key >> shift) & 0xff;
		}
		uint32_t peers = __match_any_sync(0xffffffffu, digit);
		int leader = __ffs(peers) - 1;
		uint32_t before = 0;
		if (digit < kDigits) before = warp_hist[warp][digit];
		uint32_t rank = before + __popc(peers & lt_mask);
		__syncwarp();
		if (lane == leader && digit < kDigits) warp_hist[warp][digit] = before + __popc(peers);
		__syncwarp();
		k_reg[s] = key;
		v_reg[s] = val;
		r_reg[s] = (digit < kDigits) ? rank : 0xffffffffu;
	}
	__syncthreads();
	// exclusive prefix over warps, per digit
	for (int d = threadIdx.x; d < kDigits; d += kSortThreads) {
		uint32_t run = 0;
		for (int w = 0; w < kSortWarps; w++) {
			uint32_t t = warp_hist[w][d];
			warp_hist[w][d] = run + offsets[(int64_t)d * num_tiles + blockIdx.x];
			run += t;
		}
	}
	__syncthreads();
#pragma unroll
	for (int s = 0; s < kSteps; s++) {
		if (r_reg[s] != 0xffffffffu) {
			int digit = (k_reg[s] >> shift) & 0xff;
			uint32_t pos = warp_hist[warp][digit] + r_reg[s];
			keys_out[pos] = k_reg[s];
			vals_out[pos] = v_reg[s];
		}
	}
}

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <class T>
__device__ T block_exclusive_scan(T v, T* smem_warp, T& total) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	T x = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		T y = __shfl_up_sync(0xffffffffu, x, o);
		if (lane >= o) x += y;
	}
	if (lane == 31) smem_warp[warp] = x;
	__syncthreads();
	if (warp == 0) {
		T w = (lane < (int)(blockDim.x >> 5)) ? smem_warp[lane] : T(0);
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			T y = __shfl_up_sync(0xffffffffu, w, o);
			if (lane >= o) w += y;
		}
		if (lane < (int)(blockDim.x >> 5)) smem_warp[lane] = w;
	}
	__syncthreads();
	T warp_prefix = warp > 0 ? smem_warp[warp - 1] : T(0);
	total = smem_warp[(blockDim.x >> 5) - 1];
	__syncthreads();
	return warp_prefix + x - v;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) scan_tiles(const T* __restrict__ in, T* __restrict__ out, int64_t n, T* __restrict__ tile_sums) {
	__shared__ T sw[kScanThreads / 32];
	int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
	T items[kScanItems];
	T sum = 0;
#pragma unroll
	for (int k = 0; k < kScanItems; k++) {
		int64_t i = base + k;
		items[k] = i < n ? in[i] : T(0);
		sum += items[k];
	}
	T total;
	T prefix = block_exclusive_scan<T>(sum, sw, total);
#pragma unroll
	for (int k = 0; k < kScanItems; k++) {
		int64_t i = base + k;
		if (i < n) out[i] = prefix;
		prefix += items[k];
	}
	if (threadIdx.x == 0 && tile_sums) tile_sums[blockIdx.x] = total;
}

template <class T>
__global__ void add_tile_offsets(T* __restrict__ out, int64_t n, const T* __restrict__ tile_offsets) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] += tile_offsets[i / kScanTile];
}

template <class T>
__global__ void write_total(const T* in, const T* out, int64_t n, T* total_at) {
	*total_at = n > 0 ? out[n - 1] + in[n - 1] : T(0);
}

template <class T>
void exclusive_scan_impl(const T* in, T* out, int64_t n, bool write_tot, DeviceMem& mem) {
	cudaStream_t s = mem.stream();
	if (n <= 0) {
		if (write_tot) PCG_CUDA(cudaMemsetAsync(out, 0, sizeof(T), s));
		return;
	}
	int64_t tiles = ceil_div(n, kScanTile);
	if (tiles == 1) {
		scan_tiles<T><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr);
		PCG_LAUNCHED();
	} else {
		T* sums = mem.alloc<T>(tiles);
		T* sums_scan = mem.alloc<T>(tiles);
		scan_tiles<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, sums);
		PCG_LAUNCHED();
		exclusive_scan_impl<T>(sums, sums_scan, tiles, false, mem);
		add_tile_offsets<T><<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(out, n, sums_scan);
		PCG_LAUNCHED();
		mem.free(sums);
		mem.free(sums_scan);
	}
	if (write_tot) {
		write_total<T><<<1, 1, 0, s>>>(in, out, n, out + n);
		PCG_LAUNCHED();
	}
}

}  // namespace

void exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, bool write_tot, DeviceMem& mem) {
	exclusive_scan_impl<uint32_t>(in, out, n, write_tot, mem);
}

void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, bool write_tot, DeviceMem& mem) {
	exclusive_scan_impl<int64_t>(in, out, n, write_tot, mem);
}

void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp, int64_t n,
                      int begin_bit, int end_bit, DeviceMem& mem) {
	if (n <= 1 || end_bit <= begin_bit) return;
	if (n >= (int64_t(1) << 32)) throw PcgError(1, "radix sort: more than 2^32 elements");
	cudaStream_t s = mem.stream();
	int num_tiles = (int)ceil_div(n, kTile);
	uint32_t* counts = mem.alloc<uint32_t>((size_t)kDigits * num_tiles);
	uint32_t* offsets = mem.alloc<uint32_t>((size_t)kDigits * num_tiles);
	uint32_t *ki = keys, *vi = vals, *ko = keys_tmp, *vo = vals_tmp;
	int passes = 0;
	for (int shift = begin_bit; shift < end_bit; shift += 8) {
		radix_upsweep<<<num_tiles, kSortThreads, 0, s>>>(ki, n, shift, counts, num_tiles);
		PCG_LAUNCHED();
		exclusive_scan_u32(counts, offsets, (int64_t)kDigits * num_tiles, false, mem);
		radix_downsweep<<<num_tiles, kSortThreads, 0, s>>>(ki, vi, ko, vo, n, shift, offsets, num_tiles);
		PCG_LAUNCHED();
		std::swap(ki, ko);
		std::swap(vi, vo);
		passes++;
	}
	if (passes & 1) {
		PCG_CUDA(cudaMemcpyAsync(keys, ki, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
		PCG_CUDA(cudaMemcpyAsync(vals, vi, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
	}
	mem.free(counts);
	mem.free(offsets);
}

}  // namespace pcg
