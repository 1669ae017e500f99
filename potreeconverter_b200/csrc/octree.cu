// Per-chunk octree build on the device (buildHierarchy, indexer.cpp:823-1109).
//
// One round processes every node that must be split, across all chunks at
// once: each point gets the Morton code of its 32^3 cell inside its node's
// box (indexer.cpp:851-871), the round's points are stably sorted by
// (node, Morton code) -- the reference's stable counting sort
// (indexer.cpp:874-909) -- and one CTA per node builds the 5-level sum
// pyramid in shared memory and walks it (createSumPyramid / createNodes,
// indexer.cpp:691-817), emitting leaves and nodes that need another round.

#include "kernels.h"

namespace pcg {

namespace {

__device__ __forceinline__ uint32_t split_by_3_small(uint32_t a) {  // 5-bit input, converter_utils.h:89-101
	uint32_t x = a & 0x1f;
	x = (x | (x << 8)) & 0x0000F00Fu;
	x = (x | (x << 4)) & 0x000C30C3u;
	x = (x | (x << 2)) & 0x00249249u;
	return x;
}

// mortonEncode_magicbits(z, y, x): z -> bit 0, y -> bit 1, x -> bit 2
__device__ __forceinline__ uint32_t morton15(uint32_t ix, uint32_t iy, uint32_t iz) {
	return split_by_3_small(iz) | (split_by_3_small(iy) << 1) | (split_by_3_small(ix) << 2);
}

__device__ __forceinline__ int find_segment(const SegmentDesc* segs, int num, int64_t j) {
	int lo = 0, hi = num - 1;
	while (lo < hi) {
		int mid = (lo + hi + 1) >> 1;
		if (segs[mid].coff <= j) lo = mid; else hi = mid - 1;
	}
	return lo;
}

__global__ void octree_keys_kernel(const uint32_t* __restrict__ ids, const int32_t* __restrict__ X, const int32_t* __restrict__ Y,
                                   const int32_t* __restrict__ Z, PosParams pp, const SegmentDesc* __restrict__ segs, int num_segs,
                                   int64_t total, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
	int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= total) return;
	int s = find_segment(segs, num_segs, j);
	const SegmentDesc& d = segs[s];
	uint32_t id = ids[d.start + (j - d.coff)];
	double x = ((double)X[id] * pp.scale[0]) + pp.offset[0];
	double y = ((double)Y[id] * pp.scale[1]) + pp.offset[1];
	double z = ((double)Z[id] * pp.scale[2]) + pp.offset[2];
	int64_t ix = (int64_t)(32.0 * (x - d.min[0]) / d.size[0]);
	int64_t iy = (int64_t)(32.0 * (y - d.min[1]) / d.size[1]);
	int64_t iz = (int64_t)(32.0 * (z - d.min[2]) / d.size[2]);
	ix = ix < 0 ? 0 : (ix > 31 ? 31 : ix);
	iy = iy < 0 ? 0 : (iy > 31 ? 31 : iy);
	iz = iz < 0 ? 0 : (iz > 31 ? 31 : iz);
	keys[j] = ((uint32_t)s << 15) | morton15((uint32_t)ix, (uint32_t)iy, (uint32_t)iz);
	vals[j] = id;
}

__global__ void octree_scatter_kernel(uint32_t* __restrict__ ids, const uint32_t* __restrict__ vals, const SegmentDesc* __restrict__ segs,
                                      int num_segs, int64_t total) {
	int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= total) return;
	int s = find_segment(segs, num_segs, j);
	ids[segs[s].start + (j - segs[s].coff)] = vals[j];
}

constexpr int kNodesThreads = 1024;
constexpr int kCells = 32768;                 // 32^3
constexpr int kPyr = 1 + 8 + 64 + 512 + 4096; // levels 0..4

// One CTA per segment: histogram of the segment's (sorted) Morton codes,
// sum pyramid, exclusive prefix of level 5 (= start of every cell in the
// sorted range), then the createNodes depth-first walk on one thread.
__global__ void __launch_bounds__(kNodesThreads) octree_nodes_kernel(const uint32_t* __restrict__ keys, const SegmentDesc* __restrict__ segs,
                                                                    NodeCand* __restrict__ cands, int32_t* __restrict__ num_cands,
                                                                    int64_t capacity) {
	extern __shared__ uint32_t smem[];
	uint32_t* cnt = smem;                 // level 5 counts, then exclusive prefix
	uint32_t* pyr = smem + kCells;        // levels 0..4, Morton layout, level l at pyr_base(l)
	__shared__ uint32_t warp_sums[32];
	__shared__ uint32_t total_s;
	const int seg = blockIdx.x;
	const SegmentDesc d = segs[seg];
	for (int i = threadIdx.x; i < kCells; i += blockDim.x) cnt[i] = 0;
	__syncthreads();
	for (int64_t j = threadIdx.x; j < d.count; j += blockDim.x) atomicAdd(&cnt[keys[d.coff + j] & 0x7fff], 1u);
	__syncthreads();
	// level 4 from level 5, then upwards (createSumPyramid)
	const int base4 = 1 + 8 + 64 + 512, base3 = 1 + 8 + 64, base2 = 1 + 8, base1 = 1, base0 = 0;
	for (int m = threadIdx.x; m < 4096; m += blockDim.x) {
		uint32_t s = 0;
		for (int k = 0; k < 8; k++) s += cnt[8 * m + k];
		pyr[base4 + m] = s;
	}
	__syncthreads();
	for (int m = threadIdx.x; m < 512; m += blockDim.x) {
		uint32_t s = 0;
		for (int k = 0; k < 8; k++) s += pyr[base4 + 8 * m + k];
		pyr[base3 + m] = s;
	}
	__syncthreads();
	if (threadIdx.x < 64) {
		uint32_t s = 0;
		for (int k = 0; k < 8; k++) s += pyr[base3 + 8 * threadIdx.x + k];
		pyr[base2 + threadIdx.x] = s;
	}
	__syncthreads();
	if (threadIdx.x < 8) {
		uint32_t s = 0;
		for (int k = 0; k < 8; k++) s += pyr[base2 + 8 * threadIdx.x + k];
		pyr[base1 + threadIdx.x] = s;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		uint32_t s = 0;
		for (int k = 0; k < 8; k++) s += pyr[base1 + k];
		pyr[base0] = s;
	}
	__syncthreads();
	// exclusive prefix of level 5 in place: 1024 threads x 32 cells
	{
		const int per = kCells / kNodesThreads;
		uint32_t local = 0;
		for (int k = 0; k < per; k++) local += cnt[threadIdx.x * per + k];
		uint32_t x = local;
		const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
		for (int o = 1; o < 32; o <<= 1) {
			uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
			if (lane >= o) x += y;
		}
		if (lane == 31) warp_sums[warp] = x;
		__syncthreads();
		if (warp == 0) {
			uint32_t w = warp_sums[lane];
			for (int o = 1; o < 32; o <<= 1) {
				uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
				if (lane >= o) w += y;
			}
			warp_sums[lane] = w;
			if (lane == 31) total_s = w;
		}
		__syncthreads();
		uint32_t run = (warp > 0 ? warp_sums[warp - 1] : 0) + x - local;
		for (int k = 0; k < per; k++) {
			uint32_t c = cnt[threadIdx.x * per + k];
			cnt[threadIdx.x * per + k] = run;
			run += c;
		}
	}
	__syncthreads();
	if (threadIdx.x != 0) return;
	const uint32_t total = total_s;
	auto count_at = [&](int level, int m) -> uint32_t {
		if (level == 5) return (m + 1 < kCells ? cnt[m + 1] : total) - cnt[m];
		const int bases[5] = {base0, base1, base2, base3, base4};
		return pyr[bases[level] + m];
	};
	auto emit = [&](int level, int path, int m) {
		int k = atomicAdd(num_cands, 1);
		if (k < capacity) {
			NodeCand c;
			c.seg = seg;
			c.level = level;
			c.path = path;
			c.pad = 0;
			c.start = cnt[m << (3 * (5 - level))];
			c.count = count_at(level, m);
			cands[k] = c;
		}
	};
	// depth-first walk (createNodes); m = Morton index at `level`
	struct Item { int level, path, m; };
	Item stack[64];
	int sp = 0;
	stack[sp++] = {0, 0, 0};
	while (sp > 0) {
		Item it = stack[--sp];
		uint32_t n = count_at(it.level, it.m);
		if (it.level == 5) {
			if (n > 0) emit(it.level, it.path, it.m);
		} else if (n > 10000u) {
			for (int i = 0; i < 8; i++) {
				int cm = it.m * 8 + i;
				if (count_at(it.level + 1, cm) > 0) stack[sp++] = {it.level + 1, (it.path << 3) | i, cm};
			}
		} else if (n > 0) {
			emit(it.level, it.path, it.m);
		}
	}
}

// ---- distinct positions of a range (duplicate handling, indexer.cpp:1002-1099)
__global__ void gather_coord_kernel(const uint32_t* __restrict__ ids, int64_t n, const int32_t* __restrict__ C,
                                    const uint32_t* __restrict__ order, uint32_t* __restrict__ key) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) key[i] = (uint32_t)C[ids[order[i]]] ^ 0x80000000u;
}

__global__ void iota_kernel(uint32_t* v, int64_t n) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) v[i] = (uint32_t)i;
}

__global__ void count_distinct_kernel(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ order, int64_t n,
                                      const int32_t* __restrict__ X, const int32_t* __restrict__ Y, const int32_t* __restrict__ Z,
                                      unsigned long long* out) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	uint32_t a = ids[order[i]];
	bool distinct = true;
	if (i > 0) {
		uint32_t b = ids[order[i - 1]];
		distinct = X[a] != X[b] || Y[a] != Y[b] || Z[a] != Z[b];
	}
	if (distinct) atomicAdd(out, 1ull);
}

}  // namespace

void launch_octree_round(uint32_t* ids, const int32_t* X, const int32_t* Y, const int32_t* Z, const PosParams& pp,
                         const SegmentDesc* d_segs, int num_segs, int64_t total, NodeCand* cands, int32_t* num_cands,
                         int64_t cand_capacity, DeviceMem& mem) {
	if (total == 0 || num_segs == 0) return;
	if (num_segs >= (1 << 17)) throw PcgError(5, "octree round: too many segments");
	cudaStream_t s = mem.stream();
	uint32_t* keys = mem.alloc<uint32_t>(total);
	uint32_t* vals = mem.alloc<uint32_t>(total);
	uint32_t* keys_t = mem.alloc<uint32_t>(total);
	uint32_t* vals_t = mem.alloc<uint32_t>(total);
	unsigned blocks = (unsigned)ceil_div(total, 256);
	octree_keys_kernel<<<blocks, 256, 0, s>>>(ids, X, Y, Z, pp, d_segs, num_segs, total, keys, vals);
	PCG_LAUNCHED();
	int bits = 15 + bits_for((uint64_t)(num_segs - 1));
	radix_sort_pairs(keys, vals, keys_t, vals_t, total, 0, bits, mem);
	octree_scatter_kernel<<<blocks, 256, 0, s>>>(ids, vals, d_segs, num_segs, total);
	PCG_LAUNCHED();
	size_t smem = (size_t)(kCells + kPyr) * sizeof(uint32_t);
	PCG_CUDA(cudaFuncSetAttribute(octree_nodes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	octree_nodes_kernel<<<num_segs, kNodesThreads, smem, s>>>(keys, d_segs, cands, num_cands, cand_capacity);
	PCG_LAUNCHED();
	mem.free(keys);
	mem.free(vals);
	mem.free(keys_t);
	mem.free(vals_t);
}

int64_t count_unique_positions(const uint32_t* ids, int64_t n, const int32_t* X, const int32_t* Y, const int32_t* Z, DeviceMem& mem) {
	if (n <= 1) return n;
	cudaStream_t s = mem.stream();
	uint32_t* order = mem.alloc<uint32_t>(n);
	uint32_t* key = mem.alloc<uint32_t>(n);
	uint32_t* order_t = mem.alloc<uint32_t>(n);
	uint32_t* key_t = mem.alloc<uint32_t>(n);
	unsigned long long* cnt = mem.alloc<unsigned long long>(1);
	unsigned blocks = (unsigned)ceil_div(n, 256);
	iota_kernel<<<blocks, 256, 0, s>>>(order, n);
	PCG_LAUNCHED();
	const int32_t* coords[3] = {Z, Y, X};  // least significant first
	for (int c = 0; c < 3; c++) {
		gather_coord_kernel<<<blocks, 256, 0, s>>>(ids, n, coords[c], order, key);
		PCG_LAUNCHED();
		radix_sort_pairs(key, order, key_t, order_t, n, 0, 32, mem);
	}
	PCG_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
	count_distinct_kernel<<<blocks, 256, 0, s>>>(ids, order, n, X, Y, Z, cnt);
	PCG_LAUNCHED();
	unsigned long long h = 0;
	PCG_CUDA(cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s));
	PCG_CUDA(cudaStreamSynchronize(s));
	mem.free(order); mem.free(key); mem.free(order_t); mem.free(key_t); mem.free(cnt);
	return (int64_t)h;
}

}  // namespace pcg
