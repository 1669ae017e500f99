// Exact per-node sort of a level's candidate keys without the introsort
// replay.
//
// The samplers order each node's candidates with std::sort by FP64 squared
// distance to the node centre (sampler_poisson.h:183-203). When a node's keys
// are pairwise distinct, the ascending order is unique, so any exact sort
// yields the permutation std::sort yields. Only nodes with equal keys need
// the element-for-element introsort replay of sampling.cu, because there the
// order among equal keys is an artefact of the partitions.
//
// This unit sorts every node of a level at once with a segmented LSD radix
// sort of the high 32 key bits (keys are finite and >= +0, so their IEEE bit
// patterns order like the values), puts each short run of equal high words
// in full-key order in place (a node with a run longer than 32 gets all 64
// bits by radix instead), then flags the nodes that hold two equal adjacent
// keys. Segmentation comes from the tiling: tiles never straddle a
// node, and the per-tile digit counts are laid out node-major, digit-major,
// tile-minor, so one flat exclusive scan of the count matrix yields, for
// every (node, digit, tile), the output position inside the node's own range
// [cand_off, cand_off + count). Elements therefore never leave their node, and
// no pass over the node index is needed.
//
// A pass reads 12 bytes (key, value) and writes 12 bytes per candidate; the
// counting pass reads the 8-byte key. Within a tile, ranks come from
// __match_any_sync peer masks in warp order (stable), the tile is reordered in
// shared memory, and each digit's run is written out contiguously.

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "devutil.cuh"
#include "sampling.h"

namespace pcg {

namespace {

constexpr int kSegThreads = 256;
constexpr int kSegWarps = kSegThreads / 32;
// 2048-element tiles: the downsweep keeps a tile's keys, values and ranks in
// registers, and at 8 per thread it fits 64 registers, four blocks per SM
// (16 per thread took 106 registers, two blocks, and waited on memory)
constexpr int kSegSteps = 8;
constexpr int kSegTile = kSegThreads * kSegSteps;  // 2048
constexpr int kSegDigits = 256;
static_assert(kSegThreads == kSegDigits, "one thread per digit");

struct SegTile {
	int64_t start;     // first candidate (level-wide index)
	int64_t node_off;  // cand_off of the tile's node
	int64_t adjust;    // node_off minus the candidates of the nodes before it in the count matrix
	int64_t cnt_base;  // count-matrix index of (digit 0, this tile)
	int32_t count;     // candidates in the tile, <= kSegTile
	int32_t stride;    // tiles of the node = count-matrix stride between digits
};

struct SegShared {
	uint64_t key[kSegTile];
	uint32_t val[kSegTile];
	uint32_t whist[kSegWarps][kSegDigits];
	int64_t gbase[kSegDigits];
	uint32_t wsum[kSegWarps];
};

__global__ void __launch_bounds__(kSegThreads) seg_upsweep(const SegTile* __restrict__ tiles, const uint64_t* __restrict__ keys, int shift,
                                                         uint32_t* __restrict__ counts) {
	__shared__ uint32_t hist[kSegDigits];
	const SegTile t = tiles[blockIdx.x];
	hist[threadIdx.x] = 0;
	__syncthreads();
	const int lane = threadIdx.x & 31;
	for (int base = 0; base < t.count; base += kSegThreads) {
		const int i = base + (int)threadIdx.x;
		const int digit = i < t.count ? (int)((keys[t.start + i] >> shift) & 0xff) : kSegDigits;
		const uint32_t peers = __match_any_sync(FULL, digit);
		if (digit < kSegDigits && lane == __ffs(peers) - 1) atomicAdd(&hist[digit], (uint32_t)__popc(peers));
	}
	__syncthreads();
	counts[t.cnt_base + (int64_t)threadIdx.x * t.stride] = hist[threadIdx.x];
}

// vals_in == nullptr: first pass, the value is the candidate's index in its node
__global__ void __launch_bounds__(kSegThreads, 4) seg_downsweep(const SegTile* __restrict__ tiles, const uint64_t* __restrict__ keys_in,
                                                           const uint32_t* __restrict__ vals_in, uint64_t* __restrict__ keys_out,
                                                           uint32_t* __restrict__ vals_out, int shift, const uint32_t* __restrict__ offsets) {
	extern __shared__ __align__(16) unsigned char seg_smem[];
	SegShared& sh = *reinterpret_cast<SegShared*>(seg_smem);
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const SegTile t = tiles[blockIdx.x];
	for (int i = tid; i < kSegWarps * kSegDigits; i += kSegThreads) (&sh.whist[0][0])[i] = 0;
	__syncthreads();
	uint64_t kr[kSegSteps];
	uint32_t vr[kSegSteps], rr[kSegSteps];
	const uint32_t lt = lanemask_lt();
#pragma unroll
	for (int s = 0; s < kSegSteps; s++) {
		const int li = warp * (kSegSteps * 32) + s * 32 + lane;
		uint64_t key = 0;
		uint32_t val = 0;
		int digit = kSegDigits;  // sentinel past the tile's end
		if (li < t.count) {
			const int64_t p = t.start + li;
			key = keys_in[p];
			val = vals_in ? vals_in[p] : (uint32_t)(p - t.node_off);
			digit = (int)((key >> shift) & 0xff);
		}
		const uint32_t peers = __match_any_sync(FULL, digit);
		uint32_t before = digit < kSegDigits ? sh.whist[warp][digit] : 0u;
		__syncwarp();
		if (digit < kSegDigits && lane == __ffs(peers) - 1) sh.whist[warp][digit] = before + __popc(peers);
		__syncwarp();
		kr[s] = key;
		vr[s] = val;
		rr[s] = digit < kSegDigits ? before + __popc(peers & lt) : 0xffffffffu;
	}
	__syncthreads();
	// thread d owns digit d: warp offsets, then the tile-local digit base
	const int d = tid;
	uint32_t run = 0;
#pragma unroll
	for (int w = 0; w < kSegWarps; w++) {
		uint32_t c = sh.whist[w][d];
		sh.whist[w][d] = run;
		run += c;
	}
	uint32_t x = run;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		uint32_t y = __shfl_up_sync(FULL, x, o);
		if (lane >= o) x += y;
	}
	if (lane == 31) sh.wsum[warp] = x;
	__syncthreads();
	uint32_t wbefore = 0;
	for (int w = 0; w < warp; w++) wbefore += sh.wsum[w];
	const uint32_t lbase = wbefore + x - run;  // exclusive over digits
#pragma unroll
	for (int w = 0; w < kSegWarps; w++) sh.whist[w][d] += lbase;
	sh.gbase[d] = t.adjust + (int64_t)offsets[t.cnt_base + (int64_t)d * t.stride] - (int64_t)lbase;
	__syncthreads();
#pragma unroll
	for (int s = 0; s < kSegSteps; s++) {
		if (rr[s] != 0xffffffffu) {
			const int digit = (int)((kr[s] >> shift) & 0xff);
			const uint32_t L = sh.whist[warp][digit] + rr[s];
			sh.key[L] = kr[s];
			sh.val[L] = vr[s];
		}
	}
	__syncthreads();
	for (int L = tid; L < t.count; L += kSegThreads) {
		const uint64_t key = sh.key[L];
		const int64_t pos = sh.gbase[(key >> shift) & 0xff] + L;
		keys_out[pos] = key;
		vals_out[pos] = sh.val[L];
	}
}

// After a sort on the high 32 key bits: every run of equal high words is
// put in full-key order by its first element's thread (stable insertion
// sort). Runs longer than kLowRunMax flag their node (bit 1) for a full sort.
constexpr int kLowRunMax = 32;

__global__ void seg_fix_low_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ node_of, uint64_t* __restrict__ sk,
                                   uint32_t* __restrict__ sv, int64_t M, uint8_t* __restrict__ flags) {
	const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= M) return;
	const int32_t n = node_of[t];
	const int64_t co = nodes[n].cand_off, end = co + nodes[n].count;
	const uint64_t hi = sk[t] >> 32;
	if (t > co && (sk[t - 1] >> 32) == hi) return;  // not the first of its run
	int64_t e = t + 1;
	while (e < end && (sk[e] >> 32) == hi) {
		e++;
		if (e - t > kLowRunMax) {
			flags[n] |= 2;
			return;
		}
	}
	for (int64_t i = t + 1; i < e; i++) {
		const uint64_t k = sk[i];
		const uint32_t v = sv[i];
		int64_t j = i;
		while (j > t && k < sk[j - 1]) {
			sk[j] = sk[j - 1];
			sv[j] = sv[j - 1];
			j--;
		}
		sk[j] = k;
		sv[j] = v;
	}
}

__global__ void seg_ties_kernel(const int32_t* __restrict__ node_of, const uint64_t* __restrict__ sk, int64_t M, uint8_t* __restrict__ tie) {
	const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (t + 1 >= M) return;
	const int32_t n = node_of[t];
	if (node_of[t + 1] == n && sk[t] == sk[t + 1]) tie[n] |= 1;
}

__global__ void seg_finish_kernel(const LevelNode* __restrict__ nodes, const uint8_t* __restrict__ tie, const uint64_t* __restrict__ sk,
                                  const uint32_t* __restrict__ sv, LevelBuffers lb) {
	const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= lb.M) return;
	const int32_t n = lb.node_of[t];
	if (tie[n]) return;  // left to the introsort replay
	const int64_t off = nodes[n].cand_off;
	const uint32_t local = sv[t];
	lb.keys[t] = __longlong_as_double((long long)sk[t]);
	lb.perm[t] = (int32_t)local;
	lb.pos[off + local] = (int32_t)(t - off);
}

}  // namespace

void segmented_sort_pairs(const std::vector<LevelNode>& ln, int64_t M, const uint64_t* keys_in, const uint32_t* vals_in,
                          uint64_t* keys_out, uint32_t* vals_out, int begin_bit, int end_bit, DeviceMem& mem) {
	const int K = (int)ln.size();
	if (M == 0 || K == 0 || end_bit <= begin_bit) return;
	cudaStream_t s = mem.stream();
	std::vector<SegTile> tiles;
	int64_t mat = 0, before = 0;
	for (int k = 0; k < K; k++) {
		const int64_t n = ln[k].count;
		if (n == 0) continue;
		const int64_t T = ceil_div(n, kSegTile);
		if (T > INT32_MAX / kSegDigits) throw PcgError(5, "segmented sort: node too large");
		for (int64_t i = 0; i < T; i++) {
			SegTile st;
			st.start = ln[k].cand_off + i * kSegTile;
			st.node_off = ln[k].cand_off;
			st.adjust = ln[k].cand_off - before;
			st.cnt_base = mat + i;
			st.count = (int32_t)std::min<int64_t>(kSegTile, n - i * kSegTile);
			st.stride = (int32_t)T;
			tiles.push_back(st);
		}
		mat += (int64_t)kSegDigits * T;
		before += n;
	}
	const int num_tiles = (int)tiles.size();
	const int passes = (end_bit - begin_bit + 7) / 8;
	SegTile* d_tiles = mem.alloc<SegTile>(tiles.size());
	PCG_CUDA(cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * sizeof(SegTile), cudaMemcpyHostToDevice, s));
	// the last pass writes (keys_out, vals_out)
	uint64_t* kb[2] = {keys_out, passes > 1 ? mem.alloc<uint64_t>(M) : nullptr};
	uint32_t* vb[2] = {vals_out, passes > 1 ? mem.alloc<uint32_t>(M) : nullptr};
	uint32_t* counts = mem.alloc<uint32_t>(mat);
	uint32_t* offsets = mem.alloc<uint32_t>(mat);
	static_assert(sizeof(SegShared) <= 227 * 1024, "tile does not fit shared memory");
	PCG_CUDA(cudaFuncSetAttribute(seg_downsweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SegShared)));
	const uint64_t* kin = keys_in;
	const uint32_t* vin = vals_in;
	for (int pass = 0; pass < passes; pass++) {
		const int shift = begin_bit + 8 * pass;
		const int dst = (passes - 1 - pass) & 1;
		uint64_t* kout = kb[dst];
		uint32_t* vout = vb[dst];
		seg_upsweep<<<num_tiles, kSegThreads, 0, s>>>(d_tiles, kin, shift, counts);
		PCG_LAUNCHED();
		exclusive_scan_u32(counts, offsets, mat, false, mem);
		seg_downsweep<<<num_tiles, kSegThreads, sizeof(SegShared), s>>>(d_tiles, kin, vin, kout, vout, shift, offsets);
		PCG_LAUNCHED();
		kin = kout;
		vin = vout;
	}
	mem.free(counts);
	mem.free(offsets);
	if (kb[1]) mem.free(kb[1]);
	if (vb[1]) mem.free(vb[1]);
	mem.free(d_tiles);
}

namespace {

// ties[j]: adjacent equal keys of j's node up to j (inclusive prefix of
// "sk[j] equals its predecessor in the node")
__global__ void seg_tie_flags_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ node_of, const uint64_t* __restrict__ sk,
                                     int64_t M, uint32_t* __restrict__ flags) {
	const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= M) return;
	flags[t] = t > nodes[node_of[t]].cand_off && sk[t] == sk[t - 1] ? 1u : 0u;
}

__global__ void seg_inclusive_kernel(const uint32_t* __restrict__ flags, const uint32_t* __restrict__ excl, int64_t M, int32_t* __restrict__ incl) {
	const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (t < M) incl[t] = (int32_t)(excl[t] + flags[t]);
}

}  // namespace

void build_sorted_level(const LevelNode* d_nodes, const std::vector<LevelNode>& ln, const int32_t* node_of, const uint64_t* keys, int64_t M,
                        SortedLevel& out, DeviceMem& mem) {
	out = SortedLevel{};
	if (M == 0) return;
	cudaStream_t s = mem.stream();
	uint64_t* sk = mem.alloc<uint64_t>(M);
	uint32_t* sv = mem.alloc<uint32_t>(M);
	segmented_sort_pairs(ln, M, keys, nullptr, sk, sv, 0, 64, mem);
	const unsigned blocks = (unsigned)ceil_div(M, 256);
	uint32_t* f = mem.alloc<uint32_t>(M);
	uint32_t* ex = mem.alloc<uint32_t>(M);
	int32_t* ties = mem.alloc<int32_t>(M);
	seg_tie_flags_kernel<<<blocks, 256, 0, s>>>(d_nodes, node_of, sk, M, f);
	PCG_LAUNCHED();
	exclusive_scan_u32(f, ex, M, false, mem);
	seg_inclusive_kernel<<<blocks, 256, 0, s>>>(f, ex, M, ties);
	PCG_LAUNCHED();
	mem.free(ex);
	mem.free(f);
	out.sk = sk;
	out.sv = sv;
	out.ties = ties;
	out.node_of = node_of;
	out.nodes = d_nodes;
	out.owned[0] = sk;
	out.owned[1] = sv;
	out.owned[2] = ties;
}

void free_sorted_level(SortedLevel& keep, DeviceMem& mem) {
	for (void*& p : keep.owned)
		if (p) { mem.free(p); p = nullptr; }
	keep = SortedLevel{};
}

void sort_level_distinct(const LevelNode* d_nodes, const std::vector<LevelNode>& ln, LevelBuffers& lb, DeviceMem& mem,
                         std::vector<uint8_t>& tie, SortedLevel* keep) {
	const int K = (int)ln.size();
	const int64_t M = lb.M;
	tie.assign(K, 0);
	if (M == 0 || K == 0) return;
	cudaStream_t s = mem.stream();
	uint64_t* sk = mem.alloc<uint64_t>(M);
	uint32_t* sv = mem.alloc<uint32_t>(M);
	const uint64_t* keys = reinterpret_cast<const uint64_t*>(lb.keys);
	// the high words by radix (four passes), the low words inside the short
	// runs of equal high words
	segmented_sort_pairs(ln, M, keys, nullptr, sk, sv, 32, 64, mem);
	uint8_t* d_flags = mem.alloc<uint8_t>(K);
	PCG_CUDA(cudaMemsetAsync(d_flags, 0, K, s));
	const unsigned blocks = (unsigned)ceil_div(M, 256);
	seg_fix_low_kernel<<<blocks, 256, 0, s>>>(d_nodes, lb.node_of, sk, sv, M, d_flags);
	PCG_LAUNCHED();
	std::vector<uint8_t> flags(K);
	PCG_CUDA(cudaMemcpyAsync(flags.data(), d_flags, K, cudaMemcpyDeviceToHost, s));
	PCG_CUDA(cudaStreamSynchronize(s));
	std::vector<LevelNode> redo;
	for (int k = 0; k < K; k++)
		if (flags[k] & 2) redo.push_back(ln[k]);
	// nodes with a long run of equal high words: all 64 bits by radix
	if (!redo.empty()) segmented_sort_pairs(redo, M, keys, nullptr, sk, sv, 0, 64, mem);
	PCG_CUDA(cudaMemsetAsync(d_flags, 0, K, s));
	seg_ties_kernel<<<blocks, 256, 0, s>>>(lb.node_of, sk, M, d_flags);
	PCG_LAUNCHED();
	seg_finish_kernel<<<blocks, 256, 0, s>>>(d_nodes, d_flags, sk, sv, lb);
	PCG_LAUNCHED();
	PCG_CUDA(cudaMemcpyAsync(tie.data(), d_flags, K, cudaMemcpyDeviceToHost, s));
	PCG_CUDA(cudaStreamSynchronize(s));
	mem.free(d_flags);
	bool any_tie = false;
	for (uint8_t t : tie) any_tie |= t != 0;
	if (keep && any_tie) {
		uint32_t* f = mem.alloc<uint32_t>(M);
		uint32_t* ex = mem.alloc<uint32_t>(M);
		int32_t* ties = mem.alloc<int32_t>(M);
		seg_tie_flags_kernel<<<blocks, 256, 0, s>>>(d_nodes, lb.node_of, sk, M, f);
		PCG_LAUNCHED();
		exclusive_scan_u32(f, ex, M, false, mem);
		seg_inclusive_kernel<<<blocks, 256, 0, s>>>(f, ex, M, ties);
		PCG_LAUNCHED();
		mem.free(ex);
		mem.free(f);
		*keep = SortedLevel{};
		keep->sk = sk;
		keep->sv = sv;
		keep->ties = ties;
		keep->node_of = lb.node_of;
		keep->nodes = d_nodes;
		keep->owned[0] = sk;
		keep->owned[1] = sv;
		keep->owned[2] = ties;
		return;
	}
	mem.free(sk);
	mem.free(sv);
}

}  // namespace pcg
