// The std::sort replay: libstdc++'s introsort (sampler_poisson.h:183-203 sorts
// the candidates with std::sort by squared distance to the node centre),
// reproduced element for element for keys that may compare equal.
//
//  * warp_partition / block_partition -- one Hoare partition after the
//    median-of-three pivot move. Hoare's pairing of the k-th left stop with
//    the k-th right stop is computed from stop ranks (ballot/popc or a block
//    scan), so a partition is two coalesced passes instead of a sequential
//    two-pointer walk.
//  * warp_introsort / block_std_sort -- std::__introsort_loop with its
//    depth budget and heapsort fallback (std::__partial_sort); the final
//    insertion sort is a stable sort of each <=16-element block the loop
//    leaves behind.
//  * node_sort_kernel (a warp per node) and node_sort_big_kernel (a CTA per
//    node) run the replay for the nodes of one octree level.

#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <limits>

#include "devutil.cuh"
#include "sampling.h"

namespace pcg {

namespace {

// ------------------------------------------------------ std::sort replay
struct SortScratch {
	int32_t* SL;   // [M] left stop positions
	int32_t* SR;   // [M] right stop positions
	int32_t* blk;  // [2M] final blocks (start, end)
};

__device__ void heap_adjust(double* key, int32_t* val, int64_t hole, int64_t len, double vk, int32_t vv) {
	// std::__adjust_heap followed by std::__push_heap (stl_heap.h)
	const int64_t top = hole;
	int64_t second = hole;
	while (second < (len - 1) / 2) {
		second = 2 * (second + 1);
		if (key[second] < key[second - 1]) second--;
		key[hole] = key[second];
		val[hole] = val[second];
		hole = second;
	}
	if ((len & 1) == 0 && second == (len - 2) / 2) {
		second = 2 * (second + 1);
		key[hole] = key[second - 1];
		val[hole] = val[second - 1];
		hole = second - 1;
	}
	int64_t parent = (hole - 1) / 2;
	while (hole > top && key[parent] < vk) {
		key[hole] = key[parent];
		val[hole] = val[parent];
		hole = parent;
		parent = (hole - 1) / 2;
	}
	key[hole] = vk;
	val[hole] = vv;
}

// std::__partial_sort(first, last, last): make_heap + sort_heap
__device__ void heap_sort(double* key, int32_t* val, int64_t len) {
	if (len >= 2) {
		int64_t parent = (len - 2) / 2;
		while (true) {
			heap_adjust(key, val, parent, len, key[parent], val[parent]);
			if (parent == 0) break;
			parent--;
		}
	}
	int64_t last = len;
	while (last > 1) {
		--last;
		double vk = key[last];
		int32_t vv = val[last];
		key[last] = key[0];
		val[last] = val[0];
		heap_adjust(key, val, 0, last, vk, vv);
	}
}

// One Hoare partition of [f, l) after the median-of-three pivot move
// (std::__unguarded_partition_pivot). Returns the cut.
__device__ int64_t warp_partition(double* key, int32_t* val, int64_t f, int64_t l, int32_t* SL, int32_t* SR) {
	const int lane = threadIdx.x & 31;
	if (lane == 0) {
		int64_t a = f + 1, b = f + (l - f) / 2, c = l - 1;
		double ka = key[a], kb = key[b], kc = key[c];
		int64_t m;
		if (ka < kb) {
			if (kb < kc) m = b;
			else if (ka < kc) m = c;
			else m = a;
		} else if (ka < kc) m = a;
		else if (kb < kc) m = c;
		else m = b;
		double tk = key[f]; key[f] = key[m]; key[m] = tk;
		int32_t tv = val[f]; val[f] = val[m]; val[m] = tv;
	}
	__syncwarp();
	const double P = key[f];
	const uint32_t lt = lanemask_lt();
	int cL = 0, cR = 0;
	for (int64_t base = f + 1; base < l; base += 32) {
		int64_t p = base + lane;
		bool valid = p < l;
		double k = valid ? key[p] : 0.0;
		bool isL = valid && !(k < P);
		bool isR = valid && !(P < k);
		uint32_t bL = __ballot_sync(FULL, isL), bR = __ballot_sync(FULL, isR);
		if (isL) SL[cL + __popc(bL & lt)] = (int32_t)(p - f);
		if (isR) SR[cR + __popc(bR & lt)] = (int32_t)(p - f);
		cL += __popc(bL);
		cR += __popc(bR);
	}
	__syncwarp();
	const int m = cL < cR ? cL : cR;
	int K = m;
	for (int kb = 0; kb < m; kb += 32) {
		int k = kb + lane;
		bool stop = k < m && !(SL[k] < SR[cR - 1 - k]);
		uint32_t b = __ballot_sync(FULL, stop);
		if (b) { K = kb + __ffs(b) - 1; break; }
	}
	for (int k = lane; k < K; k += 32) {
		int64_t i = f + SL[k], j = f + SR[cR - 1 - k];
		double tk = key[i]; key[i] = key[j]; key[j] = tk;
		int32_t tv = val[i]; val[i] = val[j]; val[j] = tv;
	}
	int64_t c1 = K < cL ? (int64_t)SL[K] : INT64_MAX;
	int64_t c2 = K >= 1 ? (int64_t)SR[cR - K] : INT64_MAX;
	__syncwarp();
	return f + (c1 < c2 ? c1 : c2);
}

constexpr int kStackDepth = 128;

using Seg = SortSeg;

__device__ __forceinline__ int introsort_depth(int64_t n) { return 2 * (63 - __clzll((long long)n)); }  // std::__lg(n) * 2

// Replays std::__introsort_loop on [f0, l0) with depth budget d0, one warp.
// The <= 16-element segments the loop leaves behind are appended to blk
// (counter nblk); heap-sorted segments need no final pass.
__device__ void warp_introsort(double* key, int32_t* val, int64_t f0, int64_t l0, int d0, int32_t* SL, int32_t* SR, int32_t* blk,
                               int* nblk, Seg* stack, SampleStats* st, int stack_cap = kStackDepth) {
	const int lane = threadIdx.x & 31;
	if (lane == 0) stack[0] = {f0, l0, d0, 0};
	int sp = 1;
	__syncwarp();
	while (sp > 0) {
		Seg s = stack[sp - 1];
		sp--;
		__syncwarp();
		int64_t f = s.f, l = s.l;
		int d = s.d;
		bool done = false;
		while (l - f > 16) {
			if (d == 0) {
				if (lane == 0) {
					heap_sort(key + f, val + f, l - f);
					atomicAdd(&st->heapsorts, 1ull);
				}
				__syncwarp();
				done = true;
				break;
			}
			d--;
			int64_t cut = warp_partition(key, val, f, l, SL + f, SR + f);
			if (cut <= f || cut >= l || sp >= stack_cap) {
				// cannot happen for comparable keys (the median-of-three
				// guarantees stops on both sides, and a path holds at most
				// depth-budget pending segments); record and stop
				if (lane == 0) atomicAdd(&st->timeouts, 1ull);
				done = true;
				break;
			}
			if (lane == 0) stack[sp] = {cut, l, d, 0};
			sp++;
			__syncwarp();
			l = cut;
		}
		if (!done && l - f > 1 && lane == 0) {
			int b = atomicAdd(nblk, 1);
			blk[2 * b] = (int32_t)f;
			blk[2 * b + 1] = (int32_t)l;
		}
	}
	__syncwarp();
}

// std::__final_insertion_sort: on the block structure the introsort loop
// leaves, it equals a stable insertion sort inside every block.
__device__ void insertion_blocks(double* key, int32_t* val, const int32_t* blk, int nblk, int tid, int nthreads) {
	for (int b = tid; b < nblk; b += nthreads) {
		int64_t s = blk[2 * b], e = blk[2 * b + 1];
		for (int64_t i = s + 1; i < e; i++) {
			double vk = key[i];
			int32_t vv = val[i];
			int64_t j = i;
			while (j > s && vk < key[j - 1]) {
				key[j] = key[j - 1];
				val[j] = val[j - 1];
				j--;
			}
			key[j] = vk;
			val[j] = vv;
		}
	}
}

// std::sort on key/val[0..n) with one warp.
__device__ void warp_std_sort(double* key, int32_t* val, int64_t n, int32_t* SL, int32_t* SR, int32_t* blk, Seg* stack, int* nblk,
                              SampleStats* st) {
	const int lane = threadIdx.x & 31;
	if (lane == 0) *nblk = 0;
	__syncwarp();
	if (n > 1) warp_introsort(key, val, 0, n, introsort_depth(n), SL, SR, blk, nblk, stack, st);
	__syncwarp();
	insertion_blocks(key, val, blk, *nblk, lane, 32);
	__syncwarp();
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32) node_sort_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ order,
                                                                       int node_begin, int node_end, LevelBuffers lb, SortScratch sc,
                                                                       SampleStats* st, int* next_node) {
	__shared__ Seg stacks[kWarpsPerBlock][kStackDepth];
	__shared__ int nblk[kWarpsPerBlock];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	while (true) {
		int idx = 0;
		if (lane == 0) idx = atomicAdd(next_node, 1);
		idx = __shfl_sync(FULL, idx, 0) + node_begin;
		if (idx >= node_end) break;
		const LevelNode nd = nodes[order[idx]];
		double* key = lb.keys + nd.cand_off;
		int32_t* val = lb.perm + nd.cand_off;
		warp_std_sort(key, val, nd.count, sc.SL + nd.cand_off, sc.SR + nd.cand_off, sc.blk + 2 * nd.cand_off, stacks[warp], &nblk[warp], st);
		for (int64_t t = lane; t < nd.count; t += 32) lb.pos[nd.cand_off + val[t]] = (int32_t)t;
	}
}

__global__ void sort_single_kernel(double* key, int32_t* val, int64_t n, SortScratch sc, SampleStats* st) {
	__shared__ Seg stack[kStackDepth];
	__shared__ int nblk;
	if (threadIdx.x >= 32) return;
	warp_std_sort(key, val, n, sc.SL, sc.SR, sc.blk, stack, &nblk, st);
}

// ---------------------------------------------- one CTA per large node
constexpr int kBigSortMin = 4096;    // segments this long are partitioned by the whole CTA
constexpr int kSmallQueue = 256;

// The same partition as warp_partition, computed by the whole CTA.
__device__ int64_t block_partition(double* key, int32_t* val, int64_t f, int64_t l, int32_t* SL, int32_t* SR, BlockScratch& sh) {
	const int tid = threadIdx.x;
	if (tid == 0) {
		int64_t a = f + 1, b = f + (l - f) / 2, c = l - 1;
		double ka = key[a], kb = key[b], kc = key[c];
		int64_t m;
		if (ka < kb) {
			if (kb < kc) m = b;
			else if (ka < kc) m = c;
			else m = a;
		} else if (ka < kc) m = a;
		else if (kb < kc) m = c;
		else m = b;
		double tk = key[f]; key[f] = key[m]; key[m] = tk;
		int32_t tv = val[f]; val[f] = val[m]; val[m] = tv;
	}
	__syncthreads();
	const double P = key[f];
	int64_t cL = 0, cR = 0;
	constexpr int IPT = 4;
	for (int64_t base = f + 1; base < l; base += (int64_t)kBigThreads * IPT) {
		const int64_t p0 = base + (int64_t)tid * IPT;
		unsigned lm = 0, rm = 0;
		uint32_t lc = 0, rc = 0;
#pragma unroll
		for (int k = 0; k < IPT; k++) {
			int64_t p = p0 + k;
			if (p < l) {
				double kk = key[p];
				if (!(kk < P)) { lm |= 1u << k; lc++; }
				if (!(P < kk)) { rm |= 1u << k; rc++; }
			}
		}
		unsigned long long total;
		unsigned long long pre = block_scan_u64(((unsigned long long)rc << 32) | lc, total, sh);
		int64_t lpos = cL + (int64_t)(pre & 0xffffffffull), rpos = cR + (int64_t)(pre >> 32);
#pragma unroll
		for (int k = 0; k < IPT; k++) {
			if (lm & (1u << k)) SL[lpos++] = (int32_t)(p0 + k - f);
			if (rm & (1u << k)) SR[rpos++] = (int32_t)(p0 + k - f);
		}
		cL += (int64_t)(total & 0xffffffffull);
		cR += (int64_t)(total >> 32);
	}
	__syncthreads();
	const int64_t m = cL < cR ? cL : cR;
	// first k with !(SL[k] < SR[cR-1-k]); the predicate is monotone in k
	if (tid == 0) { sh.first_true = m; sh.bracket = 0; }
	__syncthreads();
	const int64_t stride = (m + kBigThreads - 1) / kBigThreads;
	if (m > 0) {
		int64_t k = (int64_t)tid * stride;
		if (k < m && !(SL[k] < SR[cR - 1 - k])) atomicMin((unsigned long long*)&sh.first_true, (unsigned long long)k);
	}
	__syncthreads();
	const int64_t coarse = sh.first_true;  // a k where the predicate holds, or m
	const int64_t lo = coarse >= stride ? coarse - stride + 1 : 0;
	for (int64_t k = lo + tid; k < coarse && k < m; k += kBigThreads)
		if (!(SL[k] < SR[cR - 1 - k])) atomicMin((unsigned long long*)&sh.first_true, (unsigned long long)k);
	__syncthreads();
	const int64_t K = sh.first_true;
	for (int64_t k = tid; k < K; k += kBigThreads) {
		int64_t i = f + SL[k], j = f + SR[cR - 1 - k];
		double tk = key[i]; key[i] = key[j]; key[j] = tk;
		int32_t tv = val[i]; val[i] = val[j]; val[j] = tv;
	}
	int64_t c1 = K < cL ? (int64_t)SL[K] : INT64_MAX;
	int64_t c2 = K >= 1 ? (int64_t)SR[cR - K] : INT64_MAX;
	__syncthreads();
	return f + (c1 < c2 ? c1 : c2);
}

// std::sort on key/val[0..n) with one CTA: segments of at least
// kBigSortMin elements are partitioned by the block, shorter ones by warps.
__device__ void block_std_sort(double* key, int32_t* val, int64_t n, int32_t* SL, int32_t* SR, int32_t* blk, SampleStats* st,
                               int d0 = -1) {
	__shared__ Seg bstack[kStackDepth];
	__shared__ Seg queue[kSmallQueue];
	__shared__ Seg wstacks[kBigWarps][64];
	__shared__ int qn, nblk;
	__shared__ BlockScratch sh;
	const int tid = threadIdx.x, warp = tid >> 5;
	if (tid == 0) { qn = 0; nblk = 0; }
	__syncthreads();
	auto drain = [&]() {
		// warps take the queued small segments
		for (int q = warp; q < qn; q += kBigWarps)
			warp_introsort(key, val, queue[q].f, queue[q].l, queue[q].d, SL, SR, blk, &nblk, wstacks[warp], st, 64);
		__syncthreads();
		if (tid == 0) qn = 0;
		__syncthreads();
	};
	if (n > 1) {
		int sp = 1;
		if (tid == 0) bstack[0] = {0, n, d0 < 0 ? introsort_depth(n) : d0, 0};
		__syncthreads();
		while (sp > 0) {
			Seg s = bstack[sp - 1];
			sp--;
			__syncthreads();
			int64_t f = s.f, l = s.l;
			int d = s.d;
			bool done = false;
			while (l - f > 16) {
				if (l - f < kBigSortMin) {
					if (tid == 0) queue[qn++] = {f, l, d, 0};
					__syncthreads();
					if (qn == kSmallQueue) drain();
					done = true;
					break;
				}
				if (d == 0) {
					if (tid == 0) {
						heap_sort(key + f, val + f, l - f);
						atomicAdd(&st->heapsorts, 1ull);
					}
					__syncthreads();
					done = true;
					break;
				}
				d--;
				int64_t cut = block_partition(key, val, f, l, SL + f, SR + f, sh);
				if (cut <= f || cut >= l || sp >= kStackDepth) {
					if (tid == 0) atomicAdd(&st->timeouts, 1ull);
					done = true;
					break;
				}
				if (tid == 0) bstack[sp] = {cut, l, d, 0};
				sp++;
				__syncthreads();
				l = cut;
			}
			if (!done && l - f > 1 && tid == 0) {
				int b = atomicAdd(&nblk, 1);
				blk[2 * b] = (int32_t)f;
				blk[2 * b + 1] = (int32_t)l;
			}
			__syncthreads();
		}
		drain();
	}
	insertion_blocks(key, val, blk, nblk, tid, kBigThreads);
	__syncthreads();
}

__global__ void __launch_bounds__(kBigThreads) node_sort_big_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ order,
                                                                   int node_begin, LevelBuffers lb, SortScratch sc, SampleStats* st) {
	const LevelNode nd = nodes[order[node_begin + blockIdx.x]];
	int32_t* val = lb.perm + nd.cand_off;
	block_std_sort(lb.keys + nd.cand_off, val, nd.count, sc.SL + nd.cand_off, sc.SR + nd.cand_off, sc.blk + 2 * nd.cand_off, st);
	for (int64_t t = threadIdx.x; t < nd.count; t += kBigThreads) lb.pos[nd.cand_off + val[t]] = (int32_t)t;
}

__global__ void __launch_bounds__(kBigThreads) sort_single_big_kernel(double* key, int32_t* val, int64_t n, SortScratch sc, SampleStats* st) {
	block_std_sort(key, val, n, sc.SL, sc.SR, sc.blk, st);
}


// ------------------------------------------ segments replayed by the GPU
// Segments longer than kWideMin (the top partitions of large nodes) are
// partitioned level-synchronously across the whole GPU: every round
// partitions all pending long segments of all nodes at once -- pivot move,
// stop counts per 4096-element tile, one scan, stop lists, the pair search,
// the swaps -- so the first partitions of a node with millions of
// candidates no longer run on a single CTA. Both halves of a partition go on
// with the decremented depth budget (std::__introsort_loop), so the order in
// which disjoint segments are processed does not change the result.
// Segments at most kWideMin long finish on one warp each with their
// remaining depth budget (a CTA for one whose budget is spent, which is
// heap-sorted); <= 16-element segments go to the final insertion pass, and
// segments whose keys became distinct are written from the sorted keys.
// kWideMin = 1024 measured fastest on the 50M benchmark cloud (sort 36.6 ms
// per conversion against 40.1 with 4096 and 37.0 with 512): once finished
// segments leave the rounds, the rounds only carry the segments around
// equal keys, and the less of them a warp replays in global memory, the
// better.
constexpr int64_t kWideMin = 1024;
constexpr int kWideThreads = 256;
constexpr int kWideWarps = kWideThreads / 32;
constexpr int kWideSteps = 16;
constexpr int kWideTile = kWideThreads * kWideSteps;  // 4096

struct WideTile {
	int64_t p0;          // first element of the tile (after the segment's pivot slot)
	int32_t count;       // elements in the tile
	int32_t seg;         // index in the round's segment list
	int32_t first_tile;  // the segment's first tile
	int32_t last_tile;   // the segment's last tile
};

// The key range a segment's elements lie in, from the pivots of the
// partitions that made it: lo <= key <= hi. Bit 0 of inc: the element keyed
// lo is in the segment, bit 1: the element keyed hi (meaningful when that
// key occurs once in the node: a partition leaves its pivot at the front of
// its left half, and an element keyed strictly between two pivots stays
// between them).
struct SegBounds {
	double lo, hi;
	int32_t inc;
	int32_t pad;
};

struct FinSeg {          // a segment written from the sorted keys
	int64_t f, l;        // its range in key/val
	int64_t a;           // its first element in the sorted order
};

struct WideLists {       // outputs of a round (device counters)
	Seg* next; int* n_next;   // still longer than kWideMin
	SegBounds* next_b;        // their key ranges
	Seg* cta;  int* n_cta;    // CTA replay (>= kBigSortMin elements, or heapsort)
	Seg* warp; int* n_warp;   // warp replay
	int32_t* blk; int* n_blk; // <= 16 elements: final insertion pass (absolute f, l)
	FinSeg* fin; int* n_fin;  // distinct keys: written from the sorted keys
	int64_t cap_seg, cap_blk;
	SortedLevel sl;           // the sorted keys (sl.sk == nullptr: none)
	int64_t wide_min;         // segments longer than this go on with the GPU-wide rounds
};

// kWideMin, or PCG_WIDE_MIN for measurements
int64_t wide_min() {
	static const int64_t v = [] {
		const char* e = std::getenv("PCG_WIDE_MIN");
		const int64_t x = e ? std::atoll(e) : kWideMin;
		return x >= 32 ? x : kWideMin;
	}();
	return v;
}

__global__ void wide_pivot_kernel(const Seg* __restrict__ segs, int n, double* key, int32_t* val) {
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	// std::__move_median_to_first(first, first + 1, mid, last - 1)
	const int64_t f = segs[s].f, l = segs[s].l;
	const int64_t a = f + 1, b = f + (l - f) / 2, c = l - 1;
	const double ka = key[a], kb = key[b], kc = key[c];
	int64_t m;
	if (ka < kb) {
		if (kb < kc) m = b;
		else if (ka < kc) m = c;
		else m = a;
	} else if (ka < kc) m = a;
	else if (kb < kc) m = c;
	else m = b;
	const double tk = key[f]; key[f] = key[m]; key[m] = tk;
	const int32_t tv = val[f]; val[f] = val[m]; val[m] = tv;
}

// stop flags of one tile in warp-contiguous order: warp w covers tile
// elements [512w, 512w + 512) in 16 lane-striped steps
__device__ __forceinline__ void wide_flags(const WideTile& t, const double* key, double P, uint32_t& lbits, uint32_t& rbits) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	lbits = rbits = 0;
#pragma unroll
	for (int st = 0; st < kWideSteps; st++) {
		const int li = warp * (kWideSteps * 32) + st * 32 + lane;
		if (li < t.count) {
			const double k = key[t.p0 + li];
			if (!(k < P)) lbits |= 1u << st;
			if (!(P < k)) rbits |= 1u << st;
		}
	}
}

__global__ void __launch_bounds__(kWideThreads) wide_count_kernel(const WideTile* __restrict__ tiles, const Seg* __restrict__ segs,
                                                                const double* __restrict__ key, unsigned long long* __restrict__ counts) {
	__shared__ unsigned long long wsum[kWideWarps];
	const WideTile t = tiles[blockIdx.x];
	const double P = key[segs[t.seg].f];
	uint32_t lb, rb;
	wide_flags(t, key, P, lb, rb);
	unsigned long long v = ((unsigned long long)__popc(rb) << 32) | (unsigned long long)__popc(lb);
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
	if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = v;
	__syncthreads();
	if (threadIdx.x == 0) {
		unsigned long long tot = 0;
		for (int w = 0; w < kWideWarps; w++) tot += wsum[w];
		counts[blockIdx.x] = tot;
	}
}

__global__ void __launch_bounds__(kWideThreads) wide_write_kernel(const WideTile* __restrict__ tiles, const Seg* __restrict__ segs,
                                                                const double* __restrict__ key, const unsigned long long* __restrict__ offs,
                                                                int32_t* __restrict__ SL, int32_t* __restrict__ SR) {
	__shared__ unsigned long long wsum[kWideWarps];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const WideTile t = tiles[blockIdx.x];
	const int64_t f = segs[t.seg].f;
	const double P = key[f];
	uint32_t lb, rb;
	wide_flags(t, key, P, lb, rb);
	// per-warp totals, exclusive over the warps of the tile
	unsigned long long v = ((unsigned long long)__popc(rb) << 32) | (unsigned long long)__popc(lb);
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
	if (lane == 0) wsum[warp] = v;
	__syncthreads();
	unsigned long long before = offs[blockIdx.x] - offs[t.first_tile];
	for (int w = 0; w < warp; w++) before += wsum[w];
	int64_t cl = (int64_t)(before & 0xffffffffull), cr = (int64_t)(before >> 32);
	const uint32_t lt = lanemask_lt();
	int32_t* sl = SL + f;
	int32_t* sr = SR + f;
#pragma unroll
	for (int st = 0; st < kWideSteps; st++) {
		const bool isL = (lb >> st) & 1u, isR = (rb >> st) & 1u;
		const uint32_t bL = __ballot_sync(FULL, isL), bR = __ballot_sync(FULL, isR);
		const int32_t rel = (int32_t)(t.p0 + warp * (kWideSteps * 32) + st * 32 + lane - f);
		if (isL) sl[cl + __popc(bL & lt)] = rel;
		if (isR) sr[cr + __popc(bR & lt)] = rel;
		cl += __popc(bL);
		cr += __popc(bR);
	}
}

__device__ __forceinline__ void wide_push(Seg* list, int* n, int64_t cap, const Seg& s, SampleStats* st) {
	const int i = atomicAdd(n, 1);
	if (i < cap) list[i] = s;
	else atomicAdd(&st->timeouts, 1ull);
}

// position of key v in the node's sorted keys [n0, n1): the first with key
// >= v (upper = false) or > v (upper = true); keys are >= +0, so their bit
// patterns order like their values, and the open ends (-inf, +inf) map to
// the node's ends
__device__ int64_t sorted_bound(const uint64_t* sk, int64_t n0, int64_t n1, double v, bool upper) {
	if (v == -CUDART_INF) return n0;
	if (v == CUDART_INF) return n1;
	const uint64_t bv = (uint64_t)__double_as_longlong(v);
	int64_t lo = n0, hi = n1;
	while (lo < hi) {
		const int64_t mid = lo + (hi - lo) / 2;
		if (upper ? sk[mid] <= bv : sk[mid] < bv) lo = mid + 1;
		else hi = mid;
	}
	return lo;
}

// Whether segment [f, l) with bounds b holds pairwise distinct keys, and
// where its elements sit in the sorted order: the four positions
// lower(lo), upper(lo), lower(hi), upper(hi) are given. Requires lo < hi,
// each bound key at most once in the node, and a slice of the segment's
// size without adjacent equal keys.
__device__ bool distinct_slice(const SortedLevel& sl, int64_t f, int64_t l, const SegBounds& b, int64_t llo, int64_t ulo, int64_t lhi,
                               int64_t uhi, int64_t* a) {
	if (!(b.lo < b.hi) || ulo - llo > 1 || uhi - lhi > 1) return false;
	const int64_t first = (b.inc & 1) ? llo : ulo, last = (b.inc & 2) ? uhi : lhi;
	if (last - first != l - f) return false;
	if (last - first >= 2 && sl.ties[last - 1] != sl.ties[first]) return false;
	*a = first;
	return true;
}

// slice_a >= 0: the segment's keys are distinct, its elements are
// sorted[slice_a, slice_a + l - f)
__device__ void wide_classify(int64_t f, int64_t l, int d, const SegBounds& b, int64_t slice_a, const WideLists& L, SampleStats* st) {
	const int64_t n = l - f;
	if (n > 16 && slice_a >= 0) {
		const int i = atomicAdd(L.n_fin, 1);
		if (i < L.cap_seg) L.fin[i] = {f, l, slice_a};
		else atomicAdd(&st->timeouts, 1ull);
		return;
	}
	if (n <= 16) {
		if (n > 1) {
			const int i = atomicAdd(L.n_blk, 1);
			if (i < L.cap_blk) {
				L.blk[2 * (int64_t)i] = (int32_t)f;
				L.blk[2 * (int64_t)i + 1] = (int32_t)l;
			} else {
				atomicAdd(&st->timeouts, 1ull);
			}
		}
	} else if (d == 0 || (n >= kBigSortMin && n <= L.wide_min)) {
		wide_push(L.cta, L.n_cta, L.cap_seg, {f, l, d, 0}, st);
	} else if (n > L.wide_min) {
		const int i = atomicAdd(L.n_next, 1);
		if (i < L.cap_seg) {
			L.next[i] = {f, l, d, 0};
			L.next_b[i] = b;
		} else {
			atomicAdd(&st->timeouts, 1ull);
		}
	} else {
		wide_push(L.warp, L.n_warp, L.cap_seg, {f, l, d, 0}, st);
	}
}

// one warp per segment: Hoare's pair count K, the cut, the two halves
__global__ void wide_split_kernel(const Seg* __restrict__ segs, const SegBounds* __restrict__ bounds, int n, const WideTile* __restrict__ tiles,
                                  const int32_t* __restrict__ seg_tile, const unsigned long long* __restrict__ counts,
                                  const unsigned long long* __restrict__ offs, const int32_t* __restrict__ SL, const int32_t* __restrict__ SR,
                                  const double* __restrict__ key, int64_t* __restrict__ segK, int64_t* __restrict__ segCR, WideLists L,
                                  SampleStats* st) {
	const int s = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
	const int lane = threadIdx.x & 31;
	if (s >= n) return;
	const Seg g = segs[s];
	const WideTile ft = tiles[seg_tile[s]];
	const unsigned long long tot = offs[ft.last_tile] + counts[ft.last_tile] - offs[ft.first_tile];
	const int64_t cL = (int64_t)(tot & 0xffffffffull), cR = (int64_t)(tot >> 32);
	const int32_t* sl = SL + g.f;
	const int32_t* sr = SR + g.f;
	// first k in [0, m) with !(SL[k] < SR[cR-1-k]), m if none (monotone)
	int64_t lo = 0, hi = cL < cR ? cL : cR;
	while (hi - lo > 32) {
		const int64_t step = (hi - lo + 31) / 32;
		const int64_t k = lo + lane * step;
		const bool p = k < hi && !(sl[k] < sr[cR - 1 - k]);
		const uint32_t b = __ballot_sync(FULL, p);
		if (b == 0) {
			const int64_t jmax = (hi - 1 - lo) / step < 31 ? (hi - 1 - lo) / step : 31;
			lo = lo + jmax * step + 1;
		} else {
			const int j = __ffs(b) - 1;
			const int64_t nlo = j > 0 ? lo + (int64_t)(j - 1) * step + 1 : lo;
			hi = lo + (int64_t)j * step;
			lo = nlo;
		}
	}
	{
		const int64_t k = lo + lane;
		const bool p = k < hi && !(sl[k] < sr[cR - 1 - k]);
		const uint32_t b = __ballot_sync(FULL, p);
		if (b) hi = lo + __ffs(b) - 1;
	}
	const int64_t K = hi;
	const int64_t c1 = K < cL ? (int64_t)sl[K] : INT64_MAX;
	const int64_t c2 = K >= 1 ? (int64_t)sr[cR - K] : INT64_MAX;
	const int64_t cut = g.f + (c1 < c2 ? c1 : c2);
	if (cut <= g.f || cut >= g.l) {
		if (lane == 0) {
			segK[s] = 0;
			segCR[s] = cR;
			atomicAdd(&st->timeouts, 1ull);
		}
		return;
	}
	const int d = g.d - 1;
	// the halves' key ranges: the pivot (key[g.f], moved there by
	// wide_pivot_kernel) stays at the front of the left half
	const SegBounds pb = bounds[s];
	const double P = key[g.f];
	const SegBounds bR{P, pb.hi, pb.inc & 2, 0}, bL{pb.lo, P, (pb.inc & 1) | 2, 0};
	// lanes 0-7 find the halves' bound keys in the sorted order at once
	int64_t pos = 0;
	if (L.sl.sk && lane < 8) {
		const LevelNode nd = L.sl.nodes[L.sl.node_of[g.f]];
		const SegBounds& hb = lane < 4 ? bR : bL;
		const int w = lane & 3;
		pos = sorted_bound(L.sl.sk, nd.cand_off, nd.cand_off + nd.count, w < 2 ? hb.lo : hb.hi, (w & 1) != 0);
	}
	int64_t q[8];
#pragma unroll
	for (int i = 0; i < 8; i++) q[i] = __shfl_sync(FULL, pos, i);
	if (lane != 0) return;
	segK[s] = K;
	segCR[s] = cR;
	int64_t aR = -1, aL = -1;
	if (L.sl.sk) {
		if (!distinct_slice(L.sl, cut, g.l, bR, q[0], q[1], q[2], q[3], &aR)) aR = -1;
		if (!distinct_slice(L.sl, g.f, cut, bL, q[4], q[5], q[6], q[7], &aL)) aL = -1;
	}
	wide_classify(cut, g.l, d, bR, aR, L, st);
	wide_classify(g.f, cut, d, bL, aL, L, st);
}

// the segments with distinct keys get their sorted keys in order; one CTA
// per tile of kFinTile elements of a segment (tile_seg / tile_off)
constexpr int64_t kFinTile = 4096;
__global__ void __launch_bounds__(256) fin_copy_kernel(const FinSeg* __restrict__ fin, const int32_t* __restrict__ tile_seg,
                                                       const int64_t* __restrict__ tile_off, SortedLevel sl, double* key, int32_t* val) {
	const FinSeg g = fin[tile_seg[blockIdx.x]];
	const int64_t i0 = tile_off[blockIdx.x], i1 = i0 + kFinTile < g.l - g.f ? i0 + kFinTile : g.l - g.f;
	for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
		key[g.f + i] = __longlong_as_double((long long)sl.sk[g.a + i]);
		val[g.f + i] = (int32_t)sl.sv[g.a + i];
	}
}

__global__ void __launch_bounds__(kWideThreads) wide_swap_kernel(const WideTile* __restrict__ tiles, const Seg* __restrict__ segs,
                                                               const int64_t* __restrict__ segK, const int64_t* __restrict__ segCR,
                                                               const int32_t* __restrict__ SL, const int32_t* __restrict__ SR, double* key,
                                                               int32_t* val) {
	const WideTile t = tiles[blockIdx.x];
	const int64_t f = segs[t.seg].f;
	const int64_t K = segK[t.seg], cR = segCR[t.seg];
	const int64_t k0 = t.p0 - (f + 1);  // the tile's elements double as its share of the pair indices
	for (int j = threadIdx.x; j < t.count; j += kWideThreads) {
		const int64_t k = k0 + j;
		if (k >= K) break;
		const int64_t a = f + SL[f + k], b = f + SR[f + cR - 1 - k];
		const double tk = key[a]; key[a] = key[b]; key[b] = tk;
		const int32_t tv = val[a]; val[a] = val[b]; val[b] = tv;
	}
}

__global__ void __launch_bounds__(kBigThreads) seg_cta_kernel(const Seg* __restrict__ segs, double* key, int32_t* val, SortScratch sc,
                                                             SampleStats* st) {
	const Seg g = segs[blockIdx.x];
	block_std_sort(key + g.f, val + g.f, g.l - g.f, sc.SL + g.f, sc.SR + g.f, sc.blk + 2 * g.f, st, g.d);
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32) seg_warp_kernel(const Seg* __restrict__ segs, int n, double* key, int32_t* val,
                                                                      SortScratch sc, SampleStats* st, int* next_seg) {
	__shared__ Seg stacks[kWarpsPerBlock][kStackDepth];
	__shared__ int nblk[kWarpsPerBlock];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	while (true) {
		int idx = 0;
		if (lane == 0) idx = atomicAdd(next_seg, 1);
		idx = __shfl_sync(FULL, idx, 0);
		if (idx >= n) break;
		const Seg g = segs[idx];
		const int64_t len = g.l - g.f;
		if (lane == 0) nblk[warp] = 0;
		__syncwarp();
		warp_introsort(key + g.f, val + g.f, 0, len, g.d, sc.SL + g.f, sc.SR + g.f, sc.blk + 2 * g.f, &nblk[warp], stacks[warp], st);
		__syncwarp();
		insertion_blocks(key + g.f, val + g.f, sc.blk + 2 * g.f, nblk[warp], lane, 32);
		__syncwarp();
	}
}

__global__ void blk_insertion_kernel(const int32_t* __restrict__ blk, int n, double* key, int32_t* val) {
	const int b = blockIdx.x * blockDim.x + threadIdx.x;
	if (b < n) insertion_blocks(key, val, blk + 2 * (int64_t)b, 1, 0, 1);
}

__global__ void node_pos_kernel(const LevelNode* __restrict__ nodes, const uint8_t* __restrict__ pick, LevelBuffers lb) {
	const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= lb.M) return;
	const int32_t n = lb.node_of[j];
	if (!pick[n]) return;
	const int64_t co = nodes[n].cand_off;
	lb.pos[co + lb.perm[j]] = (int32_t)(j - co);
}

int host_introsort_depth(int64_t n) {
	int lg = 0;
	while ((n >> (lg + 1)) != 0) lg++;
	return 2 * lg;
}

}  // namespace

void launch_node_sort(const LevelNode* nodes, const int32_t* order, int K, LevelBuffers& lb, SampleStats* st, DeviceMem& mem,
                      int node_begin, int node_end, int num_big) {
	if (node_end < 0) node_end = K;
	if (node_end <= node_begin || lb.M == 0) return;
	SortScratch sc;
	sc.SL = mem.alloc<int32_t>(lb.M);
	sc.SR = mem.alloc<int32_t>(lb.M);
	sc.blk = mem.alloc<int32_t>(2 * lb.M);
	// nodes order[0..num_big) get a CTA each, the rest a warp each
	const int big_end = num_big < node_end ? num_big : node_end;
	if (big_end > node_begin) {
		node_sort_big_kernel<<<big_end - node_begin, kBigThreads, 0, mem.stream()>>>(nodes, order, node_begin, lb, sc, st);
		PCG_LAUNCHED();
	}
	const int small_begin = node_begin > num_big ? node_begin : num_big;
	if (node_end > small_begin) {
		int* counter = mem.alloc<int>(1);
		PCG_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), mem.stream()));
		int blocks = (int)ceil_div(node_end - small_begin, kWarpsPerBlock);
		int cap = sm_count() * 16;
		if (blocks > cap) blocks = cap;
		node_sort_kernel<<<blocks, kWarpsPerBlock * 32, 0, mem.stream()>>>(nodes, order, small_begin, node_end, lb, sc, st, counter);
		PCG_LAUNCHED();
		mem.free(counter);
	}
	mem.free(sc.SL);
	mem.free(sc.SR);
	mem.free(sc.blk);
}

void replay_segments(double* key, int32_t* val, int64_t M, const std::vector<SortSeg>& segs, SampleStats* st, DeviceMem& mem,
                     const SortedLevel* sorted) {
	if (segs.empty() || M == 0) return;
	const SortedLevel sl = sorted ? *sorted : SortedLevel{};
	cudaStream_t s = mem.stream();
	SortScratch sc;
	sc.SL = mem.alloc<int32_t>(M);
	sc.SR = mem.alloc<int32_t>(M);
	sc.blk = mem.alloc<int32_t>(2 * M);
	WideLists L;
	L.cap_seg = M / 16 + 64;
	L.cap_blk = M / 2 + 64;
	L.sl = sl;
	L.wide_min = wide_min();
	Seg* ping[2] = {mem.alloc<Seg>(L.cap_seg), mem.alloc<Seg>(L.cap_seg)};
	SegBounds* pingb[2] = {mem.alloc<SegBounds>(L.cap_seg), mem.alloc<SegBounds>(L.cap_seg)};
	L.cta = mem.alloc<Seg>(L.cap_seg);
	L.warp = mem.alloc<Seg>(L.cap_seg);
	L.blk = mem.alloc<int32_t>(2 * L.cap_blk);
	L.fin = mem.alloc<FinSeg>(L.cap_seg);
	int* counters = mem.alloc<int>(6);  // next, cta, warp, blk, warp-kernel cursor, fin
	L.n_next = counters;
	L.n_cta = counters + 1;
	L.n_warp = counters + 2;
	L.n_blk = counters + 3;
	L.n_fin = counters + 5;
	// the initial segments (whole nodes: every key in range), classified
	// like the halves of a partition
	std::vector<Seg> cur, cta, warp;
	std::vector<SegBounds> curb;
	std::vector<int32_t> blk;
	for (const SortSeg& g : segs) {
		const int64_t n = g.l - g.f;
		if (n <= 16) {
			if (n > 1) { blk.push_back((int32_t)g.f); blk.push_back((int32_t)g.l); }
		} else if (g.d == 0 || (n >= kBigSortMin && n <= L.wide_min)) {
			cta.push_back(g);
		} else if (n > L.wide_min) {
			cur.push_back(g);
			curb.push_back(SegBounds{-std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(), 0, 0});
		} else {
			warp.push_back(g);
		}
	}
	int h_counts[6] = {0, (int)cta.size(), (int)warp.size(), (int)(blk.size() / 2), 0, 0};
	if (!cta.empty()) PCG_CUDA(cudaMemcpyAsync(L.cta, cta.data(), cta.size() * sizeof(Seg), cudaMemcpyHostToDevice, s));
	if (!warp.empty()) PCG_CUDA(cudaMemcpyAsync(L.warp, warp.data(), warp.size() * sizeof(Seg), cudaMemcpyHostToDevice, s));
	if (!blk.empty()) PCG_CUDA(cudaMemcpyAsync(L.blk, blk.data(), blk.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
	PCG_CUDA(cudaMemcpyAsync(counters, h_counts, sizeof(h_counts), cudaMemcpyHostToDevice, s));
	int pp = 0;
	int64_t* segK = nullptr;
	int64_t* segCR = nullptr;
	int64_t seg_cap = 0;
	for (int round = 0; !cur.empty(); round++) {
		if (round > 128) throw PcgError(4, "sort replay: partition rounds did not converge");
		const int n = (int)cur.size();
		std::vector<WideTile> tiles;
		std::vector<int32_t> seg_tile(n);
		for (int i = 0; i < n; i++) {
			const int64_t f = cur[i].f, len = cur[i].l - cur[i].f - 1;  // elements after the pivot slot
			const int first = (int)tiles.size();
			const int nt = (int)ceil_div(len, kWideTile);
			seg_tile[i] = first;
			for (int j = 0; j < nt; j++) {
				WideTile t;
				t.p0 = f + 1 + (int64_t)j * kWideTile;
				t.count = (int32_t)std::min<int64_t>(kWideTile, len - (int64_t)j * kWideTile);
				t.seg = i;
				t.first_tile = first;
				t.last_tile = first + nt - 1;
				tiles.push_back(t);
			}
		}
		const int nt = (int)tiles.size();
		Seg* d_cur = ping[pp];
		SegBounds* d_curb = pingb[pp];
		L.next = ping[pp ^ 1];
		L.next_b = pingb[pp ^ 1];
		PCG_CUDA(cudaMemcpyAsync(d_cur, cur.data(), n * sizeof(Seg), cudaMemcpyHostToDevice, s));
		PCG_CUDA(cudaMemcpyAsync(d_curb, curb.data(), n * sizeof(SegBounds), cudaMemcpyHostToDevice, s));
		WideTile* d_tiles = mem.alloc<WideTile>(nt);
		PCG_CUDA(cudaMemcpyAsync(d_tiles, tiles.data(), nt * sizeof(WideTile), cudaMemcpyHostToDevice, s));
		int32_t* d_seg_tile = mem.alloc<int32_t>(n);
		PCG_CUDA(cudaMemcpyAsync(d_seg_tile, seg_tile.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
		if (n > seg_cap) {
			if (segK) { mem.free(segK); mem.free(segCR); }
			seg_cap = 2 * (int64_t)n;
			segK = mem.alloc<int64_t>(seg_cap);
			segCR = mem.alloc<int64_t>(seg_cap);
		}
		unsigned long long* counts = mem.alloc<unsigned long long>(nt);
		unsigned long long* offs = mem.alloc<unsigned long long>(nt);
		PCG_CUDA(cudaMemsetAsync(L.n_next, 0, sizeof(int), s));
		wide_pivot_kernel<<<(unsigned)ceil_div(n, 128), 128, 0, s>>>(d_cur, n, key, val);
		PCG_LAUNCHED();
		wide_count_kernel<<<nt, kWideThreads, 0, s>>>(d_tiles, d_cur, key, counts);
		PCG_LAUNCHED();
		exclusive_scan_i64(reinterpret_cast<const int64_t*>(counts), reinterpret_cast<int64_t*>(offs), nt, false, mem);
		wide_write_kernel<<<nt, kWideThreads, 0, s>>>(d_tiles, d_cur, key, offs, sc.SL, sc.SR);
		PCG_LAUNCHED();
		wide_split_kernel<<<(unsigned)ceil_div((int64_t)n * 32, 128), 128, 0, s>>>(d_cur, d_curb, n, d_tiles, d_seg_tile, counts, offs, sc.SL,
		                                                                          sc.SR, key, segK, segCR, L, st);
		PCG_LAUNCHED();
		wide_swap_kernel<<<nt, kWideThreads, 0, s>>>(d_tiles, d_cur, segK, segCR, sc.SL, sc.SR, key, val);
		PCG_LAUNCHED();
		int n_next = 0;
		PCG_CUDA(cudaMemcpyAsync(&n_next, L.n_next, sizeof(int), cudaMemcpyDeviceToHost, s));
		PCG_CUDA(cudaStreamSynchronize(s));
		if (n_next > L.cap_seg) throw PcgError(5, "sort replay: segment list overflow");
		cur.resize(n_next);
		curb.resize(n_next);
		if (n_next) {
			PCG_CUDA(cudaMemcpyAsync(cur.data(), L.next, n_next * sizeof(Seg), cudaMemcpyDeviceToHost, s));
			PCG_CUDA(cudaMemcpyAsync(curb.data(), L.next_b, n_next * sizeof(SegBounds), cudaMemcpyDeviceToHost, s));
		}
		PCG_CUDA(cudaStreamSynchronize(s));
		mem.free(counts);
		mem.free(offs);
		mem.free(d_tiles);
		mem.free(d_seg_tile);
		pp ^= 1;
	}
	PCG_CUDA(cudaMemcpyAsync(h_counts, counters, sizeof(h_counts), cudaMemcpyDeviceToHost, s));
	PCG_CUDA(cudaStreamSynchronize(s));
	if (h_counts[1] > L.cap_seg || h_counts[2] > L.cap_seg || h_counts[3] > L.cap_blk || h_counts[5] > L.cap_seg)
		throw PcgError(5, "sort replay: list overflow");
	if (h_counts[5] > 0) {
		std::vector<FinSeg> fin(h_counts[5]);
		PCG_CUDA(cudaMemcpyAsync(fin.data(), L.fin, fin.size() * sizeof(FinSeg), cudaMemcpyDeviceToHost, s));
		PCG_CUDA(cudaStreamSynchronize(s));
		std::vector<int32_t> ts;
		std::vector<int64_t> to;
		for (size_t i = 0; i < fin.size(); i++)
			for (int64_t o = 0; o < fin[i].l - fin[i].f; o += kFinTile) {
				ts.push_back((int32_t)i);
				to.push_back(o);
			}
		int32_t* d_ts = mem.alloc<int32_t>(ts.size());
		int64_t* d_to = mem.alloc<int64_t>(to.size());
		PCG_CUDA(cudaMemcpyAsync(d_ts, ts.data(), ts.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
		PCG_CUDA(cudaMemcpyAsync(d_to, to.data(), to.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s));
		fin_copy_kernel<<<(unsigned)ts.size(), 256, 0, s>>>(L.fin, d_ts, d_to, sl, key, val);
		PCG_LAUNCHED();
		mem.free(d_to);
		mem.free(d_ts);
	}
	if (h_counts[1] > 0) {
		seg_cta_kernel<<<h_counts[1], kBigThreads, 0, s>>>(L.cta, key, val, sc, st);
		PCG_LAUNCHED();
	}
	if (h_counts[2] > 0) {
		PCG_CUDA(cudaMemsetAsync(counters + 4, 0, sizeof(int), s));
		int blocks = (int)ceil_div(h_counts[2], kWarpsPerBlock);
		const int cap = sm_count() * 16;
		if (blocks > cap) blocks = cap;
		seg_warp_kernel<<<blocks, kWarpsPerBlock * 32, 0, s>>>(L.warp, h_counts[2], key, val, sc, st, counters + 4);
		PCG_LAUNCHED();
	}
	if (h_counts[3] > 0) {
		blk_insertion_kernel<<<(unsigned)ceil_div(h_counts[3], 128), 128, 0, s>>>(L.blk, h_counts[3], key, val);
		PCG_LAUNCHED();
	}
	if (segK) { mem.free(segK); mem.free(segCR); }
	mem.free(ping[0]);
	mem.free(ping[1]);
	mem.free(pingb[0]);
	mem.free(pingb[1]);
	mem.free(L.fin);
	mem.free(L.cta);
	mem.free(L.warp);
	mem.free(L.blk);
	mem.free(counters);
	mem.free(sc.SL);
	mem.free(sc.SR);
	mem.free(sc.blk);
}

void launch_node_pos(const LevelNode* nodes, const std::vector<uint8_t>& pick, LevelBuffers& lb, DeviceMem& mem) {
	if (lb.M == 0 || pick.empty()) return;
	uint8_t* d_pick = mem.alloc<uint8_t>(pick.size());
	PCG_CUDA(cudaMemcpyAsync(d_pick, pick.data(), pick.size(), cudaMemcpyHostToDevice, mem.stream()));
	node_pos_kernel<<<(unsigned)ceil_div(lb.M, 256), 256, 0, mem.stream()>>>(nodes, d_pick, lb);
	PCG_LAUNCHED();
	mem.free(d_pick);
}

int sort_depth_budget(int64_t n) { return host_introsort_depth(n); }

void launch_sort_keys_single(double* keys, int32_t* vals, int64_t n, DeviceMem& mem, SampleStats* st, const SortedLevel* sorted) {
	if (n <= 0) return;
	replay_segments(keys, vals, n, {SortSeg{0, n, host_introsort_depth(n), 0}}, st, mem, sorted);
}

}  // namespace pcg

// ================================================= sort without allocation
// pcg_kernel_sort_keys_noalloc: the std::sort replay for callers that cannot
// allocate device memory themselves or let a library do it -- code running
// inside a host framework that owns every device allocation (a plugin under
// a fixed memory budget). Its scratch is this file-scope array, reserved on
// every GPU that loads the library until the process exits. The call waits
// on its stream for the error word, so it cannot be part of a stream
// capture.

#include "../../include/pcgpu.h"

#include <mutex>

namespace pcg {

constexpr int64_t kNoAllocSortMax = PCG_NOALLOC_SORT_MAX;
// per key: working key (8 B), permutation (4 B), left and right stop lists
// (4 + 4 B), final blocks (8 B); then the error counters
constexpr size_t kNoAllocKeyBytes = 28;
constexpr size_t kNoAllocSortBytes = (size_t)kNoAllocSortMax * kNoAllocKeyBytes + 256;
static __device__ __align__(256) unsigned char g_noalloc_sort_scratch[kNoAllocSortBytes];

namespace {

std::mutex g_noalloc_mtx;
constexpr int kMaxDevices = 128;
void* g_noalloc_base[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device (the array's name is only a host-side handle). The address is
// kept for the process's lifetime; a cudaDeviceReset would make it stale,
// which the header tells callers.
cudaError_t noalloc_scratch(int dev, void** out) {
	std::lock_guard<std::mutex> lk(g_noalloc_mtx);
	if (!g_noalloc_base[dev]) {
		void* p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_sort_scratch);
		if (e != cudaSuccess) return e;
		g_noalloc_base[dev] = p;
	}
	*out = g_noalloc_base[dev];
	return cudaSuccess;
}

__global__ void noalloc_prepare_kernel(const double* __restrict__ in, int64_t n, double* __restrict__ key, int32_t* __restrict__ val) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) {
		key[i] = in[i];
		val[i] = (int32_t)i;
	}
}

__global__ void noalloc_finish_kernel(const int32_t* __restrict__ val, int64_t n, int32_t* __restrict__ out) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = val[i];
}

}  // namespace
}  // namespace pcg

extern "C" pcg_status pcg_kernel_sort_keys_noalloc(const double* d_keys, int64_t n, int32_t* d_perm, void* stream) {
	using namespace pcg;
	if (n < 0 || n > kNoAllocSortMax || (n > 0 && (!d_keys || !d_perm))) return PCG_BAD_INPUT;
	if (n == 0) return PCG_OK;
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
		cudaGetLastError();
		return PCG_CUDA;
	}
	// an error somebody else left pending is theirs: report it without
	// consuming it, and launch nothing
	if (cudaPeekAtLastError() != cudaSuccess) return PCG_CUDA;
	void* base = nullptr;
	if (noalloc_scratch(dev, &base) != cudaSuccess) {
		cudaGetLastError();
		return PCG_CUDA;
	}
	unsigned char* b = static_cast<unsigned char*>(base);
	double* key = reinterpret_cast<double*>(b);
	int32_t* val = reinterpret_cast<int32_t*>(b + 8 * kNoAllocSortMax);
	SortScratch sc;
	sc.SL = reinterpret_cast<int32_t*>(b + 12 * kNoAllocSortMax);
	sc.SR = reinterpret_cast<int32_t*>(b + 16 * kNoAllocSortMax);
	sc.blk = reinterpret_cast<int32_t*>(b + 20 * kNoAllocSortMax);
	SampleStats* st = reinterpret_cast<SampleStats*>(b + kNoAllocKeyBytes * kNoAllocSortMax);
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	// the array keeps the previous call's contents: only the error counters
	// must start at zero, every other byte is written before it is read
	if (cudaMemsetAsync(st, 0, sizeof(SampleStats), s) != cudaSuccess) { cudaGetLastError(); return PCG_CUDA; }
	const unsigned blocks = (unsigned)ceil_div(n, 256);
	// each launch is checked at once, so a failure is this call's own
	noalloc_prepare_kernel<<<blocks, 256, 0, s>>>(d_keys, n, key, val);
	if (cudaGetLastError() != cudaSuccess) return PCG_CUDA;
	if (n >= kBigSortMin) sort_single_big_kernel<<<1, kBigThreads, 0, s>>>(key, val, n, sc, st);
	else sort_single_kernel<<<1, 32, 0, s>>>(key, val, n, sc, st);
	if (cudaGetLastError() != cudaSuccess) return PCG_CUDA;
	noalloc_finish_kernel<<<blocks, 256, 0, s>>>(val, n, d_perm);
	if (cudaGetLastError() != cudaSuccess) return PCG_CUDA;
	SampleStats h{};
	if (cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
		cudaGetLastError();
		return PCG_CUDA;
	}
	return h.timeouts ? PCG_INTERNAL : PCG_OK;
}
