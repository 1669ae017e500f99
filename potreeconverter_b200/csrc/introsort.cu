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

struct Seg { int64_t f, l; int32_t d; int32_t pad; };

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
__device__ void block_std_sort(double* key, int32_t* val, int64_t n, int32_t* SL, int32_t* SR, int32_t* blk, SampleStats* st) {
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
		if (tid == 0) bstack[0] = {0, n, introsort_depth(n), 0};
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

void launch_sort_keys_single(double* keys, int32_t* vals, int64_t n, DeviceMem& mem, SampleStats* st) {
	if (n <= 0) return;
	SortScratch sc;
	sc.SL = mem.alloc<int32_t>(n);
	sc.SR = mem.alloc<int32_t>(n);
	sc.blk = mem.alloc<int32_t>(2 * n);
	if (n >= kBigSortMin) sort_single_big_kernel<<<1, kBigThreads, 0, mem.stream()>>>(keys, vals, n, sc, st);
	else sort_single_kernel<<<1, 32, 0, mem.stream()>>>(keys, vals, n, sc, st);
	PCG_LAUNCHED();
}

}  // namespace pcg

// ================================================= sort without allocation
// pcg_kernel_sort_keys_noalloc: the std::sort replay for callers that cannot
// allocate device memory themselves or let a library do it -- code running
// inside a host framework that owns every device allocation (a plugin under
// a fixed memory budget), or code enqueuing work while a stream is being
// captured, where cudaMalloc is not permitted. Its scratch is this
// file-scope array, reserved on every GPU that loads the library until the
// process exits.

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
// per device (the array's name is only a host-side handle).
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
	noalloc_prepare_kernel<<<blocks, 256, 0, s>>>(d_keys, n, key, val);
	if (n >= kBigSortMin) sort_single_big_kernel<<<1, kBigThreads, 0, s>>>(key, val, n, sc, st);
	else sort_single_kernel<<<1, 32, 0, s>>>(key, val, n, sc, st);
	noalloc_finish_kernel<<<blocks, 256, 0, s>>>(val, n, d_perm);
	SampleStats h{};
	if (cudaGetLastError() != cudaSuccess || cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
	    cudaStreamSynchronize(s) != cudaSuccess) {
		cudaGetLastError();
		return PCG_CUDA;
	}
	return h.timeouts ? PCG_INTERNAL : PCG_OK;
}
