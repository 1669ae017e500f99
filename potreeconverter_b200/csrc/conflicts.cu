// Conflict lists for the poisson samplers, built for all nodes of a level at
// once.
//
// The acceptance scan of sampler_poisson.h:133-245 (sampler_poisson_average.h
// :184-281 without the early exit) compares candidate p, in sorted order,
// with the points accepted before it: p is rejected by an accepted a when
// they are closer than the spacing and a lies at or beyond the early-exit
// bound, key(a) >= (sqrt(key(p)) - spacing)^2. Whether a given earlier
// candidate q could reject p is therefore fixed before any decision is made;
// only whether q gets accepted is not. This unit finds, for every candidate
// p, the earlier candidates q of its node with that property -- a
// fixed-radius neighbour search, fully parallel over the level -- so the
// acceptance kernel only has to look at those candidates' decisions.
//
//  1. cell keys: cells of one spacing (x 1.000001) over the node box, so
//     every point closer than the spacing lies in the 3 x 3 x 3 cells around
//     a candidate's own;
//  2. segmented radix sort of (cell, sorted position) per node;
//  3. a hash table per node, cell -> range of the cell-sorted records;
//  4. one thread per candidate in cell order (a warp shares neighbourhoods)
//     scans the occupied cells among its 27 up to its own sorted position:
//     the FP32 distance on node-relative coordinates decides every pair
//     outside the band s^2 (1 -/+ 1e-3); pairs inside the band are decided
//     by the reference's FP64 test and counted as escalated; then the
//     early-exit bound. Error bound (u = 2^-24): a node-relative coordinate
//     v lies in [0, L], L = 128 s, so its float differs from the FP64 value
//     by at most L u = 128 s u; a coordinate difference d (|d| about s in the
//     band) then carries at most 256 s u + |d| u, its square a relative
//     error of 2 (257 u) + u, and the sum of three squares at most 517 u
//     = 3.1e-5 of the squared distance D. The FP64 values the reference
//     compares are themselves within 1.1e-16 |x| of the exact coordinates,
//     below 1.1e-10 s when |x| < 1e6 s (checked per node; beyond it the
//     node uses FP64 alone). So D32 >= s^2 (1 + 1e-3) (rounded up by at
//     most u) implies D64 > s^2, and D32 < s^2 (1 - 1e-3) implies D64 < s^2:
//     the margin is 30x the error.
// A candidate with more than kListCap such predecessors marks its node
// dense; dense nodes keep the grid-based acceptance kernel.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "devutil.cuh"
#include "sampling.h"

namespace pcg {

namespace {

constexpr uint64_t kEmptyRun = ~0ull;
constexpr int kListsVariant = 2;  // see lists_variant(); measured fastest on the benchmark's 50M cloud
constexpr int kCellsPerAxis = 128;  // node box = 128 spacings

struct alignas(16) RunSlot {  // run table entry, one 16-byte load per probe
	uint64_t key;             // cell, kEmptyRun when free
	int32_t start, count;     // first record in the node, records
};

__device__ __forceinline__ uint64_t run_hash(uint64_t k, int64_t cap) {
	return ((k * 0x9E3779B97F4A7C15ull) >> 20) & (uint64_t)(cap - 1);
}

__device__ __forceinline__ double qcoord(int32_t X, int a, const PosParamsS& pp) {
	// (xyz[a] * scale) + offset, sampler_poisson.h:99-101
	return ((double)X * pp.scale[a]) + pp.offset[a];
}

__device__ __forceinline__ int clamp_cell(double u) {
	double f = floor(u);
	f = f < 0.0 ? 0.0 : (f > (double)(kCellsPerAxis - 1) ? (double)(kCellsPerAxis - 1) : f);
	return (int)f;
}

__global__ void conf_cell_keys_kernel(const LevelNode* __restrict__ nodes, PosParamsS pp, LevelBuffers lb, uint64_t* __restrict__ keys) {
	const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= lb.M) return;
	const LevelNode& nd = nodes[lb.node_of[j]];
	const int4 r = lb.cq[j];
	const double inv = 1.0 / (nd.spacing * 1.000001);
	const int cx = clamp_cell((qcoord(r.x, 0, pp) - nd.min[0]) * inv);
	const int cy = clamp_cell((qcoord(r.y, 1, pp) - nd.min[1]) * inv);
	const int cz = clamp_cell((qcoord(r.z, 2, pp) - nd.min[2]) * inv);
	keys[j] = ((uint64_t)cz * kCellsPerAxis + (uint64_t)cy) * kCellsPerAxis + (uint64_t)cx;
}

// cell-sorted records: (X, Y, Z, sorted position) and, for the prefilter,
// the position relative to the node's minimum corner in FP32 (w = sorted
// position). Within a cell, records are in sorted order (the cell sort is
// stable).
__global__ void conf_gather_kernel(const LevelNode* __restrict__ nodes, PosParamsS pp, LevelBuffers lb, const uint32_t* __restrict__ cvals,
                                   int4* __restrict__ crec, float4* __restrict__ crf) {
	const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= lb.M) return;
	const LevelNode& nd = nodes[lb.node_of[j]];
	const uint32_t u = cvals[j];
	int4 r = lb.cq[nd.cand_off + u];
	r.w = (int32_t)u;
	crec[j] = r;
	crf[j] = make_float4((float)(qcoord(r.x, 0, pp) - nd.min[0]), (float)(qcoord(r.y, 1, pp) - nd.min[1]),
	                     (float)(qcoord(r.z, 2, pp) - nd.min[2]), __int_as_float((int)u));
}

// occupancy bitmap of a node's cells: 128 bits per (z, y) row, 4 words
constexpr int kRowWords = kCellsPerAxis / 32;
constexpr int64_t kBitmapWords = (int64_t)kCellsPerAxis * kCellsPerAxis * kRowWords;
constexpr int64_t kBitmapMinCandidates = 2048;  // smaller nodes probe the hash for every cell

__global__ void conf_bitmap_kernel(const int32_t* __restrict__ node_of, const uint64_t* __restrict__ ck, int64_t M,
                                   const int64_t* __restrict__ bm_off, uint32_t* __restrict__ bm) {
	const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= M) return;
	const int64_t off = bm_off[node_of[j]];
	if (off < 0) return;
	const uint64_t c = ck[j];
	const int cx = (int)(c % kCellsPerAxis);
	atomicOr(&bm[off + (int64_t)(c / kCellsPerAxis) * kRowWords + (cx >> 5)], 1u << (cx & 31));
}

__device__ __forceinline__ bool run_head(const LevelNode* nodes, const int32_t* node_of, const uint64_t* ck, int64_t j) {
	return j == nodes[node_of[j]].cand_off || ck[j] != ck[j - 1];
}

// occupied cells (runs) per node
__global__ void conf_count_runs_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ node_of, const uint64_t* __restrict__ ck,
                                       int64_t M, unsigned long long* __restrict__ node_runs) {
	const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	const bool h = j < M && run_head(nodes, node_of, ck, j);
	const int32_t node = j < M ? node_of[j] : -1;
	const unsigned peers = __match_any_sync(FULL, node);
	const unsigned heads = __ballot_sync(FULL, h) & peers;
	if (node >= 0 && heads && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&node_runs[node], (unsigned long long)__popc(heads));
}

// run tables, one per node: cell -> (first record, count). A node's table
// is its own region (tab_off, power-of-two tab_cap), so the probes of the
// candidates in flight stay within the few nodes being searched and hit L2.
__global__ void conf_insert_runs_kernel(const LevelNode* __restrict__ nodes, const uint8_t* __restrict__ use, const int32_t* __restrict__ node_of,
                                        const uint64_t* __restrict__ ck, int64_t M, RunSlot* __restrict__ table,
                                        const int64_t* __restrict__ tab_off, const int64_t* __restrict__ tab_cap, SampleStats* st) {
	const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= M) return;
	const int32_t node = node_of[j];
	if (!use[node] || !run_head(nodes, node_of, ck, j)) return;
	const int64_t end = nodes[node].cand_off + nodes[node].count;
	int64_t e = j + 1;
	while (e < end && ck[e] == ck[j]) e++;
	const uint64_t key = ck[j];
	RunSlot* tb = table + tab_off[node];
	const int64_t cap = tab_cap[node];
	uint64_t s = run_hash(key, cap);
	for (int64_t probe = 0; probe < cap; probe++) {
		const unsigned long long prev = atomicCAS((unsigned long long*)&tb[s].key, (unsigned long long)kEmptyRun, (unsigned long long)key);
		if (prev == kEmptyRun) {
			tb[s].start = (int32_t)(j - nodes[node].cand_off);
			tb[s].count = (int32_t)(e - j);
			return;
		}
		s = (s + 1) & (uint64_t)(cap - 1);
	}
	atomicAdd(&st->timeouts, 1ull);
}

__device__ __forceinline__ int2 find_run(const RunSlot* table, int64_t cap, uint64_t key) {
	uint64_t s = run_hash(key, cap);
	for (int64_t probe = 0; probe < cap; probe++) {
		const RunSlot r = table[s];
		if (r.key == key) return make_int2(r.start, r.count);
		if (r.key == kEmptyRun) break;
		s = (s + 1) & (uint64_t)(cap - 1);
	}
	return make_int2(0, 0);
}

// The search waits on dependent loads (bitmap row, run table, runs) and is
// near its issue limit: MINB resident blocks of 256 threads per SM (5: 48
// registers, 4: 64), GAPS skips the neighbour cells beyond the band. The
// variant is chosen by lists_variant() (measured; PCG_LISTS overrides).
template <int MODE, int MINB, bool GAPS>
__global__ void __launch_bounds__(256, MINB) conf_lists_kernel(const LevelNode* __restrict__ nodes, const uint8_t* __restrict__ use, PosParamsS pp,
                                                        LevelBuffers lb, const uint64_t* __restrict__ ck, const int4* __restrict__ crec,
                                                        const float4* __restrict__ crf, const RunSlot* __restrict__ table,
                                                        const int64_t* __restrict__ tab_off, const int64_t* __restrict__ tab_cap,
                                                        const int64_t* __restrict__ bm_off, const uint32_t* __restrict__ bm,
                                                        ConflictLists cl, SampleStats* st) {
	const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= lb.M) return;
	const int32_t node = lb.node_of[j];
	if (!use[node]) return;
	const LevelNode& nd = nodes[node];
	const int64_t co = nd.cand_off;
	const float4 mf = crf[j];
	const int32_t t = __float_as_int(mf.w);
	const double sp = nd.spacing, s2 = sp * sp;
	double lim = 0.0;
	if (MODE == 0) {
		// the early-exit bound of the acceptance kernels, same expression
		const double cd = sqrt(lb.keys[co + t]);
		const double limit = cd - sp;
		lim = limit * limit;
	}
	// node-relative FP32 coordinates: error far below the 1e-3 margin on s^2
	// (the bound on its error, derived for node-relative coordinates below
	// 128 spacings, holds while the FP64 coordinates themselves carry a
	// rounding error far below the spacing: |coordinate| < 1e6 spacings)
	double amax = 0.0;
	for (int a = 0; a < 3; a++) amax = fmax(amax, fmax(fabs(nd.min[a]), fabs(nd.max[a])));
	const bool pre32 = s2 > 1e-30 && s2 < 1e30 && amax < 1e6 * sp;
	const float s2hi = (float)(s2 * 1.001), s2lo = (float)(s2 * 0.999);
	unsigned escalated = 0;  // pairs inside the band, decided in FP64
	const uint64_t c = ck[j];
	const int cx = (int)(c % kCellsPerAxis), cy = (int)((c / kCellsPerAxis) % kCellsPerAxis), cz = (int)(c / (kCellsPerAxis * kCellsPerAxis));
	// the first kListInline entries go to the candidate's own slot (positions
	// past the list read as 0); the rest (rare) wait in a per-thread array
	// and take exactly their room in the pool once the search is done
	int32_t* inl = reinterpret_cast<int32_t*>(cl.inl + co + t);
	cl.inl[co + t] = make_int4(0, 0, 0, 0);
	int32_t rest[kListCap - kListInline];
	int n = 0;
	const int64_t boff = bm_off[node];
	const RunSlot* tb = table + tab_off[node];
	const int64_t cap = tab_cap[node];
	// gaps from the candidate to the faces it shares with the cells below
	// and above it on each axis: a neighbour cell whose nearest point is
	// at least the band's upper edge away holds no pair (with the
	// prefilter's margin over the FP32 error; nodes without the prefilter
	// visit every cell)
	const float cs = (float)(sp * 1.000001);
	auto gap2 = [&](int d, float v, int c) {
		const float g = d < 0 ? v - (float)c * cs : (float)(c + 1) * cs - v;
		return GAPS && pre32 && d != 0 && g > 0.f ? g * g : 0.f;
	};
#pragma unroll 1
	for (int dz = -1; dz <= 1; dz++) {
		const int qz = cz + dz;
		if (qz < 0 || qz >= kCellsPerAxis) continue;
		const float dz2 = gap2(dz, mf.z, cz);
		if (dz2 >= s2hi) continue;
#pragma unroll 1
		for (int dy = -1; dy <= 1; dy++) {
			const int qy = cy + dy;
			if (qy < 0 || qy >= kCellsPerAxis) continue;
			const float dzy2 = dz2 + gap2(dy, mf.y, cy);
			if (dzy2 >= s2hi) continue;
			// occupied cells among x = cx-1 .. cx+1 of this row
			uint32_t occ = 7u;
			if (boff >= 0) {
				const uint32_t* row = bm + boff + ((int64_t)qz * kCellsPerAxis + qy) * kRowWords;
				const int x0 = cx - 1;
				occ = 0;
				for (int b = 0; b < 3; b++) {
					const int qx = x0 + b;
					if (qx >= 0 && qx < kCellsPerAxis && ((row[qx >> 5] >> (qx & 31)) & 1u)) occ |= 1u << b;
				}
			}
			for (int dx = -1; dx <= 1; dx++) {
				const int qx = cx + dx;
				if (qx < 0 || qx >= kCellsPerAxis || !((occ >> (dx + 1)) & 1u)) continue;
				if (dzy2 + gap2(dx, mf.x, cx) >= s2hi) continue;
				const uint64_t cell = ((uint64_t)qz * kCellsPerAxis + (uint64_t)qy) * kCellsPerAxis + (uint64_t)qx;
				const int2 run = find_run(tb, cap, cell);
				const int4* rp = crec + co + run.x;
				const float4* rf = crf + co + run.x;
				for (int i = 0; i < run.y; i++) {
					const float4 qf = rf[i];
					const int32_t u = __float_as_int(qf.w);
					if (u >= t) break;  // a cell's records are in sorted order: only earlier candidates
					bool inside = false;
					if (pre32) {
						// FP32 decides outside the band s^2 (1 -/+ 1e-3), well clear
						// of its rounding error; pairs in the band go to FP64
						const float fx = qf.x - mf.x, fy = qf.y - mf.y, fz = qf.z - mf.z;
						const float d2 = fx * fx + fy * fy + fz * fz;
						if (d2 >= s2hi) continue;
						inside = d2 < s2lo;
					}
					if (!inside) {
						// the FP64 positions are recomputed here, not held in
						// registers through the search (pairs in the band are rare)
						const int4 q = rp[i];
						const int4 me = crec[j];
						const double ax = qcoord(q.x, 0, pp), ay = qcoord(q.y, 1, pp), az = qcoord(q.z, 2, pp);
						const double x = qcoord(me.x, 0, pp), y = qcoord(me.y, 1, pp), z = qcoord(me.z, 2, pp);
						// squaredDistance(point, candidate), sampler_poisson.h:117-125
						const double dx_ = ax - x, dy_ = ay - y, dz_ = az - z;
						escalated++;
						if (!(dx_ * dx_ + dy_ * dy_ + dz_ * dz_ < s2)) continue;
					}
					if (MODE == 0 && !(lb.keys[co + u] >= lim)) continue;
					if (n < kListInline) inl[n] = u;
					else if (n < kListCap) rest[n - kListInline] = u;
					n++;
				}
			}
		}
	}
	bool dense = n > kListCap;
	if (!dense && n > kListInline) {
		const int extra = n - kListInline;
		const unsigned long long at = atomicAdd(cl.pool_used, (unsigned long long)extra);
		if ((int64_t)(at + extra) <= cl.pool_cap) {
			cl.ovf_off[co + t] = (int32_t)at;
			for (int e = 0; e < extra; e++) cl.pool[at + e] = rest[e];
		} else {
			dense = true;  // the pool is full: the level builds its lists again with a larger pool
		}
	}
	cl.count[co + t] = (uint8_t)(dense ? kListDense : n);
	if (dense) cl.node_dense[node] = 1;
	const unsigned active = __activemask();
	const unsigned sum = __reduce_add_sync(active, (unsigned)(dense ? 0 : n));
	const unsigned esc = __reduce_add_sync(active, escalated);
	if ((int)(threadIdx.x & 31) == __ffs(active) - 1) {
		atomicAdd(&st->list_entries, (unsigned long long)sum);
		if (esc) atomicAdd(&st->escalated, (unsigned long long)esc);
	}
}

// 0: five blocks per SM with the cell skip, 1: four blocks with it, 2: five
// blocks without it; PCG_LISTS=<n> overrides the measured default
int lists_variant() {
	static const int v = [] {
		const char* e = std::getenv("PCG_LISTS");
		return e ? std::atoi(e) : kListsVariant;
	}();
	return v;
}

// st += the list build's own counters
__global__ void add_list_stats_kernel(SampleStats* st, const SampleStats* lst) {
	atomicAdd(&st->list_entries, lst->list_entries);
	atomicAdd(&st->escalated, lst->escalated);
	atomicAdd(&st->timeouts, lst->timeouts);
}

}  // namespace

void build_conflict_lists(int mode, const LevelNode* d_nodes, const std::vector<LevelNode>& ln, const std::vector<uint8_t>& use,
                          const PosParamsS& pp, LevelBuffers& lb, ConflictLists& cl, std::vector<uint8_t>& dense, SampleStats* st,
                          DeviceMem& mem) {
	const int K = (int)ln.size();
	const int64_t M = lb.M;
	dense.assign(K, 0);
	if (M == 0 || K == 0) return;
	cudaStream_t s = mem.stream();
	const unsigned blocks = (unsigned)ceil_div(M, 256);
	uint64_t* keys = mem.alloc<uint64_t>(M);
	conf_cell_keys_kernel<<<blocks, 256, 0, s>>>(d_nodes, pp, lb, keys);
	PCG_LAUNCHED();
	uint64_t* ck = mem.alloc<uint64_t>(M);
	uint32_t* cv = mem.alloc<uint32_t>(M);
	segmented_sort_pairs(ln, M, keys, nullptr, ck, cv, 0, 21, mem);
	mem.free(keys);
	int4* crec = mem.alloc<int4>(M);
	float4* crf = mem.alloc<float4>(M);
	conf_gather_kernel<<<blocks, 256, 0, s>>>(d_nodes, pp, lb, cv, crec, crf);
	PCG_LAUNCHED();
	mem.free(cv);
	unsigned long long* d_runs = mem.alloc<unsigned long long>(K);
	PCG_CUDA(cudaMemsetAsync(d_runs, 0, K * sizeof(unsigned long long), s));
	conf_count_runs_kernel<<<blocks, 256, 0, s>>>(d_nodes, lb.node_of, ck, M, d_runs);
	PCG_LAUNCHED();
	std::vector<unsigned long long> runs(K);
	PCG_CUDA(cudaMemcpyAsync(runs.data(), d_runs, K * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
	PCG_CUDA(cudaStreamSynchronize(s));
	mem.free(d_runs);
	// per-node tables at most half full
	std::vector<int64_t> tab(2 * (size_t)K, 0);  // offsets, then capacities
	int64_t slots = 0;
	for (int k = 0; k < K; k++) {
		int64_t cap = 0;
		if (use[k] && runs[k] > 0) {
			cap = 16;
			while (cap < 2 * (int64_t)runs[k]) cap <<= 1;
		}
		tab[k] = slots;
		tab[K + k] = cap;
		slots += cap;
	}
	int64_t* d_tab = mem.alloc<int64_t>(2 * (size_t)K);
	PCG_CUDA(cudaMemcpyAsync(d_tab, tab.data(), tab.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s));
	const int64_t* tab_off = d_tab;
	const int64_t* tab_cap = d_tab + K;
	RunSlot* table = mem.alloc<RunSlot>(slots > 0 ? slots : 1);
	if (slots > 0) PCG_CUDA(cudaMemsetAsync(table, 0xff, slots * sizeof(RunSlot), s));
	uint8_t* d_use = mem.alloc<uint8_t>(K);
	PCG_CUDA(cudaMemcpyAsync(d_use, use.data(), K, cudaMemcpyHostToDevice, s));
	conf_insert_runs_kernel<<<blocks, 256, 0, s>>>(d_nodes, d_use, lb.node_of, ck, M, table, tab_off, tab_cap, st);
	PCG_LAUNCHED();
	// occupancy bitmaps of the larger nodes
	std::vector<int64_t> bm_off(K, -1);
	int64_t bm_words = 0;
	for (int k = 0; k < K; k++)
		if (use[k] && ln[k].count >= kBitmapMinCandidates) { bm_off[k] = bm_words; bm_words += kBitmapWords; }
	int64_t* d_bm_off = mem.alloc<int64_t>(K);
	PCG_CUDA(cudaMemcpyAsync(d_bm_off, bm_off.data(), K * sizeof(int64_t), cudaMemcpyHostToDevice, s));
	uint32_t* bm = mem.alloc<uint32_t>(bm_words > 0 ? bm_words : 1);
	if (bm_words > 0) {
		PCG_CUDA(cudaMemsetAsync(bm, 0, bm_words * sizeof(uint32_t), s));
		conf_bitmap_kernel<<<blocks, 256, 0, s>>>(lb.node_of, ck, M, d_bm_off, bm);
		PCG_LAUNCHED();
	}
	cl.inl = mem.alloc<int4>(M);
	cl.ovf_off = mem.alloc<int32_t>(M);
	// entries past the inline ones: room for 8 more per candidate on
	// average (lists average about one entry; the top levels' dense nodes
	// need more than 4). When the lists need more, the build runs again
	// with a pool of the exact size they asked for. A pool the device cannot
	// hold is made smaller: the candidates it cannot take mark their nodes
	// dense, which keep the lookup kernels.
	auto alloc_pool = [&](int64_t want) {
		int64_t cap = std::max<int64_t>(want, 1);
		while (true) {
			try {
				cl.pool = mem.alloc<int32_t>(cap);
				cl.pool_cap = cap;
				return;
			} catch (const PcgError& e) {
				if (e.status != 3 || cap <= 4096) throw;  // 3: PCG_OOM
				cap /= 2;
			}
		}
	};
	alloc_pool(std::min<int64_t>((int64_t)M * 2 * kListInline, (int64_t)INT32_MAX));
	cl.pool_used = mem.alloc<unsigned long long>(1);
	cl.count = mem.alloc<uint8_t>(M);
	cl.node_dense = mem.alloc<uint8_t>(K);
	SampleStats* lst = mem.alloc<SampleStats>(1);
	for (int attempt = 0; attempt < 2; attempt++) {
		PCG_CUDA(cudaMemsetAsync(cl.pool_used, 0, sizeof(unsigned long long), s));
		PCG_CUDA(cudaMemsetAsync(cl.node_dense, 0, K, s));
		PCG_CUDA(cudaMemsetAsync(lst, 0, sizeof(SampleStats), s));
		auto run = [&](auto kernel) {
			kernel<<<blocks, 256, 0, s>>>(d_nodes, d_use, pp, lb, ck, crec, crf, table, tab_off, tab_cap, d_bm_off, bm, cl, lst);
		};
		const int v = lists_variant();
		if (mode == 0) {
			if (v == 1) run(conf_lists_kernel<0, 4, true>);
			else if (v == 2) run(conf_lists_kernel<0, 5, false>);
			else run(conf_lists_kernel<0, 5, true>);
		} else {
			if (v == 1) run(conf_lists_kernel<1, 4, true>);
			else if (v == 2) run(conf_lists_kernel<1, 5, false>);
			else run(conf_lists_kernel<1, 5, true>);
		}
		PCG_LAUNCHED();
		unsigned long long used = 0;
		PCG_CUDA(cudaMemcpyAsync(&used, cl.pool_used, sizeof(used), cudaMemcpyDeviceToHost, s));
		PCG_CUDA(cudaStreamSynchronize(s));
		if ((int64_t)used <= cl.pool_cap || attempt == 1 || (int64_t)used > (int64_t)INT32_MAX) break;
		mem.free(cl.pool);
		alloc_pool((int64_t)used);
	}
	add_list_stats_kernel<<<1, 1, 0, s>>>(st, lst);
	PCG_LAUNCHED();
	PCG_CUDA(cudaMemcpyAsync(dense.data(), cl.node_dense, K, cudaMemcpyDeviceToHost, s));
	PCG_CUDA(cudaStreamSynchronize(s));
	mem.free(lst);
	mem.free(d_use);
	mem.free(d_bm_off);
	mem.free(bm);
	mem.free(table);
	mem.free(d_tab);
	mem.free(crec);
	mem.free(crf);
	mem.free(ck);
}

void free_conflict_lists(ConflictLists& cl, DeviceMem& mem) {
	if (cl.inl) mem.free(cl.inl);
	if (cl.ovf_off) mem.free(cl.ovf_off);
	if (cl.pool) mem.free(cl.pool);
	if (cl.pool_used) mem.free(cl.pool_used);
	if (cl.count) mem.free(cl.count);
	if (cl.node_dense) mem.free(cl.node_dense);
	cl = ConflictLists{};
}

}  // namespace pcg
