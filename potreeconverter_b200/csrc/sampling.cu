// Sampler kernels. One launch covers one octree level across all of its
// inner nodes (the batched form) or a single node (the plain form). The
// candidates arrive sorted (segsort.cu, introsort.cu).
//
//  * greedy_kernel      -- the sequential acceptance scan of
//    sampler_poisson.h:133-245 (and the grid variant of
//    sampler_poisson_average.h:184-281), one warp per node, 32 candidates
//    per step. Each lane looks up conflicts among the already accepted
//    points through a per-node spatial hash (cells of two spacings, so 8
//    cells cover the spacing ball), conflicts inside the step come from
//    lane shuffles, and the 32 decisions are resolved in order. The
//    reference's early exit (accepted points closer to the centre than
//    |c| - s stop the scan) and its 10,001-check cap become two static
//    conditions on a conflicting accepted point a of candidate p:
//    key(a) >= (sqrt(key(p)) - s)^2, and at most 10,000 points accepted
//    after a. Together they give exactly the reference's decision.
//  * average_colors     -- poisson_average's colour sums
//    (sampler_poisson_average.h:357-416) in closed form: every rejected
//    candidate adds its colour to each accepted point within the spacing,
//    doubled when it precedes that point in sorted order (the reference
//    doubles an accepted point's running sum when its own turn comes), and
//    every accepted point adds twice its own colour.
//  * random_accept      -- sampler_random.h:146-178: a point is accepted if
//    its child holds < 100 points, or if it is the first point of its
//    128^3 cell that is eligible; first-eligible is an atomicMin per cell.
//  * shuffle_leaves     -- std::shuffle(..., std::default_random_engine(seed))
//    of sampler_random.h:97-118, libstdc++'s two-draws-per-call variant.

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math_constants.h>

#include <cstdio>
#include <cstdlib>

#include "devutil.cuh"
#include "sampling.h"
#include "tuned_schedule.h"

namespace pcg {

namespace {

constexpr uint64_t EMPTY_KEY = ~0ull;

// ---------------------------------------------------------------- gather
// one CTA per piece of kGatherPiece ids of an item (piece_item / piece_start
// give the item and the piece's first id in it)
__global__ void gather_kernel(const GatherItem* __restrict__ items, const int32_t* __restrict__ piece_item,
                              const int64_t* __restrict__ piece_start, LevelBuffers lb) {
	const GatherItem it = items[piece_item[blockIdx.x]];
	const int64_t t0 = piece_start[blockIdx.x];
	const int64_t t1 = t0 + kGatherPiece < it.count ? t0 + kGatherPiece : it.count;
	for (int64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
		int64_t j = it.dst_off + t;
		lb.ids[j] = it.src_ids[t];
		if (lb.cols) lb.cols[j] = it.src_cols ? it.src_cols[t] : 0ull;
		if (lb.rec) lb.rec[j] = it.src_rec[t];
		lb.child[j] = (uint8_t)it.child;
		lb.node_of[j] = it.node;
		lb.count_in_child[j] = (int32_t)it.count;
	}
}

__device__ __forceinline__ void point_xyz(const int32_t* X, const int32_t* Y, const int32_t* Z, const PosParamsS& pp, uint32_t id,
                                          double& x, double& y, double& z) {
	// (xyz[0] * scale.x) + offset.x, sampler_poisson.h:99-101
	x = ((double)X[id] * pp.scale[0]) + pp.offset[0];
	y = ((double)Y[id] * pp.scale[1]) + pp.offset[1];
	z = ((double)Z[id] * pp.scale[2]) + pp.offset[2];
}

// squared distance to the node centre, center = (min + max) * 0.5
// (sampler_poisson.h:127, 183-203); the one expression every kernel uses
__device__ __forceinline__ double center_key(const LevelNode& nd, double x, double y, double z) {
	double cx = (nd.min[0] + nd.max[0]) * 0.5, cy = (nd.min[1] + nd.max[1]) * 0.5, cz = (nd.min[2] + nd.max[2]) * 0.5;
	double ax = x - cx, ay = y - cy, az = z - cz;
	return ax * ax + ay * ay + az * az;
}

__global__ void keys_kernel(const LevelNode* __restrict__ nodes, PosParamsS pp, LevelBuffers lb) {
	int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= lb.M) return;
	const LevelNode& nd = nodes[lb.node_of[j]];
	const int4 r = lb.rec[j];
	// (xyz * scale) + offset, sampler_poisson.h:99-101
	const double x = ((double)r.x * pp.scale[0]) + pp.offset[0];
	const double y = ((double)r.y * pp.scale[1]) + pp.offset[1];
	const double z = ((double)r.z * pp.scale[2]) + pp.offset[2];
	lb.keys[j] = center_key(nd, x, y, z);
	lb.perm[j] = (int32_t)(j - nd.cand_off);
}

__global__ void gather_records_kernel(const uint32_t* __restrict__ ids, int64_t n, const int32_t* __restrict__ X,
                                      const int32_t* __restrict__ Y, const int32_t* __restrict__ Z, int4* __restrict__ rec) {
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint32_t id = ids[i];
	rec[i] = make_int4(X[id], Y[id], Z[id], 0);
}

// (X, Y, Z, 0) of every point, so that a gather in a scattered order reads
// one 16-byte record per point instead of three 4-byte words from three arrays
__global__ void pack_records_kernel(int64_t n, const int32_t* __restrict__ X, const int32_t* __restrict__ Y, const int32_t* __restrict__ Z,
                                    int4* __restrict__ xyz) {
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) xyz[i] = make_int4(X[i], Y[i], Z[i], 0);
}

__global__ void gather_packed_kernel(const uint32_t* __restrict__ ids, int64_t n, const int4* __restrict__ xyz, int4* __restrict__ rec) {
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) rec[i] = xyz[ids[i]];
}

// sorted candidate records: (X, Y, Z, local index) at each sorted position
__global__ void cand_records_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ X, const int32_t* __restrict__ Y,
                                    const int32_t* __restrict__ Z, LevelBuffers lb) {
	const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= lb.M) return;
	const int64_t off = nodes[lb.node_of[j]].cand_off;
	const int32_t local = lb.perm[j];
	int4 r = lb.rec[off + local];
	r.w = local;
	lb.cq[j] = r;
}

// --------------------------------------------------------------- hashing
__device__ __forceinline__ uint64_t hash_slot(uint64_t k, int64_t cap) {
	return ((k * 0x9E3779B97F4A7C15ull) >> 17) & (uint64_t)(cap - 1);
}

// cells of 2*spacing*(1+1e-6): points closer than the spacing are in
// neighbouring cells along each axis, and a candidate needs 8 cells
struct CellGrid {
	double min[3];
	double inv;
};

__device__ __forceinline__ void cell_of(const CellGrid& g, double x, double y, double z, int c[3], double fr[3]) {
	double u[3] = {(x - g.min[0]) * g.inv, (y - g.min[1]) * g.inv, (z - g.min[2]) * g.inv};
	for (int a = 0; a < 3; a++) {
		double fl = floor(u[a]);
		fl = fl < -1000.0 ? -1000.0 : (fl > 1000.0 ? 1000.0 : fl);
		c[a] = (int)fl;
		fr[a] = u[a] - fl;
	}
}

__device__ __forceinline__ uint64_t cell_key(int cx, int cy, int cz) {
	return ((uint64_t)(cx + 1024) << 22) | ((uint64_t)(cy + 1024) << 11) | (uint64_t)(cz + 1024);
}

__device__ __forceinline__ int32_t hash_find(const uint64_t* keys, const int32_t* heads, int64_t cap, uint64_t k) {
	uint64_t s = hash_slot(k, cap);
	for (int64_t probe = 0; probe < cap; probe++) {
		uint64_t kk = keys[s];
		if (kk == k) return heads[s];
		if (kk == EMPTY_KEY) return -1;
		s = (s + 1) & (uint64_t)(cap - 1);
	}
	return -1;
}

// inserts item into the cell's list; returns false if the table is full
__device__ __forceinline__ bool hash_push(uint64_t* keys, int32_t* heads, int32_t* next, int64_t cap, uint64_t k, int32_t item) {
	uint64_t s = hash_slot(k, cap);
	for (int64_t probe = 0; probe < cap; probe++) {
		uint64_t prev = atomicCAS((unsigned long long*)&keys[s], (unsigned long long)EMPTY_KEY, (unsigned long long)k);
		if (prev == EMPTY_KEY || prev == k) {
			next[item] = atomicExch(&heads[s], item);
			return true;
		}
		s = (s + 1) & (uint64_t)(cap - 1);
	}
	return false;
}

// ------------------------------------------------------------- greedy
struct GreedyArgs {
	uint64_t* hkeys;
	int32_t* hheads;
	double* axyz;   // accepted positions, 3 per slot (slot = cand_off + rank)
	double* akey;   // accepted sort keys
	int32_t* anext; // per-cell list links
	int32_t* apos;  // accepted sorted positions
};

__device__ __forceinline__ double sqdist(double ax, double ay, double az, double bx, double by, double bz) {
	// squaredDistance(point, candidate), sampler_poisson.h:117-125
	double dx = ax - bx, dy = ay - by, dz = az - bz;
	return dx * dx + dy * dy + dz * dz;
}

template <int MODE, bool GUARD>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) greedy_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ order,
                                                                    int node_begin, int node_end, const int32_t* __restrict__ X,
                                                                    const int32_t* __restrict__ Y, const int32_t* __restrict__ Z,
                                                                    PosParamsS pp, LevelBuffers lb, GreedyArgs ga, SampleStats* st,
                                                                    int* next_node) {
	const int lane = threadIdx.x & 31;
	const uint32_t lt = lanemask_lt();
	while (true) {
		int idx = 0;
		if (lane == 0) idx = atomicAdd(next_node, 1);
		idx = __shfl_sync(FULL, idx, 0) + node_begin;
		if (idx >= node_end) break;
		const LevelNode nd = nodes[order[idx]];
		const int64_t n = nd.count, co = nd.cand_off;
		uint64_t* hk = ga.hkeys + nd.hash_off;
		int32_t* hh = ga.hheads + nd.hash_off;
		for (int64_t s = lane; s < nd.hash_cap; s += 32) { hk[s] = EMPTY_KEY; hh[s] = -1; }
		__syncwarp();
		const double sp = nd.spacing;
		const double s2 = sp * sp;
		const double cx = (nd.min[0] + nd.max[0]) * 0.5, cy = (nd.min[1] + nd.max[1]) * 0.5, cz = (nd.min[2] + nd.max[2]) * 0.5;
		CellGrid g;
		g.min[0] = nd.min[0]; g.min[1] = nd.min[1]; g.min[2] = nd.min[2];
		g.inv = 1.0 / (2.0 * sp * 1.000001);
		// FP32 guard band: node-relative float coordinates decide pairs whose
		// squared distance is clearly away from s^2; the rest are re-decided
		// in FP64 exactly as the reference computes them.
		const float s2f = (float)s2;
		const float lo = s2f * (1.0f - 2e-3f), hi = s2f * (1.0f + 2e-3f);
		int64_t cnt = 0;  // accepted so far
		unsigned long long escalated = 0;
		for (int64_t b0 = 0; b0 < n; b0 += 32) {
			const int64_t t = b0 + lane;
			const bool valid = t < n;
			double x = 0, y = 0, z = 0, key = 0, lim = -CUDART_INF;
			int32_t local = 0;
			if (valid) {
				local = lb.perm[co + t];
				point_xyz(X, Y, Z, pp, lb.ids[co + local], x, y, z);
				key = lb.keys[co + t];
				if (MODE == 0) {
					// cd = sqrt(cdd); limit = cd - spacing (sampler_poisson.h:135-141)
					double cd = sqrt(key);
					double limit = cd - sp;
					lim = limit * limit;
				}
			}
			const float xf = (float)(x - cx), yf = (float)(y - cy), zf = (float)(z - cz);
			// 1) conflicts with points accepted before this step
			int64_t maxrank = -1;
			if (valid) {
				int c[3];
				double fr[3];
				cell_of(g, x, y, z, c, fr);
				int o[3];
				for (int a = 0; a < 3; a++) o[a] = fr[a] < 0.5 ? -1 : 1;
#pragma unroll
				for (int q = 0; q < 8; q++) {
					int qx = c[0] + ((q & 4) ? o[0] : 0), qy = c[1] + ((q & 2) ? o[1] : 0), qz = c[2] + ((q & 1) ? o[2] : 0);
					int32_t r = hash_find(hk, hh, nd.hash_cap, cell_key(qx, qy, qz));
					int64_t guard = 0;
					while (r >= 0 && guard++ <= n) {
						const int64_t slot = co + r;
						if (MODE == 1 || ga.akey[slot] >= lim) {
							double ax = ga.axyz[3 * slot], ay = ga.axyz[3 * slot + 1], az = ga.axyz[3 * slot + 2];
							bool conflict;
							if (GUARD) {
								float dxf = (float)(ax - cx) - xf, dyf = (float)(ay - cy) - yf, dzf = (float)(az - cz) - zf;
								float ddf = dxf * dxf + dyf * dyf + dzf * dzf;
								if (ddf < lo) conflict = true;
								else if (ddf > hi) conflict = false;
								else { conflict = sqdist(ax, ay, az, x, y, z) < s2; escalated++; }
							} else {
								conflict = sqdist(ax, ay, az, x, y, z) < s2;
							}
							if (conflict && r > maxrank) maxrank = r;
						}
						r = ga.anext[slot];
					}
					if (guard > n + 1) atomicAdd(&st->timeouts, 1ull);
				}
			}
			// 2) conflicts inside the step: earlier lanes that would be
			//    accepted before this candidate
			uint32_t mask = 0;
			for (int j = 0; j < 32; j++) {
				double xj = __shfl_sync(FULL, x, j), yj = __shfl_sync(FULL, y, j), zj = __shfl_sync(FULL, z, j);
				double kj = __shfl_sync(FULL, key, j);
				if (valid && j < lane) {
					if (MODE == 1 || kj >= lim) {
						if (sqdist(xj, yj, zj, x, y, z) < s2) mask |= 1u << j;
					}
				}
			}
			// 3) decisions in sorted order
			uint32_t accmask = 0;
			const int nvalid = (int)((n - b0) < 32 ? (n - b0) : 32);
			bool acc = false;
			for (int i = 0; i < nvalid; i++) {
				bool dec = false;
				if (lane == i) {
					int64_t m_i = __popc(accmask);
					bool old_conflict = maxrank >= 0 && (MODE == 1 || maxrank >= cnt + m_i - 10001);
					bool new_conflict = (mask & accmask) != 0;
					dec = !old_conflict && !new_conflict;
					acc = dec;
				}
				dec = __shfl_sync(FULL, dec, i);
				if (dec) accmask |= 1u << i;
			}
			// 4) publish accepted points
			if (valid) {
				lb.accepted[co + local] = acc ? 1 : 0;
				if (acc) {
					int32_t rank = (int32_t)(cnt + __popc(accmask & lt));
					lb.acc_rank[co + local] = rank;
					const int64_t slot = co + rank;
					ga.axyz[3 * slot] = x;
					ga.axyz[3 * slot + 1] = y;
					ga.axyz[3 * slot + 2] = z;
					ga.akey[slot] = key;
					ga.apos[slot] = (int32_t)t;
					int c[3];
					double fr[3];
					cell_of(g, x, y, z, c, fr);
					if (!hash_push(hk, hh, ga.anext + co, nd.hash_cap, cell_key(c[0], c[1], c[2]), rank)) atomicAdd(&st->timeouts, 1ull);
				}
			}
			cnt += __popc(accmask);
			__syncwarp();
		}
		if (GUARD) {
			for (int o = 16; o > 0; o >>= 1) escalated += __shfl_down_sync(FULL, escalated, o);
			if (lane == 0 && escalated) atomicAdd(&st->escalated, escalated);
		}
	}
}

// --------------------------------------------------- poisson_average colours
__global__ void average_colors_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ X, const int32_t* __restrict__ Y,
                                      const int32_t* __restrict__ Z, PosParamsS pp, LevelBuffers lb, GreedyArgs ga,
                                      long long* __restrict__ sums) {
	int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= lb.M) return;
	const LevelNode& nd = nodes[lb.node_of[j]];
	const int64_t co = nd.cand_off;
	const uint64_t col = lb.cols[j];
	const long long r = (long long)(col & 0xffff), g = (long long)((col >> 16) & 0xffff), b = (long long)((col >> 32) & 0xffff);
	if (lb.accepted[j]) {
		long long* s = sums + 4 * (co + lb.acc_rank[j]);
		atomicAdd((unsigned long long*)&s[0], (unsigned long long)(2 * r));
		atomicAdd((unsigned long long*)&s[1], (unsigned long long)(2 * g));
		atomicAdd((unsigned long long*)&s[2], (unsigned long long)(2 * b));
		atomicAdd((unsigned long long*)&s[3], 2ull);
		return;
	}
	double x, y, z;
	point_xyz(X, Y, Z, pp, lb.ids[j], x, y, z);
	const double s2 = nd.spacing * nd.spacing;
	const int32_t my_pos = lb.pos[j];
	CellGrid gr;
	gr.min[0] = nd.min[0]; gr.min[1] = nd.min[1]; gr.min[2] = nd.min[2];
	gr.inv = 1.0 / (2.0 * nd.spacing * 1.000001);
	int c[3];
	double fr[3];
	cell_of(gr, x, y, z, c, fr);
	int o[3];
	for (int a = 0; a < 3; a++) o[a] = fr[a] < 0.5 ? -1 : 1;
	const uint64_t* hk = ga.hkeys + nd.hash_off;
	const int32_t* hh = ga.hheads + nd.hash_off;
	for (int q = 0; q < 8; q++) {
		int qx = c[0] + ((q & 4) ? o[0] : 0), qy = c[1] + ((q & 2) ? o[1] : 0), qz = c[2] + ((q & 1) ? o[2] : 0);
		int32_t a = hash_find(hk, hh, nd.hash_cap, cell_key(qx, qy, qz));
		int64_t guard = 0;
		while (a >= 0 && guard++ <= nd.count) {
			const int64_t slot = co + a;
			if (sqdist(ga.axyz[3 * slot], ga.axyz[3 * slot + 1], ga.axyz[3 * slot + 2], x, y, z) < s2) {
				long long f = my_pos < ga.apos[slot] ? 2 : 1;
				long long* s = sums + 4 * slot;
				atomicAdd((unsigned long long*)&s[0], (unsigned long long)(f * r));
				atomicAdd((unsigned long long*)&s[1], (unsigned long long)(f * g));
				atomicAdd((unsigned long long*)&s[2], (unsigned long long)(f * b));
				atomicAdd((unsigned long long*)&s[3], (unsigned long long)f);
			}
			a = ga.anext[slot];
		}
	}
}

__global__ void average_finish_kernel(const LevelNode* __restrict__ nodes, LevelBuffers lb, const long long* __restrict__ sums) {
	int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= lb.M || !lb.accepted[j]) return;
	const int64_t slot = nodes[lb.node_of[j]].cand_off + lb.acc_rank[j];
	const long long* s = sums + 4 * slot;
	// rgbTarget = p.r / p.w (sampler_poisson_average.h:443-445)
	uint64_t r = (uint16_t)(s[0] / s[3]), g = (uint16_t)(s[1] / s[3]), b = (uint16_t)(s[2] / s[3]);
	lb.cols[j] = r | (g << 16) | (b << 32);
}

// ---------------------------------------------------------------- random
__device__ __forceinline__ void random_cell(const LevelNode& nd, double x, double y, double z, int64_t& index, double& distance) {
	// toCellIndex, sampler_random.h:64-87
	const double G = 128.0;
	double sx = nd.max[0] - nd.min[0], sy = nd.max[1] - nd.min[1], sz = nd.max[2] - nd.min[2];
	double nx = (x - nd.min[0]) / sx, ny = (y - nd.min[1]) / sy, nz = (z - nd.min[2]) / sz;
	double lx = 2.0 * fmod(G * nx, 1.0) - 1.0;
	double ly = 2.0 * fmod(G * ny, 1.0) - 1.0;
	double lz = 2.0 * fmod(G * nz, 1.0) - 1.0;
	distance = sqrt(lx * lx + ly * ly + lz * lz);
	int64_t cx = (int64_t)(G * nx), cy = (int64_t)(G * ny), cz = (int64_t)(G * nz);
	cx = cx < 0 ? 0 : (cx > 127 ? 127 : cx);
	cy = cy < 0 ? 0 : (cy > 127 ? 127 : cy);
	cz = cz < 0 ? 0 : (cz > 127 ? 127 : cz);
	index = cx + cy * 128 + cz * 128 * 128;
}

__global__ void random_first_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ X, const int32_t* __restrict__ Y,
                                    const int32_t* __restrict__ Z, PosParamsS pp, LevelBuffers lb, uint64_t* hkeys, int32_t* hvals,
                                    SampleStats* st) {
	int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= lb.M) return;
	const LevelNode& nd = nodes[lb.node_of[j]];
	double x, y, z;
	point_xyz(X, Y, Z, pp, lb.ids[j], x, y, z);
	int64_t index;
	double distance;
	random_cell(nd, x, y, z, index, distance);
	const double all = sqrt(3.0);
	bool small = lb.count_in_child[j] < 100;
	bool dist_ok = distance < 0.7 * all;
	if (!(small || dist_ok)) return;
	uint64_t* hk = hkeys + nd.hash_off;
	int32_t* hv = hvals + nd.hash_off;
	uint64_t k = (uint64_t)index;
	uint64_t s = hash_slot(k, nd.hash_cap);
	const int32_t me = (int32_t)(j - nd.cand_off);
	for (int64_t probe = 0; probe < nd.hash_cap; probe++) {
		uint64_t prev = atomicCAS((unsigned long long*)&hk[s], (unsigned long long)EMPTY_KEY, (unsigned long long)k);
		if (prev == EMPTY_KEY || prev == k) {
			atomicMin(&hv[s], me);
			return;
		}
		s = (s + 1) & (uint64_t)(nd.hash_cap - 1);
	}
	atomicAdd(&st->timeouts, 1ull);
}

__global__ void random_accept_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ X, const int32_t* __restrict__ Y,
                                     const int32_t* __restrict__ Z, PosParamsS pp, LevelBuffers lb, const uint64_t* hkeys,
                                     const int32_t* hvals) {
	int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= lb.M) return;
	const LevelNode& nd = nodes[lb.node_of[j]];
	double x, y, z;
	point_xyz(X, Y, Z, pp, lb.ids[j], x, y, z);
	int64_t index;
	double distance;
	random_cell(nd, x, y, z, index, distance);
	const double all = sqrt(3.0);
	bool small = lb.count_in_child[j] < 100;
	bool dist_ok = distance < 0.7 * all;
	bool acc = small;
	if (!acc && dist_ok) {
		int32_t first = hash_find(hkeys + nd.hash_off, hvals + nd.hash_off, nd.hash_cap, (uint64_t)index);
		acc = first == (int32_t)(j - nd.cand_off);
	}
	lb.accepted[j] = acc ? 1 : 0;
}

__global__ void clear_hash_kernel(uint64_t* keys, int32_t* vals, int64_t n, int32_t fill) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) { keys[i] = EMPTY_KEY; vals[i] = fill; }
}

// --------------------------------------------------------------- shuffle
// std::default_random_engine = minstd_rand0 (16807, 0, 2^31 - 1)
struct MinStd {
	uint64_t x;
	__device__ explicit MinStd(uint32_t seed) {
		uint64_t s = (uint64_t)seed % 2147483647ull;
		x = s == 0 ? 1 : s;
	}
	__device__ uint64_t operator()() {
		x = (x * 16807ull) % 2147483647ull;
		return x;
	}
};

// uniform_int_distribution<unsigned long>{a, b}(minstd), downscaling branch
__device__ __forceinline__ uint64_t uniform(MinStd& g, uint64_t a, uint64_t b) {
	const uint64_t urngrange = 2147483646ull - 1ull;
	const uint64_t urange = b - a;
	uint64_t ret;
	if (urngrange > urange) {
		const uint64_t uerange = urange + 1;
		const uint64_t scaling = urngrange / uerange;
		const uint64_t past = uerange * scaling;
		do ret = g() - 1ull; while (ret >= past);
		ret /= scaling;
	} else {
		ret = g() - 1ull;  // urange == urngrange; larger ranges do not occur (n < 46341)
	}
	return ret + a;
}

__device__ void std_shuffle(int32_t* v, int64_t n, uint32_t seed) {
	if (n == 0) return;
	MinStd g(seed);
	const uint64_t urngrange = 2147483645ull;
	const uint64_t urange = (uint64_t)n;
	if (urngrange / urange >= urange) {
		int64_t i = 1;
		if ((urange % 2) == 0) {
			int64_t k = (int64_t)uniform(g, 0, 1);
			int32_t t = v[i]; v[i] = v[k]; v[k] = t;
			i++;
		}
		while (i != n) {
			const uint64_t swap_range = (uint64_t)i + 1;
			uint64_t xx = uniform(g, 0, swap_range * (swap_range + 1) - 1);
			int64_t p1 = (int64_t)(xx / (swap_range + 1)), p2 = (int64_t)(xx % (swap_range + 1));
			int32_t t = v[i]; v[i] = v[p1]; v[p1] = t;
			i++;
			t = v[i]; v[i] = v[p2]; v[p2] = t;
			i++;
		}
	} else {
		for (int64_t i = 1; i < n; i++) {
			int64_t k = (int64_t)uniform(g, 0, (uint64_t)i);
			int32_t t = v[i]; v[i] = v[k]; v[k] = t;
		}
	}
}

__global__ void shuffle_leaves_kernel(const int64_t* __restrict__ off, const int64_t* __restrict__ cnt, int num, const uint32_t* __restrict__ in,
                                      uint32_t* __restrict__ out, int32_t* scratch, uint32_t seed) {
	int l = blockIdx.x * blockDim.x + threadIdx.x;
	if (l >= num) return;
	const int64_t o = off[l], n = cnt[l];
	int32_t* idx = scratch + o;
	for (int64_t i = 0; i < n; i++) idx[i] = (int32_t)i;
	std_shuffle(idx, n, seed);
	// buffer[indices[i]] = points[i] (sampler_random.h:106-115)
	for (int64_t i = 0; i < n; i++) out[o + idx[i]] = in[o + i];
}

__global__ void shuffle_single_kernel(int64_t n, uint32_t seed, int32_t* perm) {
	for (int64_t i = 0; i < n; i++) perm[i] = (int32_t)i;
	std_shuffle(perm, n, seed);
}

// ============================================ one CTA per large node
// Nodes with many candidates (upper octree levels, dense 3D data) would keep
// a single warp busy for a long time while the GPU idles. They get a whole
// CTA, which decides 512 candidates per round.

// Greedy acceptance for a large node, one CTA, 512 candidates per round:
//  A. each thread looks up its candidate's conflicts among the points
//     accepted in earlier rounds. They live in a dense grid over the node
//     box: 64^3 cells of two spacings, each one 128-byte line holding the
//     count and up to 7 accepted points inline as (X, Y, Z, rank) -- the
//     quantized coordinates, from which the FP64 position and key are
//     recomputed bit for bit -- with an overflow list beyond that. The
//     eight cells around a candidate are fetched as independent 64-byte
//     loads, so a lookup costs one memory latency, not a chain per point;
//  B. conflicts among the round's own candidates are found through a shared
//     memory hash of the round (earlier candidates within the spacing);
//  C. decisions: parallel passes decide every candidate whose earlier
//     conflicts are all decided (accepted once none of them is accepted,
//     rejected once one is); warp 0 then decides what is left in sorted
//     order -- candidates whose old conflict sits at the edge of the
//     10,001-check window, which depends on how many were accepted before;
//  D. the round's accepted points get their ranks and enter the grid.
// The grid starts empty; at the end of its node a CTA empties the cells it
// filled, so the next node on the same slot finds it clean.
constexpr int kRound = kBigThreads;
constexpr int kRoundHash = 2 * kRound;
constexpr int kMaxLocal = 12;
constexpr int kGridDim = 64;  // node box = 128 spacings = 64 cells of 2 spacings
constexpr int64_t kGridCells = (int64_t)kGridDim * kGridDim * kGridDim;
constexpr int kCellSlots = 7;
constexpr int32_t kEmptyCell = -1;

struct alignas(128) AccCell {
	int32_t count;
	int32_t pad[3];
	int4 slot[kCellSlots];  // (X, Y, Z, rank)
};
static_assert(sizeof(AccCell) == 128, "one cache line per cell");

struct GridArena {
	AccCell* cells;  // kGridCells per CTA slot
	int32_t* ovf;    // overflow list heads, kGridCells per CTA slot
	int32_t* link;   // overflow list links, one per candidate (cand_off + rank)
	int4* accq;      // accepted points in rank order (cand_off + rank): X, Y, Z
};

struct RoundShared {
	double x[kRound], y[kRound], z[kRound], key[kRound], lim[kRound];
	int32_t maxrank[kRound];
	int32_t local[kRound];
	int32_t hkey[kRoundHash];
	int32_t hhead[kRoundHash];
	int16_t hnext[kRound];
	int16_t conf[kRound][kMaxLocal];
	uint8_t nconf[kRound];
	uint8_t state[kRound];   // 0 undecided, 1 accepted, 2 rejected
	uint8_t old[kRound];     // old-window status: 0 no conflict, 1 conflict, 2 depends on the count
	int32_t cnt;             // accepted before this round
	int32_t changed;
	unsigned long long warp_sums[kBigWarps];
};

__device__ __forceinline__ uint32_t round_slot(int32_t k) { return ((uint32_t)k * 0x9E3779B1u) >> (32 - 10); }
static_assert(kRoundHash == 1024, "round_slot yields 10 bits");

// 10 bits per axis: cells -512..511 (a node's points lie in cells 0..63)
__device__ __forceinline__ int32_t round_cell_key(int cx, int cy, int cz) {
	return ((cx + 512) << 20) | ((cy + 512) << 10) | (cz + 512);
}
__device__ __forceinline__ bool round_cell_ok(int cx, int cy, int cz) {
	return cx >= -512 && cx < 512 && cy >= -512 && cy < 512 && cz >= -512 && cz < 512;
}

__device__ __forceinline__ int grid_clamp(int c) { return c < 0 ? 0 : (c >= kGridDim ? kGridDim - 1 : c); }
__device__ __forceinline__ int64_t grid_index(int cx, int cy, int cz) {
	return ((int64_t)grid_clamp(cz) * kGridDim + grid_clamp(cy)) * kGridDim + grid_clamp(cx);
}

// conflict test of candidate (x, y, z) against an accepted point stored as
// quantized (X, Y, Z, rank): within the spacing and, for poisson, not behind
// the early-exit bound lim (sampler_poisson.h:150-167)
struct SlotTest {
	float sf[3];   // scale as float, for the prefilter
	float s2hi;    // s^2 (1 + 1e-3) as float
	bool pre32;    // prefilter usable: small quantized extent, s^2 in float range
};

template <int MODE>
__device__ __forceinline__ void test_slot(const int4& q, const int4& me, const SlotTest& T, const PosParamsS& pp, const LevelNode& nd, double x,
                                          double y, double z, double s2, double lim, int32_t& maxrank) {
	if (q.w <= maxrank) return;  // cannot raise the maximum
	if (T.pre32) {
		// FP32 distance from exact integer deltas: rules out every point
		// farther than the spacing by a margin far above its rounding error
		const float fx = (float)(q.x - me.x) * T.sf[0], fy = (float)(q.y - me.y) * T.sf[1], fz = (float)(q.z - me.z) * T.sf[2];
		if (fx * fx + fy * fy + fz * fz >= T.s2hi) return;
	}
	const double ax = ((double)q.x * pp.scale[0]) + pp.offset[0];
	const double ay = ((double)q.y * pp.scale[1]) + pp.offset[1];
	const double az = ((double)q.z * pp.scale[2]) + pp.offset[2];
	if (sqdist(ax, ay, az, x, y, z) < s2) {
		if (MODE == 1 || center_key(nd, ax, ay, az) >= lim) maxrank = q.w;
	}
}

template <int MODE>
__global__ void __launch_bounds__(kBigThreads) greedy_big_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ order, int node_begin,
                                                                PosParamsS pp, LevelBuffers lb, GreedyArgs ga, GridArena arena, SampleStats* st) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	RoundShared& R = *reinterpret_cast<RoundShared*>(smem_raw);
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const LevelNode nd = nodes[order[node_begin + blockIdx.x]];
	const int64_t n = nd.count, co = nd.cand_off;
	AccCell* cells = arena.cells + (int64_t)blockIdx.x * kGridCells;
	int32_t* ovf = arena.ovf + (int64_t)blockIdx.x * kGridCells;
	uint64_t* hk = ga.hkeys + nd.hash_off;
	int32_t* hh = ga.hheads + nd.hash_off;
	if (MODE == 1) {
		// poisson_average's colour pass finds accepted points through the hash
		for (int64_t i = tid; i < nd.hash_cap; i += kBigThreads) { hk[i] = EMPTY_KEY; hh[i] = -1; }
	}
	if (tid == 0) R.cnt = 0;
	__syncthreads();
	const double sp = nd.spacing, s2 = sp * sp;
	CellGrid g;
	g.min[0] = nd.min[0]; g.min[1] = nd.min[1]; g.min[2] = nd.min[2];
	g.inv = 1.0 / (2.0 * sp * 1.000001);
	SlotTest T;
	{
		bool ok = s2 > 1e-30 && s2 < 1e30;
		for (int a = 0; a < 3; a++) {
			T.sf[a] = (float)pp.scale[a];
			// all points of the node lie in its box: integer deltas stay below 2^23
			ok = ok && pp.scale[a] > 0.0 && (nd.max[a] - nd.min[a]) / pp.scale[a] < 8.0e6;
		}
		T.s2hi = (float)(s2 * 1.001);
		T.pre32 = ok;
	}
	unsigned long long n_past3 = 0, n_ovf = 0;
	for (int64_t r0 = 0; r0 < n; r0 += kRound) {
		const int64_t t = r0 + tid;
		const bool valid = t < n;
		const int nr = (int)((n - r0) < kRound ? (n - r0) : kRound);
		const int32_t cnt0 = R.cnt;
		// ---- A
		long long clk0 = clock64();
		double x = 0, y = 0, z = 0, key = 0, lim = -CUDART_INF;
		int32_t local = 0, maxrank = -1;
		int4 me = make_int4(0, 0, 0, 0);
		int c[3] = {0, 0, 0}, o[3] = {1, 1, 1};
		if (valid) {
			me = lb.cq[co + t];
			local = me.w;
			x = ((double)me.x * pp.scale[0]) + pp.offset[0];
			y = ((double)me.y * pp.scale[1]) + pp.offset[1];
			z = ((double)me.z * pp.scale[2]) + pp.offset[2];
			key = lb.keys[co + t];
			if (MODE == 0) {
				double cd = sqrt(key);
				double limit = cd - sp;
				lim = limit * limit;
			}
			double fr[3];
			cell_of(g, x, y, z, c, fr);
			for (int a = 0; a < 3; a++) o[a] = fr[a] < 0.5 ? -1 : 1;
#pragma unroll
			for (int h = 0; h < 2; h++) {
				// four cells at a time: count and the first three points in one 64-byte read each
				int64_t cidx[4];
				int4 v[4][4];
#pragma unroll
				for (int q = 0; q < 4; q++) {
					const int qq = 4 * h + q;
					cidx[q] = grid_index(c[0] + ((qq & 4) ? o[0] : 0), c[1] + ((qq & 2) ? o[1] : 0), c[2] + ((qq & 1) ? o[2] : 0));
					const int4* cp = reinterpret_cast<const int4*>(cells + cidx[q]);
#pragma unroll
					for (int w = 0; w < 4; w++) v[q][w] = cp[w];
				}
#pragma unroll
				for (int q = 0; q < 4; q++) {
					// a clamped neighbour may repeat a cell; scanning it twice is harmless
					const int cntq = v[q][0].x;
#pragma unroll
					for (int k = 0; k < 3; k++)
						if (k < cntq) test_slot<MODE>(v[q][1 + k], me, T, pp, nd, x, y, z, s2, lim, maxrank);
					if (cntq > 3) {
						const int4* cp = reinterpret_cast<const int4*>(cells + cidx[q]);
						int4 u[4];
#pragma unroll
						for (int w = 0; w < 4; w++) u[w] = cp[4 + w];
#pragma unroll
						for (int k = 0; k < 4; k++)
							if (3 + k < cntq) test_slot<MODE>(u[k], me, T, pp, nd, x, y, z, s2, lim, maxrank);
					}
					if (cntq > 3) n_past3++;
					if (cntq > kCellSlots) {
						n_ovf += cntq - kCellSlots;
						int32_t rr = ovf[cidx[q]];
						int64_t guard = 0;
						while (rr >= 0 && guard++ <= n) {
							int4 a = arena.accq[co + rr];
							a.w = rr;
							test_slot<MODE>(a, me, T, pp, nd, x, y, z, s2, lim, maxrank);
							rr = arena.link[co + rr];
						}
						if (guard > n + 1) atomicAdd(&st->timeouts, 1ull);
					}
				}
			}
		}
		R.x[tid] = x; R.y[tid] = y; R.z[tid] = z; R.key[tid] = key; R.lim[tid] = lim;
		R.maxrank[tid] = maxrank;
		R.local[tid] = local;
		R.nconf[tid] = 0;
		R.state[tid] = valid ? 0 : 2;
		{
			uint8_t os = 0;
			if (maxrank >= 0) {
				if (MODE == 1) os = 1;
				else if (maxrank >= cnt0 + tid - 10001) os = 1;       // conflicts whatever was accepted before it
				else if (maxrank < cnt0 - 10001) os = 0;              // outside the window in any case
				else os = 2;
			}
			R.old[tid] = os;
		}
		for (int s = tid; s < kRoundHash; s += kBigThreads) { R.hkey[s] = kEmptyCell; R.hhead[s] = -1; }
		__syncthreads();
		// ---- B: hash the round by cell, then collect earlier conflicting candidates
		long long clk1 = clock64();
		if (valid) {
			if (!round_cell_ok(c[0], c[1], c[2])) atomicAdd(&st->timeouts, 1ull);
			const int32_t k = round_cell_key(c[0], c[1], c[2]);
			uint32_t s = round_slot(k);
			for (int probe = 0; probe < kRoundHash; probe++) {
				const int32_t prev = atomicCAS(&R.hkey[s], kEmptyCell, k);
				if (prev == kEmptyCell || prev == k) break;
				s = (s + 1) & (kRoundHash - 1);
			}
			R.hnext[tid] = (int16_t)atomicExch(&R.hhead[s], tid);
		}
		__syncthreads();
		if (valid) {
			int nc = 0;
			for (int q = 0; q < 8; q++) {
				const int qx = c[0] + ((q & 4) ? o[0] : 0), qy = c[1] + ((q & 2) ? o[1] : 0), qz = c[2] + ((q & 1) ? o[2] : 0);
				if (!round_cell_ok(qx, qy, qz)) continue;
				const int32_t k = round_cell_key(qx, qy, qz);
				uint32_t s = round_slot(k);
				int j = -1;
				for (int probe = 0; probe < kRoundHash; probe++) {
					const int32_t kk = R.hkey[s];
					if (kk == k) { j = R.hhead[s]; break; }
					if (kk == kEmptyCell) break;
					s = (s + 1) & (kRoundHash - 1);
				}
				while (j >= 0) {
					if (j < tid && (MODE == 1 || R.key[j] >= lim) && sqdist(R.x[j], R.y[j], R.z[j], x, y, z) < s2) {
						if (nc < kMaxLocal) R.conf[tid][nc] = (int16_t)j;
						nc++;
					}
					j = R.hnext[j];
				}
			}
			R.nconf[tid] = (uint8_t)(nc < 255 ? nc : 255);
		}
		__syncthreads();
		// ---- C1: parallel passes
		long long clk2 = clock64();
		volatile uint8_t* vstate = R.state;
		for (int pass = 0; pass < 64; pass++) {
			bool changed = false;
			if (valid && vstate[tid] == 0 && R.nconf[tid] <= kMaxLocal) {
				const uint8_t os = R.old[tid];
				uint8_t dec = 0;
				if (os == 1) {
					dec = 2;
				} else {
					bool any_acc = false, all_done = true;
					for (int e = 0; e < R.nconf[tid]; e++) {
						uint8_t sj = vstate[R.conf[tid][e]];
						any_acc |= sj == 1;
						all_done &= sj != 0;
					}
					if (any_acc) dec = 2;
					else if (all_done && os == 0) dec = 1;
				}
				if (dec) { vstate[tid] = dec; changed = true; }
			}
			if (!__syncthreads_or(changed)) {
				if (tid == 0) atomicAdd(&st->passes, (unsigned long long)pass + 1);
				break;
			}
		}
		const bool left = __syncthreads_or(valid && vstate[tid] == 0);
		if (tid == 0) {
			atomicAdd(&st->rounds, 1ull);
			if (left) atomicAdd(&st->serial, 1ull);
		}
		long long clk3 = clock64();
		// ---- C2: warp 0 decides the rest in sorted order
		if (left && warp == 0) {
			int32_t cnt = cnt0;
			const uint32_t ltm = lanemask_lt();
			for (int cb = 0; cb < nr; cb += 32) {
				const int i = cb + lane;
				const bool v = i < nr;
				const uint8_t si = v ? vstate[i] : 2;
				const bool undec = v && si == 0;
				uint32_t accmask = __ballot_sync(FULL, v && si == 1);
				if (__ballot_sync(FULL, undec) != 0) {
					bool prev_conflict = false;
					uint32_t mask = 0;
					if (undec) {
						const int nc = R.nconf[i];
						if (nc <= kMaxLocal) {
							for (int e = 0; e < nc; e++) {
								int j = R.conf[i][e];
								if (j < cb) prev_conflict |= vstate[j] == 1;
								else mask |= 1u << (j - cb);
							}
						} else {  // list overflow: every earlier candidate of the round
							for (int j = 0; j < i; j++) {
								if ((MODE == 1 || R.key[j] >= R.lim[i]) && sqdist(R.x[j], R.y[j], R.z[j], R.x[i], R.y[i], R.z[i]) < s2) {
									if (j < cb) prev_conflict |= vstate[j] == 1;
									else mask |= 1u << (j - cb);
								}
							}
						}
					}
					const int nvalid = nr - cb < 32 ? nr - cb : 32;
					for (int b = 0; b < nvalid; b++) {
						bool dec = false;
						const bool ub = __shfl_sync(FULL, undec, b);
						if (!ub) continue;
						if (lane == b) {
							int32_t m_i = cnt + __popc(accmask & ltm);
							bool old_conflict = R.maxrank[i] >= 0 && (MODE == 1 || R.maxrank[i] >= m_i - 10001);
							dec = !old_conflict && !prev_conflict && !(mask & accmask);
							vstate[i] = dec ? 1 : 2;
						}
						dec = __shfl_sync(FULL, dec, b);
						if (dec) accmask |= 1u << b;
					}
				}
				cnt += __popc(accmask);
				__syncwarp();
			}
		}
		__syncthreads();
		// ---- D: publish
		long long clk4 = clock64();
		const bool acc = valid && vstate[tid] == 1;
		unsigned long long total;
		unsigned long long pre;
		{
			BlockScratch& bs = *reinterpret_cast<BlockScratch*>(R.warp_sums);
			pre = block_scan_u64(acc ? 1ull : 0ull, total, bs);
		}
		if (valid) {
			lb.accepted[co + local] = acc ? 1 : 0;
			if (acc) {
				const int32_t rank = cnt0 + (int32_t)pre;
				lb.acc_rank[co + local] = rank;
				const int64_t slot = co + rank;
				arena.accq[slot] = make_int4(me.x, me.y, me.z, 0);
				const int64_t ci = grid_index(c[0], c[1], c[2]);
				const int32_t pos = atomicAdd(&cells[ci].count, 1);
				if (pos < kCellSlots) cells[ci].slot[pos] = make_int4(me.x, me.y, me.z, rank);
				else arena.link[slot] = atomicExch(&ovf[ci], rank);
				if (MODE == 1) {
					// the colour pass walks the hash lists (linked through anext)
					ga.axyz[3 * slot] = x;
					ga.axyz[3 * slot + 1] = y;
					ga.axyz[3 * slot + 2] = z;
					ga.akey[slot] = key;
					ga.apos[slot] = (int32_t)t;
					if (!hash_push(hk, hh, ga.anext + co, nd.hash_cap, cell_key(c[0], c[1], c[2]), rank)) atomicAdd(&st->timeouts, 1ull);
				}
			}
		}
		__syncthreads();
		if (tid == 0) {
			R.cnt = cnt0 + (int32_t)total;
			const long long clk5 = clock64();
			atomicAdd(&st->cycles[0], (unsigned long long)(clk1 - clk0));
			atomicAdd(&st->cycles[1], (unsigned long long)(clk2 - clk1));
			atomicAdd(&st->cycles[2], (unsigned long long)(clk3 - clk2));
			atomicAdd(&st->cycles[3], (unsigned long long)(clk4 - clk3));
			atomicAdd(&st->cycles[4], (unsigned long long)(clk5 - clk4));
		}
		__syncthreads();
	}
	if (n_past3) atomicAdd(&st->cycles[5], n_past3);
	if (n_ovf) atomicAdd(&st->cycles[6], n_ovf);
	// empty the cells this node filled (count and overflow head)
	const int32_t total = R.cnt;
	for (int32_t r = tid; r < total; r += kBigThreads) {
		const int4 q = arena.accq[co + r];
		const double ax = ((double)q.x * pp.scale[0]) + pp.offset[0];
		const double ay = ((double)q.y * pp.scale[1]) + pp.offset[1];
		const double az = ((double)q.z * pp.scale[2]) + pp.offset[2];
		int cc[3];
		double fr[3];
		cell_of(g, ax, ay, az, cc, fr);
		const int64_t ci = grid_index(cc[0], cc[1], cc[2]);
		cells[ci].count = 0;
		ovf[ci] = -1;
	}
}


// Pulls the list row, list length and record of sorted position u into L2
// ahead of the round that reads them (they were written by an earlier kernel
// and usually sit in DRAM).
__device__ __forceinline__ void prefetch_list(const ConflictLists& cl, const LevelBuffers& lb, int64_t co, int64_t u) {
	asm volatile("prefetch.global.L2 [%0];" ::"l"(cl.inl + co + u));
	asm volatile("prefetch.global.L2 [%0];" ::"l"(cl.count + co + u));
	asm volatile("prefetch.global.L2 [%0];" ::"l"(lb.cq + co + u));
}

// Rounds of 1024 candidates, one per thread of a 1024-thread CTA.
constexpr int kListThreads = 1024;
constexpr int kListWarps = kListThreads / 32;
constexpr int kListRound = kListThreads;

// exclusive scan over the CTA of one count per thread
__device__ __forceinline__ uint32_t list_block_scan(uint32_t v, uint32_t& total, uint32_t* warp_sums) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	uint32_t x = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const uint32_t y = __shfl_up_sync(FULL, x, o);
		if (lane >= o) x += y;
	}
	if (lane == 31) warp_sums[warp] = x;
	__syncthreads();
	if (warp == 0) {
		uint32_t w = warp_sums[lane];
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t y = __shfl_up_sync(FULL, w, o);
			if (lane >= o) w += y;
		}
		warp_sums[lane] = w;
	}
	__syncthreads();
	const uint32_t before = warp > 0 ? warp_sums[warp - 1] : 0u;
	total = warp_sums[kListWarps - 1];
	__syncthreads();
	return before + x - v;
}
static_assert(kListWarps == 32, "one warp-sum per lane of warp 0");

// Greedy acceptance for a large node from its conflict lists (conflicts.cu),
// one CTA, 1024 candidates per round. A candidate's list names every earlier
// candidate that would reject it if accepted, so the round needs no spatial
// lookups: earlier rounds' decisions are read from srank (rank, or -1 for
// rejected), this round's are resolved by the same parallel passes and
// in-order warp as the grid kernel.
struct ListRound {
	int32_t maxrank[kListRound];
	int32_t local[kListRound];
	int16_t conf[kListRound][kListCap];
	uint8_t nconf[kListRound];
	uint8_t state[kListRound];   // 0 undecided, 1 accepted, 2 rejected
	uint8_t old[kListRound];     // old-window status: 0 no conflict, 1 conflict, 2 depends on the count
	int32_t cnt;             // accepted before this round
	uint32_t warp_sums[kListWarps];
};

template <int MODE>
__global__ void __launch_bounds__(kListThreads) greedy_list_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ order,
                                                                 int node_begin, PosParamsS pp, LevelBuffers lb, GreedyArgs ga,
                                                                 ConflictLists cl, int32_t* __restrict__ srank, SampleStats* st) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	ListRound& R = *reinterpret_cast<ListRound*>(smem_raw);
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const LevelNode nd = nodes[order[node_begin + blockIdx.x]];
	const int64_t n = nd.count, co = nd.cand_off;
	uint64_t* hk = ga.hkeys + nd.hash_off;
	int32_t* hh = ga.hheads + nd.hash_off;
	if (MODE == 1) {
		// poisson_average's colour pass finds accepted points through the hash
		for (int64_t i = tid; i < nd.hash_cap; i += kListThreads) { hk[i] = EMPTY_KEY; hh[i] = -1; }
	}
	if (tid == 0) R.cnt = 0;
	__syncthreads();
	CellGrid g;
	g.min[0] = nd.min[0]; g.min[1] = nd.min[1]; g.min[2] = nd.min[2];
	g.inv = 1.0 / (2.0 * nd.spacing * 1.000001);
	for (int64_t r0 = 0; r0 < n; r0 += kListRound) {
		const int64_t t = r0 + tid;
		const bool valid = t < n;
		const int nr = (int)((n - r0) < kListRound ? (n - r0) : kListRound);
		const int32_t cnt0 = R.cnt;
		// ---- A: the candidate's list
		long long clk0 = clock64();
		if (t + kListRound < n) prefetch_list(cl, lb, co, t + kListRound);
		int32_t maxrank = -1, local = 0;
		int nc = 0, nl = 0;
		int4 me = make_int4(0, 0, 0, 0);
		if (valid) {
			me = lb.cq[co + t];
			local = me.w;
			nl = cl.count[co + t];
		}
		{
			// lists are short (about one entry on average): loop to the
			// warp's longest list, four entries at a time (the first four in one
			// 16-byte load)
			const int wmax = (int)__reduce_max_sync(FULL, (unsigned)nl);
			for (int w = 0; 4 * w < wmax; w++) {
				const int4 v = 4 * w < nl ? list_quad(cl, co + t, nl, w) : make_int4(0, 0, 0, 0);
				const int32_t u4[4] = {v.x, v.y, v.z, v.w};
				int32_t rk4[4];
#pragma unroll
				for (int k = 0; k < 4; k++) rk4[k] = (4 * w + k < nl && u4[k] < r0) ? srank[co + u4[k]] : -1;
#pragma unroll
				for (int k = 0; k < 4; k++) {
					if (4 * w + k < nl) {
						if (u4[k] < r0) maxrank = rk4[k] > maxrank ? rk4[k] : maxrank;
						else R.conf[tid][nc++] = (int16_t)(u4[k] - r0);
					}
				}
			}
		}
		R.maxrank[tid] = maxrank;
		R.local[tid] = local;
		R.nconf[tid] = (uint8_t)nc;
		R.state[tid] = valid ? 0 : 2;
		{
			uint8_t os = 0;
			if (maxrank >= 0) {
				if (MODE == 1) os = 1;
				else if (maxrank >= cnt0 + tid - 10001) os = 1;       // conflicts whatever was accepted before it
				else if (maxrank < cnt0 - 10001) os = 0;              // outside the window in any case
				else os = 2;
			}
			R.old[tid] = os;
		}
		__syncthreads();
		long long clk1 = clock64();
		long long clk2 = clk1;
		// ---- C1: parallel passes
		volatile uint8_t* vstate = R.state;
		for (int pass = 0; pass < 64; pass++) {
			bool changed = false;
			if (valid && vstate[tid] == 0) {
				const uint8_t os = R.old[tid];
				uint8_t dec = 0;
				if (os == 1) {
					dec = 2;
				} else {
					bool any_acc = false, all_done = true;
					for (int e = 0; e < R.nconf[tid]; e++) {
						uint8_t sj = vstate[R.conf[tid][e]];
						any_acc |= sj == 1;
						all_done &= sj != 0;
					}
					if (any_acc) dec = 2;
					else if (all_done && os == 0) dec = 1;
				}
				if (dec) { vstate[tid] = dec; changed = true; }
			}
			if (!__syncthreads_or(changed)) {
				if (tid == 0) atomicAdd(&st->passes, (unsigned long long)pass + 1);
				break;
			}
		}
		const bool left = __syncthreads_or(valid && vstate[tid] == 0);
		if (tid == 0) {
			atomicAdd(&st->rounds, 1ull);
			if (left) atomicAdd(&st->serial, 1ull);
		}
		long long clk3 = clock64();
		// ---- C2: warp 0 decides the rest in sorted order
		if (left && warp == 0) {
			int32_t cnt = cnt0;
			const uint32_t ltm = lanemask_lt();
			for (int cb = 0; cb < nr; cb += 32) {
				const int i = cb + lane;
				const bool v = i < nr;
				const uint8_t si = v ? vstate[i] : 2;
				const bool undec = v && si == 0;
				uint32_t accmask = __ballot_sync(FULL, v && si == 1);
				if (__ballot_sync(FULL, undec) != 0) {
					bool prev_conflict = false;
					uint32_t mask = 0;
					if (undec) {
						const int ncf = R.nconf[i];
						for (int e = 0; e < ncf; e++) {
							int j = R.conf[i][e];
							if (j < cb) prev_conflict |= vstate[j] == 1;
							else mask |= 1u << (j - cb);
						}
					}
					const int nvalid = nr - cb < 32 ? nr - cb : 32;
					for (int b = 0; b < nvalid; b++) {
						bool dec = false;
						const bool ub = __shfl_sync(FULL, undec, b);
						if (!ub) continue;
						if (lane == b) {
							int32_t m_i = cnt + __popc(accmask & ltm);
							bool old_conflict = R.maxrank[i] >= 0 && (MODE == 1 || R.maxrank[i] >= m_i - 10001);
							dec = !old_conflict && !prev_conflict && !(mask & accmask);
							vstate[i] = dec ? 1 : 2;
						}
						dec = __shfl_sync(FULL, dec, b);
						if (dec) accmask |= 1u << b;
					}
				}
				cnt += __popc(accmask);
				__syncwarp();
			}
		}
		__syncthreads();
		// ---- D: publish
		long long clk4 = clock64();
		const bool acc = valid && vstate[tid] == 1;
		uint32_t total;
		uint32_t pre;
		{
			pre = list_block_scan(acc ? 1u : 0u, total, R.warp_sums);
		}
		if (valid) {
			const int32_t rank = cnt0 + (int32_t)pre;
			srank[co + t] = acc ? rank : -1;
			lb.accepted[co + local] = acc ? 1 : 0;
			if (acc) {
				lb.acc_rank[co + local] = rank;
				if (MODE == 1) {
					// the colour pass walks the hash lists (linked through anext)
					const int64_t slot = co + rank;
					const double x = ((double)me.x * pp.scale[0]) + pp.offset[0];
					const double y = ((double)me.y * pp.scale[1]) + pp.offset[1];
					const double z = ((double)me.z * pp.scale[2]) + pp.offset[2];
					ga.axyz[3 * slot] = x;
					ga.axyz[3 * slot + 1] = y;
					ga.axyz[3 * slot + 2] = z;
					ga.akey[slot] = lb.keys[co + t];
					ga.apos[slot] = (int32_t)t;
					int c[3];
					double fr[3];
					cell_of(g, x, y, z, c, fr);
					if (!hash_push(hk, hh, ga.anext + co, nd.hash_cap, cell_key(c[0], c[1], c[2]), rank)) atomicAdd(&st->timeouts, 1ull);
				}
			}
		}
		__syncthreads();
		if (tid == 0) {
			R.cnt = cnt0 + (int32_t)total;
			const long long clk5 = clock64();
			atomicAdd(&st->cycles[0], (unsigned long long)(clk1 - clk0));
			atomicAdd(&st->cycles[1], (unsigned long long)(clk2 - clk1));
			atomicAdd(&st->cycles[2], (unsigned long long)(clk3 - clk2));
			atomicAdd(&st->cycles[3], (unsigned long long)(clk4 - clk3));
			atomicAdd(&st->cycles[4], (unsigned long long)(clk5 - clk4));
		}
		__syncthreads();
	}
}


// Greedy acceptance for the largest nodes on a cluster of CS CTAs (CS x
// 1024 threads, CS = 4, or 8 for the few largest nodes of a level): a
// super-round decides CS x 1024 candidates, CTA k holding candidates
// [1024k, 1024k + 1024) of it. Each CTA keeps its candidates' states in its
// own shared memory; a candidate's conflicts inside the super-round (always
// with lower indices) are read from the owning CTA's shared memory through
// the cluster's distributed shared memory. Passes, the in-order warp (CTA
// 0, warp 0, reading and writing all CTAs' states) and the rank prefix are
// separated by cluster barriers, which every CTA reaches the same number of
// times. A node's serial chain of super-rounds sets a level's acceptance
// time, so its largest nodes take the wider cluster: half the super-rounds.
constexpr int kClusterCtas = 4;
constexpr int kWideClusterCtas = 8;  // portable maximum cluster size
constexpr int64_t kClusterMinCandidates = 65536;  // smallest cluster node the shared-memory layout is sized for
static_assert(kListRound * kWideClusterCtas <= 32767, "conflict indices are int16");
// A level's cluster nodes take 8-CTA clusters only when there are at most
// this many of them (the top levels): an 8-CTA cluster needs eight free SMs
// of one GPC at once, and beside many other nodes' CTAs it waits for them
// (measured: the 50M cloud's levels 3-5 lost 2-4x).
constexpr int kMaxWideClusterNodes = 4;

struct ClusterRound {
	int32_t maxrank[kListRound];
	int32_t local[kListRound];
	int16_t conf[kListRound][kListCap];  // indices inside the super-round
	uint8_t nconf[kListRound];
	uint8_t state[kListRound];   // 0 undecided, 1 accepted, 2 rejected
	uint8_t old[kListRound];     // old-window status as in ListRound
	uint32_t warp_sums[kListWarps];
	int32_t changed[2];          // per pass parity: this CTA changed a state
	int32_t left;                // this CTA has undecided candidates
	int32_t total;               // accepted in this CTA's part of the super-round
};

template <int MODE, int CS>
__global__ void __cluster_dims__(CS, 1, 1) __launch_bounds__(kListThreads, 1)
    greedy_list_cluster_kernel(const LevelNode* __restrict__ nodes, const int32_t* __restrict__ order, PosParamsS pp, LevelBuffers lb,
                               GreedyArgs ga, ConflictLists cl, int32_t* __restrict__ srank, SampleStats* st) {
	constexpr int kSuper = kListRound * CS;
	namespace cgr = cooperative_groups;
	cgr::cluster_group cluster = cgr::this_cluster();
	extern __shared__ __align__(16) unsigned char smem_raw[];
	ClusterRound& R = *reinterpret_cast<ClusterRound*>(smem_raw);
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int crank = (int)cluster.block_rank();
	// another CTA's round state (distributed shared memory)
	auto peer = [&](int r) { return cluster.map_shared_rank(&R, r); };
	const LevelNode nd = nodes[order[blockIdx.x / CS]];
	const int64_t n = nd.count, co = nd.cand_off;
	uint64_t* hk = ga.hkeys + nd.hash_off;
	int32_t* hh = ga.hheads + nd.hash_off;
	if (MODE == 1) {
		for (int64_t i = crank * kListThreads + tid; i < nd.hash_cap; i += kSuper) { hk[i] = EMPTY_KEY; hh[i] = -1; }
	}
	CellGrid g;
	g.min[0] = nd.min[0]; g.min[1] = nd.min[1]; g.min[2] = nd.min[2];
	g.inv = 1.0 / (2.0 * nd.spacing * 1.000001);
	int32_t cnt0 = 0;  // accepted before the super-round, the same in every CTA
	if (crank == 0 && tid == 0) atomicAdd(&st->cluster_nodes, 1ull);
	cluster.sync();
	for (int64_t r0 = 0; r0 < n; r0 += kSuper) {
		const int idx = crank * kListThreads + tid;  // index inside the super-round
		const int64_t t = r0 + idx;
		const bool valid = t < n;
		const int nr = (int)((n - r0) < kSuper ? (n - r0) : kSuper);
		// ---- A: the candidate's list
		const long long clk0 = clock64();
		if (t + kSuper < n) prefetch_list(cl, lb, co, t + kSuper);
		int32_t maxrank = -1, local = 0;
		int nc = 0, nl = 0;
		int4 me = make_int4(0, 0, 0, 0);
		if (valid) {
			me = lb.cq[co + t];
			local = me.w;
			nl = cl.count[co + t];
		}
		{
			const int wmax = (int)__reduce_max_sync(FULL, (unsigned)nl);
			for (int w = 0; 4 * w < wmax; w++) {
				const int4 v = 4 * w < nl ? list_quad(cl, co + t, nl, w) : make_int4(0, 0, 0, 0);
				const int32_t u4[4] = {v.x, v.y, v.z, v.w};
				int32_t rk4[4];
#pragma unroll
				for (int k = 0; k < 4; k++) rk4[k] = (4 * w + k < nl && u4[k] < r0) ? srank[co + u4[k]] : -1;
#pragma unroll
				for (int k = 0; k < 4; k++) {
					if (4 * w + k < nl) {
						if (u4[k] < r0) maxrank = rk4[k] > maxrank ? rk4[k] : maxrank;
						else R.conf[tid][nc++] = (int16_t)(u4[k] - r0);
					}
				}
			}
		}
		R.maxrank[tid] = maxrank;
		R.local[tid] = local;
		R.nconf[tid] = (uint8_t)nc;
		R.state[tid] = valid ? 0 : 2;
		{
			uint8_t os = 0;
			if (maxrank >= 0) {
				if (MODE == 1) os = 1;
				else if (maxrank >= cnt0 + idx - 10001) os = 1;       // conflicts whatever was accepted before it
				else if (maxrank < cnt0 - 10001) os = 0;              // outside the window in any case
				else os = 2;
			}
			R.old[tid] = os;
		}
		cluster.sync();
		const long long clk1 = clock64();
		// ---- C1: parallel passes. Decisions only go from undecided to final,
		// so a stale read of another CTA's state only delays a decision:
		// each CTA repeats local passes (block barriers) while it makes
		// progress, then the cluster barrier publishes whether any CTA did;
		// the fixpoint is a cluster round in which none did.
		int passes = 0;
		for (int gpass = 0; gpass < 64; gpass++) {
			int progressed = 0;
			for (int lp = 0; lp < 64; lp++) {
				bool changed = false;
				if (valid && R.state[tid] == 0) {
					const uint8_t os = R.old[tid];
					uint8_t dec = 0;
					if (os == 1) {
						dec = 2;
					} else {
						bool any_acc = false, all_done = true;
						for (int e = 0; e < R.nconf[tid]; e++) {
							const int j = R.conf[tid][e];
							const uint8_t sj = *(volatile uint8_t*)&peer(j / kListRound)->state[j % kListRound];
							any_acc |= sj == 1;
							all_done &= sj != 0;
						}
						if (any_acc) dec = 2;
						else if (all_done && os == 0) dec = 1;
					}
					if (dec) {
						*(volatile uint8_t*)&R.state[tid] = dec;
						changed = true;
					}
				}
				passes++;
				if (!__syncthreads_or(changed)) break;
				progressed = 1;
			}
			if (tid == 0) R.changed[gpass & 1] = progressed;
			cluster.sync();
			int all = 0;
#pragma unroll
			for (int r = 0; r < CS; r++) all |= *(volatile int32_t*)&peer(r)->changed[gpass & 1];
			if (!all) break;
		}
		if (tid == 0 && crank == 0) atomicAdd(&st->passes, (unsigned long long)passes);
		const int left_here = __syncthreads_or(valid && R.state[tid] == 0);
		if (tid == 0) R.left = left_here;
		cluster.sync();
		int left = 0;
#pragma unroll
		for (int r = 0; r < CS; r++) left |= *(volatile int32_t*)&peer(r)->left;
		if (crank == 0 && tid == 0) {
			atomicAdd(&st->rounds, 1ull);
			if (left) atomicAdd(&st->serial, 1ull);
		}
		const long long clk2 = clock64();
		// ---- C2: one warp decides the rest in order
		if (left && crank == 0 && warp == 0) {
			int32_t cnt = cnt0;
			const uint32_t ltm = lanemask_lt();
			for (int cb = 0; cb < nr; cb += 32) {
				const int i = cb + lane;
				const bool v = i < nr;
				ClusterRound* Ri = peer((v ? i : 0) / kListRound);
				const int li = (v ? i : 0) % kListRound;
				const uint8_t si = v ? *(volatile uint8_t*)&Ri->state[li] : 2;
				const bool undec = v && si == 0;
				uint32_t accmask = __ballot_sync(FULL, v && si == 1);
				if (__ballot_sync(FULL, undec) != 0) {
					bool prev_conflict = false;
					uint32_t mask = 0;
					if (undec) {
						const int ncf = Ri->nconf[li];
						for (int e = 0; e < ncf; e++) {
							const int j = Ri->conf[li][e];
							if (j < cb) prev_conflict |= *(volatile uint8_t*)&peer(j / kListRound)->state[j % kListRound] == 1;
							else mask |= 1u << (j - cb);
						}
					}
					const int nvalid = nr - cb < 32 ? nr - cb : 32;
					for (int b = 0; b < nvalid; b++) {
						bool dec = false;
						const bool ub = __shfl_sync(FULL, undec, b);
						if (!ub) continue;
						if (lane == b) {
							const int32_t m_i = cnt + __popc(accmask & ltm);
							const int32_t mr = Ri->maxrank[li];
							const bool old_conflict = mr >= 0 && (MODE == 1 || mr >= m_i - 10001);
							dec = !old_conflict && !prev_conflict && !(mask & accmask);
							*(volatile uint8_t*)&Ri->state[li] = dec ? 1 : 2;
						}
						dec = __shfl_sync(FULL, dec, b);
						if (dec) accmask |= 1u << b;
					}
				}
				cnt += __popc(accmask);
				__syncwarp();
			}
		}
		cluster.sync();
		const long long clk3 = clock64();
		// ---- D: ranks across the cluster, publish
		const bool acc = valid && R.state[tid] == 1;
		uint32_t total;
		const uint32_t pre = list_block_scan(acc ? 1u : 0u, total, R.warp_sums);
		if (tid == 0) R.total = (int32_t)total;
		cluster.sync();
		int32_t before = 0, all_acc = 0;
#pragma unroll
		for (int r = 0; r < CS; r++) {
			const int32_t tr = *(volatile int32_t*)&peer(r)->total;
			if (r < crank) before += tr;
			all_acc += tr;
		}
		if (valid) {
			const int32_t rank = cnt0 + before + (int32_t)pre;
			srank[co + t] = acc ? rank : -1;
			lb.accepted[co + local] = acc ? 1 : 0;
			if (acc) {
				lb.acc_rank[co + local] = rank;
				if (MODE == 1) {
					const int64_t slot = co + rank;
					const double x = ((double)me.x * pp.scale[0]) + pp.offset[0];
					const double y = ((double)me.y * pp.scale[1]) + pp.offset[1];
					const double z = ((double)me.z * pp.scale[2]) + pp.offset[2];
					ga.axyz[3 * slot] = x;
					ga.axyz[3 * slot + 1] = y;
					ga.axyz[3 * slot + 2] = z;
					ga.akey[slot] = lb.keys[co + t];
					ga.apos[slot] = (int32_t)t;
					int c[3];
					double fr[3];
					cell_of(g, x, y, z, c, fr);
					if (!hash_push(hk, hh, ga.anext + co, nd.hash_cap, cell_key(c[0], c[1], c[2]), rank)) atomicAdd(&st->timeouts, 1ull);
				}
			}
		}
		cnt0 += all_acc;
		// the next super-round rewrites states, flags and totals other CTAs read
		cluster.sync();
		if (crank == 0 && tid == 0) {
			const long long clk4 = clock64();
			atomicAdd(&st->cycles[0], (unsigned long long)(clk1 - clk0));
			atomicAdd(&st->cycles[2], (unsigned long long)(clk2 - clk1));
			atomicAdd(&st->cycles[3], (unsigned long long)(clk3 - clk2));
			atomicAdd(&st->cycles[4], (unsigned long long)(clk4 - clk3));
		}
	}
}

// Greedy acceptance from conflict lists for the smaller nodes, one warp per
// node, 32 candidates per step. Conflicts with earlier steps come from
// srank; inside a step they are a lane mask, resolved by ballot passes (a
// lane decides once its earlier conflicting lanes have) or, when a lane's
// old conflict sits at the edge of the 10,001-check window, in lane order.
template <int MODE>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) greedy_list_warp_kernel(const LevelNode* __restrict__ nodes,
                                                                              const int32_t* __restrict__ order, int num, PosParamsS pp,
                                                                              LevelBuffers lb, GreedyArgs ga, ConflictLists cl,
                                                                              int32_t* __restrict__ srank, SampleStats* st,
                                                                              int* next_node) {
	const int lane = threadIdx.x & 31;
	const uint32_t lt = lanemask_lt();
	while (true) {
		int idx = 0;
		if (lane == 0) idx = atomicAdd(next_node, 1);
		idx = __shfl_sync(FULL, idx, 0);
		if (idx >= num) break;
		const LevelNode nd = nodes[order[idx]];
		const int64_t n = nd.count, co = nd.cand_off;
		uint64_t* hk = ga.hkeys + nd.hash_off;
		int32_t* hh = ga.hheads + nd.hash_off;
		CellGrid g;
		g.min[0] = nd.min[0]; g.min[1] = nd.min[1]; g.min[2] = nd.min[2];
		g.inv = 1.0 / (2.0 * nd.spacing * 1.000001);
		if (MODE == 1) {
			for (int64_t s = lane; s < nd.hash_cap; s += 32) { hk[s] = EMPTY_KEY; hh[s] = -1; }
			__syncwarp();
		}
		int32_t cnt = 0;  // accepted so far
		for (int64_t b0 = 0; b0 < n; b0 += 32) {
			const int64_t t = b0 + lane;
			const bool valid = t < n;
			if (t + 64 < n) prefetch_list(cl, lb, co, t + 64);
			int4 me = make_int4(0, 0, 0, 0);
			int32_t maxrank = -1;
			uint32_t mask = 0;  // earlier lanes of this step that conflict
			int nl = 0;
			if (valid) {
				me = lb.cq[co + t];
				nl = cl.count[co + t];
			}
			{
				const int wmax = (int)__reduce_max_sync(FULL, (unsigned)nl);
				for (int w = 0; 4 * w < wmax; w++) {
					const int4 v = 4 * w < nl ? list_quad(cl, co + t, nl, w) : make_int4(0, 0, 0, 0);
					const int32_t u4[4] = {v.x, v.y, v.z, v.w};
					int32_t rk4[4];
#pragma unroll
					for (int k = 0; k < 4; k++) rk4[k] = (4 * w + k < nl && u4[k] < b0) ? srank[co + u4[k]] : -1;
#pragma unroll
					for (int k = 0; k < 4; k++) {
						if (4 * w + k < nl) {
							if (u4[k] < b0) maxrank = rk4[k] > maxrank ? rk4[k] : maxrank;
							else mask |= 1u << (u4[k] - b0);
						}
					}
				}
			}
			int os = 0;
			if (maxrank >= 0) {
				if (MODE == 1) os = 1;
				else if (maxrank >= cnt + lane - 10001) os = 1;  // conflicts whatever was accepted before it
				else if (maxrank < cnt - 10001) os = 0;          // outside the window in any case
				else os = 2;
			}
			const uint32_t validmask = __ballot_sync(FULL, valid);
			uint32_t accmask = 0;
			if (__ballot_sync(FULL, valid && os == 2) == 0) {
				uint32_t undec = validmask & ~__ballot_sync(FULL, valid && os == 1);
				for (int it = 0; it < 33 && undec; it++) {
					const bool mine = (undec >> lane) & 1u;
					const bool ready = mine && (mask & undec) == 0;
					const bool a = ready && (mask & accmask) == 0;
					accmask |= __ballot_sync(FULL, a);
					undec &= ~__ballot_sync(FULL, ready);
				}
			} else {
				for (int b = 0; b < 32; b++) {
					if (!((validmask >> b) & 1u)) continue;
					bool dec = false;
					if (lane == b && os != 1) {
						const int32_t m_i = cnt + __popc(accmask & lt);
						const bool old_conflict = maxrank >= 0 && (MODE == 1 || maxrank >= m_i - 10001);
						dec = !old_conflict && !(mask & accmask);
					}
					dec = __shfl_sync(FULL, dec, b);
					if (dec) accmask |= 1u << b;
				}
			}
			const bool acc = (accmask >> lane) & 1u;
			if (valid) {
				const int32_t rank = cnt + __popc(accmask & lt);
				const int32_t local = me.w;
				srank[co + t] = acc ? rank : -1;
				lb.accepted[co + local] = acc ? 1 : 0;
				if (acc) {
					lb.acc_rank[co + local] = rank;
					if (MODE == 1) {
						const int64_t slot = co + rank;
						const double x = ((double)me.x * pp.scale[0]) + pp.offset[0];
						const double y = ((double)me.y * pp.scale[1]) + pp.offset[1];
						const double z = ((double)me.z * pp.scale[2]) + pp.offset[2];
						ga.axyz[3 * slot] = x;
						ga.axyz[3 * slot + 1] = y;
						ga.axyz[3 * slot + 2] = z;
						ga.akey[slot] = lb.keys[co + t];
						ga.apos[slot] = (int32_t)t;
						int c[3];
						double fr[3];
						cell_of(g, x, y, z, c, fr);
						if (!hash_push(hk, hh, ga.anext + co, nd.hash_cap, cell_key(c[0], c[1], c[2]), rank)) atomicAdd(&st->timeouts, 1ull);
					}
				}
			}
			cnt += __popc(accmask);
		}
	}
}

}  // namespace

// ----------------------------------------------------------------- launchers
void launch_gather(const std::vector<GatherItem>& h_items, const GatherItem* items, LevelBuffers& lb, DeviceMem& mem) {
	std::vector<int32_t> pi;
	std::vector<int64_t> ps;
	for (size_t k = 0; k < h_items.size(); k++)
		for (int64_t t = 0; t < h_items[k].count; t += kGatherPiece) {
			pi.push_back((int32_t)k);
			ps.push_back(t);
		}
	if (pi.empty()) return;
	int32_t* d_pi = mem.alloc<int32_t>(pi.size());
	int64_t* d_ps = mem.alloc<int64_t>(ps.size());
	PCG_CUDA(cudaMemcpyAsync(d_pi, pi.data(), pi.size() * sizeof(int32_t), cudaMemcpyHostToDevice, mem.stream()));
	PCG_CUDA(cudaMemcpyAsync(d_ps, ps.data(), ps.size() * sizeof(int64_t), cudaMemcpyHostToDevice, mem.stream()));
	gather_kernel<<<(unsigned)pi.size(), 256, 0, mem.stream()>>>(items, d_pi, d_ps, lb);
	PCG_LAUNCHED();
	mem.free(d_ps);
	mem.free(d_pi);
}

void launch_keys(const LevelNode* nodes, const PosParamsS& pp, LevelBuffers& lb, DeviceMem& mem) {
	if (lb.M == 0) return;
	keys_kernel<<<(unsigned)ceil_div(lb.M, 256), 256, 0, mem.stream()>>>(nodes, pp, lb);
	PCG_LAUNCHED();
}

void launch_gather_records(const uint32_t* ids, int64_t n, const int32_t* X, const int32_t* Y, const int32_t* Z, int4* rec, DeviceMem& mem,
                           int64_t n_src) {
	if (n > 0 && n_src >= (int64_t(1) << 20)) {
		// a permutation of many points: pack first, then one load per point
		int4* xyz = mem.alloc<int4>(n_src);
		pack_records_kernel<<<(unsigned)ceil_div(n_src, 256), 256, 0, mem.stream()>>>(n_src, X, Y, Z, xyz);
		PCG_LAUNCHED();
		gather_packed_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(ids, n, xyz, rec);
		PCG_LAUNCHED();
		mem.free(xyz);
		return;
	}
	if (n == 0) return;
	gather_records_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(ids, n, X, Y, Z, rec);
	PCG_LAUNCHED();
}


void launch_cand_records(const LevelNode* nodes, const int32_t* X, const int32_t* Y, const int32_t* Z, LevelBuffers& lb, DeviceMem& mem) {
	if (lb.M == 0) return;
	cand_records_kernel<<<(unsigned)ceil_div(lb.M, 256), 256, 0, mem.stream()>>>(nodes, X, Y, Z, lb);
	PCG_LAUNCHED();
}

void greedy_arena_reserve(GreedyArena& a, int slots, DeviceMem& mem) {
	if (slots <= a.slots) return;
	if (a.cells) { mem.free(a.cells); mem.free(a.ovf); }
	a.cells = mem.alloc<AccCell>((size_t)slots * kGridCells);
	a.ovf = mem.alloc<int32_t>((size_t)slots * kGridCells);
	PCG_CUDA(cudaMemsetAsync(a.cells, 0, (size_t)slots * kGridCells * sizeof(AccCell), mem.stream()));
	PCG_CUDA(cudaMemsetAsync(a.ovf, 0xff, (size_t)slots * kGridCells * sizeof(int32_t), mem.stream()));
	a.slots = slots;
}

void launch_greedy(int mode, bool fp32_guard, const LevelNode* nodes, const int32_t* order, int K, const int32_t* X, const int32_t* Y,
                   const int32_t* Z, const PosParamsS& pp, LevelBuffers& lb, uint64_t* hash_keys, int32_t* hash_heads,
                   double* acc_xyz, double* acc_key, int32_t* acc_next, int32_t* acc_pos, SampleStats* st, DeviceMem& mem,
                   GreedyArena* grid, int node_begin, int node_end, int num_big) {
	if (node_end < 0) node_end = K;
	if (lb.M == 0) return;
	GreedyArgs ga{hash_keys, hash_heads, acc_xyz, acc_key, acc_next, acc_pos};
	cudaStream_t s = mem.stream();
	if (node_end <= node_begin) return;
	const int big_end = num_big < node_end ? num_big : node_end;
	if (big_end > node_begin) {
		size_t smem = sizeof(RoundShared);
		// one dense acceptance grid per resident CTA (kept empty between
		// nodes); large levels go in batches
		const int batch = sm_count() * 2;
		const int nbig = big_end - node_begin;
		const int slots = nbig < batch ? nbig : batch;
		greedy_arena_reserve(*grid, slots, mem);
		GridArena arena;
		arena.cells = static_cast<AccCell*>(grid->cells);
		arena.ovf = grid->ovf;
		arena.link = mem.alloc<int32_t>((size_t)lb.M);
		arena.accq = mem.alloc<int4>((size_t)lb.M);
		if (mode == 0) PCG_CUDA(cudaFuncSetAttribute(greedy_big_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
		else PCG_CUDA(cudaFuncSetAttribute(greedy_big_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
		for (int b0 = node_begin; b0 < big_end; b0 += slots) {
			const int cnt = big_end - b0 < slots ? big_end - b0 : slots;
			if (mode == 0) greedy_big_kernel<0><<<cnt, kBigThreads, smem, s>>>(nodes, order, b0, pp, lb, ga, arena, st);
			else greedy_big_kernel<1><<<cnt, kBigThreads, smem, s>>>(nodes, order, b0, pp, lb, ga, arena, st);
			PCG_LAUNCHED();
		}
		mem.free(arena.link);
		mem.free(arena.accq);
	}
	const int small_begin = node_begin > num_big ? node_begin : num_big;
	if (node_end > small_begin) {
		int* counter = mem.alloc<int>(1);
		PCG_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), s));
		int blocks = (int)ceil_div(node_end - small_begin, kWarpsPerBlock);
		int cap = sm_count() * 16;
		if (blocks > cap) blocks = cap;
		dim3 grid(blocks), block(kWarpsPerBlock * 32);
		if (mode == 0 && fp32_guard) greedy_kernel<0, true><<<grid, block, 0, s>>>(nodes, order, small_begin, node_end, X, Y, Z, pp, lb, ga, st, counter);
		else if (mode == 0) greedy_kernel<0, false><<<grid, block, 0, s>>>(nodes, order, small_begin, node_end, X, Y, Z, pp, lb, ga, st, counter);
		else if (fp32_guard) greedy_kernel<1, true><<<grid, block, 0, s>>>(nodes, order, small_begin, node_end, X, Y, Z, pp, lb, ga, st, counter);
		else greedy_kernel<1, false><<<grid, block, 0, s>>>(nodes, order, small_begin, node_end, X, Y, Z, pp, lb, ga, st, counter);
		PCG_LAUNCHED();
		mem.free(counter);
	}
}

LevelSchedule level_schedule() {
	// read at every level, so the autotuner can sweep in one process
	LevelSchedule v{PCG_TUNED_CTA_MIN, PCG_TUNED_SMALL_LEVEL_CTA_MIN, PCG_TUNED_CLUSTER_MIN, PCG_TUNED_WARP_BLOCKS_PER_SM};
	if (const char* e = std::getenv("PCG_SCHEDULE")) {
		long long a = 0, b = 0, c = 0, d = 0;
		if (std::sscanf(e, "%lld,%lld,%lld,%lld", &a, &b, &c, &d) == 4 && a > 0 && b > 0 && c > 0 && d > 0 && d <= 64)
			v = LevelSchedule{a, b, c, (int)d};
	}
	return v;
}

void launch_greedy_lists(int mode, const LevelNode* nodes, const std::vector<int32_t>& cta_nodes, const std::vector<int32_t>& warp_nodes,
                         const PosParamsS& pp, LevelBuffers& lb, uint64_t* hash_keys, int32_t* hash_heads, double* acc_xyz,
                         double* acc_key, int32_t* acc_next, int32_t* acc_pos, const ConflictLists& cl, SampleStats* st, DeviceMem& mem,
                         const std::vector<LevelNode>& ln) {
	if (lb.M == 0 || (cta_nodes.empty() && warp_nodes.empty())) return;
	GreedyArgs ga{hash_keys, hash_heads, acc_xyz, acc_key, acc_next, acc_pos};
	cudaStream_t s = mem.stream();
	// the largest nodes (cta_nodes is largest first) on a cluster each, the
	// other CTA nodes on one CTA, the rest on a warp
	std::vector<int32_t> wide, clu, one;
	const int64_t cluster_min = std::max(level_schedule().cluster_min, kClusterMinCandidates);
	for (int32_t k : cta_nodes) (ln[k].count >= cluster_min ? clu : one).push_back(k);
	if (!clu.empty() && (int)clu.size() <= kMaxWideClusterNodes) wide.swap(clu);
	int32_t* srank = mem.alloc<int32_t>((size_t)lb.M);
	int32_t* d_wide = wide.empty() ? nullptr : mem.alloc<int32_t>(wide.size());
	int32_t* d_clu = clu.empty() ? nullptr : mem.alloc<int32_t>(clu.size());
	int32_t* d_one = one.empty() ? nullptr : mem.alloc<int32_t>(one.size());
	int32_t* d_warp = warp_nodes.empty() ? nullptr : mem.alloc<int32_t>(warp_nodes.size());
	int* counter = mem.alloc<int>(1);
	if (d_wide) PCG_CUDA(cudaMemcpyAsync(d_wide, wide.data(), wide.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
	if (d_clu) PCG_CUDA(cudaMemcpyAsync(d_clu, clu.data(), clu.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
	if (d_one) PCG_CUDA(cudaMemcpyAsync(d_one, one.data(), one.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
	if (d_warp) PCG_CUDA(cudaMemcpyAsync(d_warp, warp_nodes.data(), warp_nodes.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
	PCG_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), s));
	// the node sets are independent: the first runs on the job's stream, the
	// second on one forked stream, the others on a second one
	constexpr int kSides = DeviceArena::kSides;
	cudaStream_t side[kSides] = {nullptr, nullptr};
	cudaEvent_t fork[kSides] = {nullptr, nullptr}, join[kSides] = {nullptr, nullptr};
	const int sets = (d_wide ? 1 : 0) + (d_clu ? 1 : 0) + (d_one ? 1 : 0) + (d_warp ? 1 : 0);
	const int nsides = mem.arena() ? std::min(sets - 1, kSides) : 0;
	for (int k = 0; k < nsides; k++) {
		side[k] = mem.arena()->side_stream(fork[k], join[k], k);
		PCG_CUDA(cudaEventRecord(fork[k], s));
		PCG_CUDA(cudaStreamWaitEvent(side[k], fork[k], 0));
	}
	int next_set = 0;
	auto stream_for_set = [&]() {
		const int i = next_set++;
		if (i == 0 || nsides == 0) return s;
		return side[std::min(i, nsides) - 1];
	};
	auto launch_cluster = [&](auto kernel, int cs_ctas, const int32_t* d_set, size_t count, cudaStream_t cs) {
		const size_t smem = sizeof(ClusterRound);
		PCG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
		kernel<<<(unsigned)(count * cs_ctas), kListThreads, smem, cs>>>(nodes, d_set, pp, lb, ga, cl, srank, st);
		PCG_LAUNCHED();
	};
	if (d_wide) {
		cudaStream_t cs = stream_for_set();
		if (mode == 0) launch_cluster(greedy_list_cluster_kernel<0, kWideClusterCtas>, kWideClusterCtas, d_wide, wide.size(), cs);
		else launch_cluster(greedy_list_cluster_kernel<1, kWideClusterCtas>, kWideClusterCtas, d_wide, wide.size(), cs);
	}
	if (d_clu) {
		cudaStream_t cs = stream_for_set();
		if (mode == 0) launch_cluster(greedy_list_cluster_kernel<0, kClusterCtas>, kClusterCtas, d_clu, clu.size(), cs);
		else launch_cluster(greedy_list_cluster_kernel<1, kClusterCtas>, kClusterCtas, d_clu, clu.size(), cs);
	}
	if (d_one) {
		const size_t smem = sizeof(ListRound);
		const int nc = (int)one.size();
		cudaStream_t cs = stream_for_set();
		if (mode == 0) {
			PCG_CUDA(cudaFuncSetAttribute(greedy_list_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
			greedy_list_kernel<0><<<nc, kListThreads, smem, cs>>>(nodes, d_one, 0, pp, lb, ga, cl, srank, st);
		} else {
			PCG_CUDA(cudaFuncSetAttribute(greedy_list_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
			greedy_list_kernel<1><<<nc, kListThreads, smem, cs>>>(nodes, d_one, 0, pp, lb, ga, cl, srank, st);
		}
		PCG_LAUNCHED();
	}
	if (d_warp) {
		cudaStream_t ws = stream_for_set();
		const int nw = (int)warp_nodes.size();
		int blocks = (int)ceil_div(nw, kWarpsPerBlock);
		const int cap = sm_count() * level_schedule().warp_blocks_per_sm;
		if (blocks > cap) blocks = cap;
		if (mode == 0) greedy_list_warp_kernel<0><<<blocks, kWarpsPerBlock * 32, 0, ws>>>(nodes, d_warp, nw, pp, lb, ga, cl, srank, st, counter);
		else greedy_list_warp_kernel<1><<<blocks, kWarpsPerBlock * 32, 0, ws>>>(nodes, d_warp, nw, pp, lb, ga, cl, srank, st, counter);
		PCG_LAUNCHED();
	}
	for (int k = 0; k < nsides; k++) {
		PCG_CUDA(cudaEventRecord(join[k], side[k]));
		PCG_CUDA(cudaStreamWaitEvent(s, join[k], 0));
	}
	mem.free(srank);
	if (d_wide) mem.free(d_wide);
	if (d_clu) mem.free(d_clu);
	if (d_one) mem.free(d_one);
	if (d_warp) mem.free(d_warp);
	mem.free(counter);
}

void launch_average_colors(const LevelNode* nodes, const int32_t* X, const int32_t* Y, const int32_t* Z, const PosParamsS& pp,
                           LevelBuffers& lb, const uint64_t* hash_keys, const int32_t* hash_heads, const double* acc_xyz,
                           const int32_t* acc_next, const int32_t* acc_pos, const int64_t* /*acc_base*/, long long* sums,
                           DeviceMem& mem) {
	if (lb.M == 0) return;
	GreedyArgs ga{const_cast<uint64_t*>(hash_keys), const_cast<int32_t*>(hash_heads), const_cast<double*>(acc_xyz), nullptr,
	              const_cast<int32_t*>(acc_next), const_cast<int32_t*>(acc_pos)};
	PCG_CUDA(cudaMemsetAsync(sums, 0, sizeof(long long) * 4 * lb.M, mem.stream()));
	unsigned blocks = (unsigned)ceil_div(lb.M, 256);
	average_colors_kernel<<<blocks, 256, 0, mem.stream()>>>(nodes, X, Y, Z, pp, lb, ga, sums);
	PCG_LAUNCHED();
	average_finish_kernel<<<blocks, 256, 0, mem.stream()>>>(nodes, lb, sums);
	PCG_LAUNCHED();
}

void launch_random_accept_sized(const LevelNode* nodes, const int32_t* X, const int32_t* Y, const int32_t* Z, const PosParamsS& pp,
                                LevelBuffers& lb, uint64_t* hash_keys, int32_t* hash_vals, int64_t hash_total, SampleStats* st,
                                DeviceMem& mem) {
	if (lb.M == 0) return;
	clear_hash_kernel<<<(unsigned)ceil_div(hash_total, 256), 256, 0, mem.stream()>>>(hash_keys, hash_vals, hash_total, 0x7fffffff);
	PCG_LAUNCHED();
	unsigned blocks = (unsigned)ceil_div(lb.M, 256);
	random_first_kernel<<<blocks, 256, 0, mem.stream()>>>(nodes, X, Y, Z, pp, lb, hash_keys, hash_vals, st);
	PCG_LAUNCHED();
	random_accept_kernel<<<blocks, 256, 0, mem.stream()>>>(nodes, X, Y, Z, pp, lb, hash_keys, hash_vals);
	PCG_LAUNCHED();
}

void launch_shuffle_leaves(const int64_t* leaf_off, const int64_t* leaf_cnt, int num_leaves, const uint32_t* ids_in,
                           uint32_t* ids_out, int32_t* scratch, uint32_t seed, DeviceMem& mem) {
	if (num_leaves == 0) return;
	shuffle_leaves_kernel<<<(unsigned)ceil_div(num_leaves, 64), 64, 0, mem.stream()>>>(leaf_off, leaf_cnt, num_leaves, ids_in, ids_out,
	                                                                                    scratch, seed);
	PCG_LAUNCHED();
}


void launch_shuffle_single(int64_t n, uint32_t seed, int32_t* perm, DeviceMem& mem) {
	if (n <= 0) return;
	shuffle_single_kernel<<<1, 1, 0, mem.stream()>>>(n, seed, perm);
	PCG_LAUNCHED();
}

}  // namespace pcg
