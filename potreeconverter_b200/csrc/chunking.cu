// Chunker on the device: LAS record decode + quantize + count grid
// (countPointsInCells, chunker_countsort_laszip.cpp:131-361, and the decode
// half of distributePoints, :749-803 with the handlers of :380-658), the
// pyramid cell merge (createLUT, :1074-1204) and the chunk lookup that feeds
// the stable scatter (:837-904).
//
// All FP64 expressions are evaluated in the reference's order; the library
// is compiled with --fmad=false so no multiply-add is contracted, matching
// x86-64 SSE2 code without FMA.

#include <math_constants.h>

#include "bulk.cuh"
#include "devutil.cuh"
#include "kernels.h"

namespace pcg {

namespace {

__device__ __forceinline__ unsigned long long ordered(double d) {
	unsigned long long b = (unsigned long long)__double_as_longlong(d);
	return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

template <class T> __device__ __forceinline__ T ld(const uint8_t* p) {
	T v;
	memcpy(&v, p, sizeof(T));
	return v;
}

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min(a, b)
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max(a, b)

constexpr int kDecodeThreads = 256;

// min / max of one extra-attribute element as ordered bit patterns
struct ExtraRange {
	unsigned long long mn = ~0ull, mx = 0ull;
	__device__ void add(unsigned long long o) { mn = o < mn ? o : mn; mx = o > mx ? o : mx; }
};

struct IntRange {
	int mn, mx;
	__device__ void init() { mn = 0x7fffffff; mx = -0x7fffffff - 1; }
	__device__ void add(int v) { mn = v < mn ? v : mn; mx = v > mx ? v : mx; }
};

__device__ void flush_int(AttrStatsDev* st, int comp, const IntRange& r, unsigned long long* smem_mn, unsigned long long* smem_mx) {
	if (r.mn <= r.mx) {
		atomicMin(smem_mn + comp, ordered((double)r.mn));
		atomicMax(smem_mx + comp, ordered((double)r.mx));
	}
}

// The count-grid cell of a quantized point (countPointsInCells, :232-257):
// unit-cube coordinates from the output transform, out-of-box test, cell
// index ix + iy G + iz G^2. False when the point lies outside the box.
__device__ __forceinline__ bool grid_cell(const DecodeParams& p, int32_t X, int32_t Y, int32_t Z, uint32_t& cell) {
	const int G = p.grid;
	const double dG = (double)G;
	double ux = ((double)X * p.pos_scale[0] + p.pos_offset[0] - p.cmin[0]) / p.csize;
	double uy = ((double)Y * p.pos_scale[1] + p.pos_offset[1] - p.cmin[1]) / p.csize;
	double uz = ((double)Z * p.pos_scale[2] + p.pos_offset[2] - p.cmin[2]) / p.csize;
	bool in_box = ux >= 0.0 && uy >= 0.0 && uz >= 0.0 && ux <= 1.0 && uy <= 1.0 && uz <= 1.0;
	cell = 0;
	if (!in_box) return false;
	int64_t ix = (int64_t)dmin(dG * ux, dG - 1.0);
	int64_t iy = (int64_t)dmin(dG * uy, dG - 1.0);
	int64_t iz = (int64_t)dmin(dG * uz, dG - 1.0);
	cell = (uint32_t)(ix + iy * G + iz * (int64_t)G * G);
	return true;
}

// Records per tile of the staged decode: a block brings tiles of records
// into shared memory by bulk copies (the tile is 16-byte aligned when the
// source's records are, since kDecodeTile x record length is a multiple of
// 16), two buffers deep, and decodes its points from there.
constexpr int kDecodeTile = 512;
constexpr int kRegExtras = 2;
constexpr int kDecodeStageMaxRec = 96;  // two buffers: 96 KB of shared memory per block

// One thread per point. Writes the quantized position SoA and the count-grid
// cell, counts into the grid with warp-aggregated atomics and reduces
// attribute min/max (in registers, then shared memory, then one global atomic
// per block and statistic). With kStaged (one source, 16-byte aligned
// records, short records) the block walks tiles of kDecodeTile records staged
// in shared memory; else it reads each record in place (grid-stride).
template <bool kMulti, bool kStaged>
__global__ void __launch_bounds__(kDecodeThreads, 3) decode_count_kernel(DecodeParams p, uint32_t* __restrict__ grid, ChunkingOut out) {
	extern __shared__ uint4 stage16[];
	// shared statistics: [attr][comp] ordered min / max
	__shared__ unsigned long long s_mn[MAX_ATTRS][3];
	__shared__ unsigned long long s_mx[MAX_ATTRS][3];
	__shared__ unsigned int s_hist[256];
	for (int i = threadIdx.x; i < MAX_ATTRS * 3; i += blockDim.x) {
		(&s_mn[0][0])[i] = ~0ull;
		(&s_mx[0][0])[i] = 0ull;
	}
	for (int i = threadIdx.x; i < 256; i += blockDim.x) s_hist[i] = 0;
	__syncthreads();

	double pmn[3] = {CUDART_INF, CUDART_INF, CUDART_INF}, pmx[3] = {-CUDART_INF, -CUDART_INF, -CUDART_INF};
	double gmn = CUDART_INF, gmx = -CUDART_INF;
	// the first kRegExtras extra-attribute elements keep their min / max in
	// registers (ordered bit patterns), the others go to shared memory
	ExtraRange ex[kRegExtras];
	IntRange r_int, r_ret, r_nret, r_cls, r_sar, r_user, r_psid, r_r, r_g, r_b;
	r_int.init(); r_ret.init(); r_nret.init(); r_cls.init(); r_sar.init(); r_user.init(); r_psid.init(); r_r.init(); r_g.init(); r_b.init();

	auto point = [&](int64_t i, const uint8_t* r, const SourceDesc& sd) {
		double x, y, z;
		int32_t X, Y, Z;
		quantize_record(p, sd, r, x, y, z, X, Y, Z);
		uint32_t cell;
		const bool in_box = grid_cell(p, X, Y, Z, cell);
		if (!in_box) atomicCAS((unsigned long long*)&out.error[0], 0ull, (unsigned long long)(i + 1));
		out.X[i] = X;
		out.Y[i] = Y;
		out.Z[i] = Z;
		out.cell[i] = cell;
		// warp-aggregated increment of the count grid
		{
			unsigned active = __activemask();
			unsigned key = in_box ? cell : 0xffffffffu;
			unsigned peers = __match_any_sync(active, key);
			if (in_box && (__ffs(peers) - 1) == (int)(threadIdx.x & 31)) atomicAdd(grid + cell, (uint32_t)__popc(peers));
		}
		// attribute statistics (handlers, :391-545); position uses the
		// unquantized coordinate (:789-795)
		pmn[0] = dmin(pmn[0], x); pmn[1] = dmin(pmn[1], y); pmn[2] = dmin(pmn[2], z);
		pmx[0] = dmax(pmx[0], x); pmx[1] = dmax(pmx[1], y); pmx[2] = dmax(pmx[2], z);
		if (p.stat_intensity >= 0) r_int.add(ld<uint16_t>(r + 12));
		uint8_t bits = r[14];
		if (p.stat_retnum >= 0) r_ret.add(bits & 7);
		if (p.stat_nret >= 0) r_nret.add((bits >> 3) & 7);
		if (p.stat_class >= 0) {
			int c = r[15] & 31;
			r_cls.add(c);
			// one shared-memory add per class present in the warp
			const unsigned act = __activemask();
			const unsigned peers = __match_any_sync(act, c);
			if ((__ffs(peers) - 1) == (int)(threadIdx.x & 31)) atomicAdd(&s_hist[c], (unsigned)__popc(peers));
		}
		if (p.stat_sar >= 0) r_sar.add((int8_t)r[16]);
		if (p.stat_user >= 0) r_user.add(r[17]);
		if (p.stat_psid >= 0) r_psid.add(ld<uint16_t>(r + 18));
		if (p.stat_gps >= 0 && sd.src_gps >= 0) {
			double g = ld<double>(r + sd.src_gps);
			gmn = dmin(gmn, g);
			gmx = dmax(gmx, g);
		}
		if (p.stat_rgb >= 0 && sd.src_rgb >= 0) {
			r_r.add(ld<uint16_t>(r + sd.src_rgb));
			r_g.add(ld<uint16_t>(r + sd.src_rgb + 2));
			r_b.add(ld<uint16_t>(r + sd.src_rgb + 4));
		}
		int k = 0;  // element index over all extra attributes
		for (int e = 0; e < sd.n_extra; e++) {
			const ExtraDesc& d = sd.extra[e];
			for (int c = 0; c < d.num_elements && c < 3; c++, k++) {
				const uint8_t* q = r + d.src_off + c * d.element_size;
				double v = 0.0;
				switch (d.type) {
				case 0: v = (double)ld<int8_t>(q); break;
				case 1: v = (double)ld<int16_t>(q); break;
				case 2: v = (double)ld<int32_t>(q); break;
				case 3: v = (double)ld<int64_t>(q); break;
				case 10: v = (double)ld<uint8_t>(q); break;
				case 11: v = (double)ld<uint16_t>(q); break;
				case 12: v = (double)ld<uint32_t>(q); break;
				case 13: v = (double)ld<uint64_t>(q); break;
				case 20: v = (double)ld<float>(q); break;
				case 21: v = ld<double>(q); break;
				default: v = 0.0;
				}
				const unsigned long long o = ordered(v);
				if (!kMulti && k < kRegExtras) {  // one source: element k is the same statistic for every point
					// constant indices keep the accumulators in registers
#pragma unroll
					for (int q = 0; q < kRegExtras; q++)
						if (q == k) ex[q].add(o);
				} else {
					atomicMin(&s_mn[d.stat_index][c], o);
					atomicMax(&s_mx[d.stat_index][c], o);
				}
			}
		}
	};
	if constexpr (kStaged) {
		// tiles t0 = (blockIdx.x + k gridDim.x) kDecodeTile, k = 0, 1, ...;
		// tile k lands in buffer k & 1 by a bulk copy issued two tiles ahead,
		// so the copy of the next tile runs while this one is decoded
		__shared__ uint64_t bars[2];
		const SourceDesc& sd = p.src0;
		const int rl = sd.rec_len;
		uint8_t* const stage = reinterpret_cast<uint8_t*>(stage16);
		const size_t buf_bytes = (size_t)kDecodeTile * rl;
		auto buf = [&](int b) { return stage + b * buf_bytes; };
		const int64_t step = (int64_t)gridDim.x * kDecodeTile;
		const int64_t first = (int64_t)blockIdx.x * kDecodeTile;
		auto tile_count = [&](int64_t t0) { return (int)(p.n - t0 < kDecodeTile ? p.n - t0 : kDecodeTile); };
		// every tile but the cloud's last is a multiple of 16 bytes (kDecodeTile is)
		auto by_bulk = [&](int64_t t0) { return t0 < p.n && ((int64_t)tile_count(t0) * rl) % 16 == 0; };
		auto issue = [&](int64_t t0, int b) {
			bulk_load(buf(b), sd.recs + (t0 - sd.first) * rl, (uint32_t)(tile_count(t0) * rl), &bars[b]);
		};
		if (threadIdx.x == 0) {
			bulk_bar_init(&bars[0]);
			bulk_bar_init(&bars[1]);
			bulk_bar_fence_init();
		}
		__syncthreads();
		if (threadIdx.x == 0) {
			if (by_bulk(first)) issue(first, 0);
			if (by_bulk(first + step)) issue(first + step, 1);
		}
		uint32_t parity = 0u;  // bit b: phase parity of buffer b's barrier
		int k = 0;
		for (int64_t t0 = first; t0 < p.n; t0 += step, k++) {
			const int b = k & 1;
			const int cnt = tile_count(t0);
			if (by_bulk(t0)) {
				const bool ok = bulk_wait(&bars[b], (parity >> b) & 1u);
				parity ^= 1u << b;
				if (__syncthreads_or(!ok)) {
					// a copy that did not complete: report it; the other
					// buffer's copy, if one was issued, gets a bounded wait
					if (threadIdx.x == 0) {
						atomicCAS((unsigned long long*)&out.error[0], 0ull, (unsigned long long)(long long)-1);
						if (by_bulk(t0 + step)) bulk_wait(&bars[b ^ 1], (parity >> (b ^ 1)) & 1u);
					}
					return;
				}
			} else {
				// the cloud's last tile, not a multiple of 16 bytes
				const uint8_t* src = sd.recs + (t0 - sd.first) * rl;
				for (int i = threadIdx.x; i < cnt * rl; i += blockDim.x) buf(b)[i] = src[i];
				__syncthreads();
			}
			for (int j = threadIdx.x; j < cnt; j += blockDim.x) point(t0 + j, buf(b) + (size_t)j * rl, sd);
			__syncthreads();  // buffer b is free again
			if (threadIdx.x == 0 && by_bulk(t0 + 2 * step)) issue(t0 + 2 * step, b);
		}
	} else {
		const int64_t stride = (int64_t)gridDim.x * blockDim.x;
		for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride)
			with_source<kMulti>(p, i, [&](const SourceDesc& sd) { point(i, sd.recs + (i - sd.first) * sd.rec_len, sd); });
	}
	// block reduction of the register accumulators
	if (pmn[0] <= pmx[0]) {
		for (int c = 0; c < 3; c++) {
			atomicMin(&s_mn[p.stat_pos][c], ordered(pmn[c]));
			atomicMax(&s_mx[p.stat_pos][c], ordered(pmx[c]));
		}
	}
	if (p.stat_intensity >= 0) flush_int(out.stats, 0, r_int, s_mn[p.stat_intensity], s_mx[p.stat_intensity]);
	if (p.stat_retnum >= 0) flush_int(out.stats, 0, r_ret, s_mn[p.stat_retnum], s_mx[p.stat_retnum]);
	if (p.stat_nret >= 0) flush_int(out.stats, 0, r_nret, s_mn[p.stat_nret], s_mx[p.stat_nret]);
	if (p.stat_class >= 0) flush_int(out.stats, 0, r_cls, s_mn[p.stat_class], s_mx[p.stat_class]);
	if (p.stat_sar >= 0) flush_int(out.stats, 0, r_sar, s_mn[p.stat_sar], s_mx[p.stat_sar]);
	if (p.stat_user >= 0) flush_int(out.stats, 0, r_user, s_mn[p.stat_user], s_mx[p.stat_user]);
	if (p.stat_psid >= 0) flush_int(out.stats, 0, r_psid, s_mn[p.stat_psid], s_mx[p.stat_psid]);
	if (p.stat_rgb >= 0) {
		flush_int(out.stats, 0, r_r, s_mn[p.stat_rgb], s_mx[p.stat_rgb]);
		flush_int(out.stats, 1, r_g, s_mn[p.stat_rgb], s_mx[p.stat_rgb]);
		flush_int(out.stats, 2, r_b, s_mn[p.stat_rgb], s_mx[p.stat_rgb]);
	}
	if (p.stat_gps >= 0 && gmn <= gmx) {
		atomicMin(&s_mn[p.stat_gps][0], ordered(gmn));
		atomicMax(&s_mx[p.stat_gps][0], ordered(gmx));
	}
	if (!kMulti) {
		const SourceDesc& sd = p.src0;
		int k = 0;
		for (int e = 0; e < sd.n_extra; e++) {
			const ExtraDesc& d = sd.extra[e];
			for (int c = 0; c < d.num_elements && c < 3 && k < kRegExtras; c++, k++) {
#pragma unroll
				for (int q = 0; q < kRegExtras; q++) {
					if (q != k) continue;
					if (ex[q].mn != ~0ull) atomicMin(&s_mn[d.stat_index][c], ex[q].mn);
					if (ex[q].mx != 0ull) atomicMax(&s_mx[d.stat_index][c], ex[q].mx);
				}
			}
		}
	}
	__syncthreads();
	for (int i = threadIdx.x; i < MAX_ATTRS * 3; i += blockDim.x) {
		int a = i / 3, c = i % 3;
		unsigned long long vmn = s_mn[a][c], vmx = s_mx[a][c];
		if (vmn != ~0ull) atomicMin(&out.stats[a].mn[c], vmn);
		if (vmx != 0ull) atomicMax(&out.stats[a].mx[c], vmx);
	}
	for (int i = threadIdx.x; i < 256; i += blockDim.x)
		if (s_hist[i]) atomicAdd(&out.histogram[i], (unsigned long long)s_hist[i]);
}

// One pyramid level of createLUT: low cell (x, y, z) merges its 8 high
// cells unless one of them is already split (-1) or the sum exceeds the
// chunk capacity; then every non-empty high cell becomes a chunk.
template <class TH>
__global__ void lut_merge_kernel(const TH* __restrict__ high, int64_t* __restrict__ low, int level_low, int g_low,
                                 int64_t max_points, ChunkCell* __restrict__ chunks, int32_t* __restrict__ num_chunks, int capacity) {
	int64_t cells = (int64_t)g_low * g_low * g_low;
	int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= cells) return;
	int x = (int)(t % g_low), y = (int)((t / g_low) % g_low), z = (int)(t / ((int64_t)g_low * g_low));
	int g_high = 2 * g_low;
	int64_t vals[8];
	int64_t sum = 0;
	bool unmergeable = false;
	for (int j = 0; j < 8; j++) {
		int nx = 2 * x + ((j & 4) >> 2), ny = 2 * y + ((j & 2) >> 1), nz = 2 * z + (j & 1);
		int64_t v = (int64_t)high[nx + (int64_t)ny * g_high + (int64_t)nz * g_high * g_high];
		if (sizeof(TH) == 4) v = (int64_t)(uint32_t)v;
		vals[j] = v;
		if (v == -1) unmergeable = true; else sum += v;
	}
	int64_t idx_low = x + (int64_t)y * g_low + (int64_t)z * g_low * g_low;
	if (unmergeable || sum > max_points) {
		for (int j = 0; j < 8; j++) {
			if (vals[j] > 0) {
				int k = atomicAdd(num_chunks, 1);
				if (k < capacity) {
					ChunkCell c;
					c.level = level_low + 1;
					c.x = 2 * x + ((j & 4) >> 2);
					c.y = 2 * y + ((j & 2) >> 1);
					c.z = 2 * z + (j & 1);
					c.count = vals[j];
					chunks[k] = c;
				}
			}
		}
		low[idx_low] = -1;
	} else {
		low[idx_low] = sum;
	}
}

__global__ void lut_fill_kernel(const ChunkCell* __restrict__ chunks, int grid_size, int level_max, int32_t* __restrict__ lut) {
	ChunkCell c = chunks[blockIdx.x];
	int size = 1 << (level_max - c.level);
	int64_t cells = (int64_t)size * size * size;
	for (int64_t t = threadIdx.x; t < cells; t += blockDim.x) {
		int ox = (int)(t % size), oy = (int)((t / size) % size), oz = (int)(t / ((int64_t)size * size));
		int64_t x = (int64_t)size * c.x + ox, y = (int64_t)size * c.y + oy, z = (int64_t)size * c.z + oz;
		lut[x + y * grid_size + z * (int64_t)grid_size * grid_size] = (int32_t)blockIdx.x;
	}
}

__global__ void assign_kernel(const uint32_t* __restrict__ cell, const int32_t* __restrict__ lut, int64_t n, int chunk_base,
                              uint32_t* __restrict__ chunk_of, uint32_t* __restrict__ ids, int64_t* error) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	int32_t c = lut[cell[i]];
	c = c < 0 ? -1 : c - chunk_base;
	if (c < 0) {
		atomicCAS((unsigned long long*)&error[1], 0ull, (unsigned long long)(i + 1));
		c = 0;
	}
	chunk_of[i] = (uint32_t)c;
	ids[i] = (uint32_t)i;
}

// ---------------------------------------------------- parts of a large cloud
// A part of a cloud is the run of chunks k0 .. k1 - 1; its points are
// selected from the records of one source in input order (the order the
// reference's single chunker thread appends them to the chunk files).
constexpr int kSelThreads = 256;
constexpr int kSelItems = 8;
constexpr int64_t kSelTile = (int64_t)kSelThreads * kSelItems;

__device__ __forceinline__ bool in_part(const DecodeParams& p, const uint8_t* r, const int32_t* __restrict__ lut, int k0, int k1) {
	double x, y, z;
	int32_t X, Y, Z;
	quantize_record(p, p.src0, r, x, y, z, X, Y, Z);
	uint32_t cell;
	if (!grid_cell(p, X, Y, Z, cell)) return false;
	const int c = __ldg(lut + cell);
	return c >= k0 && c < k1;
}

// points of the part among recs[0..n), per tile of kSelTile points
__global__ void __launch_bounds__(kSelThreads) select_count_kernel(DecodeParams p, const uint8_t* __restrict__ recs, int64_t n,
                                                                  const int32_t* __restrict__ lut, int k0, int k1,
                                                                  uint32_t* __restrict__ counts) {
	__shared__ uint32_t s_cnt;
	if (threadIdx.x == 0) s_cnt = 0;
	__syncthreads();
	const int64_t base = (int64_t)blockIdx.x * kSelTile;
	const int rl = p.src0.rec_len;
	uint32_t c = 0;
	for (int e = 0; e < kSelItems; e++) {
		const int64_t i = base + (int64_t)e * kSelThreads + threadIdx.x;
		if (i < n && in_part(p, recs + i * rl, lut, k0, k1)) c++;
	}
	for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
	if ((threadIdx.x & 31) == 0 && c) atomicAdd(&s_cnt, c);
	__syncthreads();
	if (threadIdx.x == 0) counts[blockIdx.x] = s_cnt;
}

// copies the part's records, in input order, to out at *fill + tile offset
__global__ void __launch_bounds__(kSelThreads) select_copy_kernel(DecodeParams p, const uint8_t* __restrict__ recs, int64_t n,
                                                                 const int32_t* __restrict__ lut, int k0, int k1,
                                                                 const uint32_t* __restrict__ tile_off, const int64_t* __restrict__ fill,
                                                                 uint8_t* __restrict__ out) {
	__shared__ uint32_t s_warp[kSelThreads / 32];
	const int64_t base = (int64_t)blockIdx.x * kSelTile;
	const int rl = p.src0.rec_len;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int64_t pos = *fill + tile_off[blockIdx.x];
	for (int e = 0; e < kSelItems; e++) {
		const int64_t i = base + (int64_t)e * kSelThreads + threadIdx.x;
		const bool f = i < n && in_part(p, recs + i * rl, lut, k0, k1);
		const unsigned ballot = __ballot_sync(0xffffffffu, f);
		if (lane == 0) s_warp[warp] = __popc(ballot);
		__syncthreads();
		uint32_t before = 0, total = 0;
		for (int w = 0; w < kSelThreads / 32; w++) {
			const uint32_t v = s_warp[w];
			before += w < warp ? v : 0;
			total += v;
		}
		if (f) {
			const uint8_t* r = recs + i * rl;
			uint8_t* o = out + (pos + before + __popc(ballot & ((1u << lane) - 1))) * rl;
			for (int b = 0; b < rl; b++) o[b] = r[b];
		}
		pos += total;
		__syncthreads();
	}
}

__global__ void select_advance_kernel(int64_t* fill, const uint32_t* __restrict__ tile_off, int64_t tiles) { *fill += tile_off[tiles]; }

// out_recs[i] = recs[ids[i]], oX/oY/oZ[i] = X/Y/Z[ids[i]]
__global__ void gather_points_kernel(const uint32_t* __restrict__ ids, int64_t n, const uint8_t* __restrict__ recs, int rec_len,
                                     const int32_t* __restrict__ X, const int32_t* __restrict__ Y, const int32_t* __restrict__ Z,
                                     uint8_t* __restrict__ out_recs, int32_t* __restrict__ oX, int32_t* __restrict__ oY,
                                     int32_t* __restrict__ oZ) {
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint32_t id = ids[i];
	const uint8_t* r = recs + (int64_t)id * rec_len;
	uint8_t* o = out_recs + i * rec_len;
	for (int b = 0; b < rec_len; b++) o[b] = r[b];
	oX[i] = X[id];
	oY[i] = Y[id];
	oZ[i] = Z[id];
}

// starts[k] = first position of key k in the ascending keys[0..n), for every
// k in 0..num_keys (starts[num_keys] = n); keys absent get the next start
__global__ void segment_starts_kernel(const uint32_t* __restrict__ keys, int64_t n, int num_keys, int64_t* __restrict__ starts) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i > n) return;
	const int64_t lo = i == 0 ? -1 : (int64_t)keys[i - 1];
	const int64_t hi = i == n ? (int64_t)num_keys : (int64_t)keys[i];
	for (int64_t k = lo + 1; k <= hi && k <= num_keys; k++) starts[k] = i;
}

__global__ void iota_kernel(uint32_t* __restrict__ out, int64_t n) {
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = (uint32_t)i;
}

}  // namespace

void launch_iota(uint32_t* out, int64_t n, DeviceMem& mem) {
	if (n == 0) return;
	iota_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(out, n);
	PCG_LAUNCHED();
}

void launch_segment_starts(const uint32_t* keys, int64_t n, int num_keys, int64_t* starts, DeviceMem& mem) {
	segment_starts_kernel<<<(unsigned)ceil_div(n + 1, 256), 256, 0, mem.stream()>>>(keys, n, num_keys, starts);
	PCG_LAUNCHED();
}

void launch_select_part(const DecodeParams& p, const uint8_t* recs, int64_t n, const int32_t* lut, int k0, int k1, int64_t* fill,
                        uint8_t* out, DeviceMem& mem) {
	if (n == 0) return;
	const int64_t tiles = ceil_div(n, kSelTile);
	uint32_t* counts = mem.alloc<uint32_t>(tiles);
	uint32_t* offs = mem.alloc<uint32_t>(tiles + 1);
	select_count_kernel<<<(unsigned)tiles, kSelThreads, 0, mem.stream()>>>(p, recs, n, lut, k0, k1, counts);
	PCG_LAUNCHED();
	exclusive_scan_u32(counts, offs, tiles, true, mem);
	select_copy_kernel<<<(unsigned)tiles, kSelThreads, 0, mem.stream()>>>(p, recs, n, lut, k0, k1, offs, fill, out);
	PCG_LAUNCHED();
	select_advance_kernel<<<1, 1, 0, mem.stream()>>>(fill, offs, tiles);
	PCG_LAUNCHED();
	mem.free(counts);
	mem.free(offs);
}

void launch_gather_points(const uint32_t* ids, int64_t n, const uint8_t* recs, int rec_len, const int32_t* X, const int32_t* Y,
                          const int32_t* Z, uint8_t* out_recs, int32_t* oX, int32_t* oY, int32_t* oZ, DeviceMem& mem) {
	if (n == 0) return;
	gather_points_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(ids, n, recs, rec_len, X, Y, Z, out_recs, oX, oY, oZ);
	PCG_LAUNCHED();
}

void launch_decode_count(const DecodeParams& p, uint32_t* grid, ChunkingOut& out, DeviceMem& mem) {
	if (p.n == 0) return;
	int dev = 0;
	PCG_CUDA(cudaGetDevice(&dev));
	int sms = 0;
	PCG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
	int64_t blocks = ceil_div(p.n, kDecodeThreads * 4);
	int64_t cap = (int64_t)sms * 8;
	if (blocks > cap) blocks = cap;
	if (blocks < 1) blocks = 1;
	// bulk copies of whole tiles: 16-byte aligned records (kDecodeTile
	// records are a multiple of 16 bytes, so every tile starts aligned)
	const bool staged = p.nsrc == 1 && p.src0.rec_len <= kDecodeStageMaxRec && (reinterpret_cast<uintptr_t>(p.src0.recs) & 15) == 0 &&
	                    p.src0.first == 0;
	if (p.nsrc > 1) {
		decode_count_kernel<true, false><<<(unsigned)blocks, kDecodeThreads, 0, mem.stream()>>>(p, grid, out);
	} else if (staged) {
		const size_t smem = 2 * (size_t)kDecodeTile * p.src0.rec_len;
		if (smem > 48 * 1024)
			PCG_CUDA(cudaFuncSetAttribute(decode_count_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
		int64_t tb = ceil_div(p.n, kDecodeTile);
		if (tb > cap) tb = cap;
		decode_count_kernel<false, true><<<(unsigned)tb, kDecodeThreads, smem, mem.stream()>>>(p, grid, out);
	} else {
		decode_count_kernel<false, false><<<(unsigned)blocks, kDecodeThreads, 0, mem.stream()>>>(p, grid, out);
	}
	PCG_LAUNCHED();
}

void launch_lut_merge(const uint32_t* grid, int grid_size, int64_t max_points_per_chunk, ChunkCell* chunks,
                      int32_t* num_chunks, int capacity, DeviceMem& mem) {
	cudaStream_t s = mem.stream();
	int level_max = bits_for((uint64_t)grid_size) - 1;
	int64_t* prev = nullptr;
	for (int level_low = level_max - 1; level_low >= 0; level_low--) {
		int g_low = 1 << level_low;
		int64_t cells = (int64_t)g_low * g_low * g_low;
		int64_t* low = mem.alloc<int64_t>(cells);
		unsigned blocks = (unsigned)ceil_div(cells, 256);
		if (level_low == level_max - 1)
			lut_merge_kernel<uint32_t><<<blocks, 256, 0, s>>>(grid, low, level_low, g_low, max_points_per_chunk, chunks, num_chunks, capacity);
		else
			lut_merge_kernel<int64_t><<<blocks, 256, 0, s>>>(prev, low, level_low, g_low, max_points_per_chunk, chunks, num_chunks, capacity);
		PCG_LAUNCHED();
		if (prev) mem.free(prev);
		prev = low;
	}
	if (prev) mem.free(prev);
}

void launch_lut_fill(const ChunkCell* chunks, int num_chunks, int grid_size, int32_t* lut, DeviceMem& mem) {
	if (num_chunks == 0) return;
	int level_max = bits_for((uint64_t)grid_size) - 1;
	lut_fill_kernel<<<num_chunks, 256, 0, mem.stream()>>>(chunks, grid_size, level_max, lut);
	PCG_LAUNCHED();
}

void launch_assign_chunks(const uint32_t* cell, const int32_t* lut, int64_t n, int chunk_base, uint32_t* chunk_of, uint32_t* ids,
                          int64_t* error, DeviceMem& mem) {
	if (n == 0) return;
	assign_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(cell, lut, n, chunk_base, chunk_of, ids, error);
	PCG_LAUNCHED();
}

}  // namespace pcg
