// Output stage: node payloads are written into the octree.bin image in
// completion order (Writer::writeAndUnload, indexer.cpp:1453-1516). Every
// point record is assembled from its LAS record exactly like the chunker's
// attribute handlers build it (chunker_countsort_laszip.cpp:380-658,
// 770-803), so the sampling stages only move 4-byte point ids.

#include "output.h"

namespace pcg {

namespace {

template <class T> __device__ __forceinline__ void st(uint8_t* p, T v) { memcpy(p, &v, sizeof(T)); }

// Output record of point `id`; cols != ~0 overrides rgb (poisson_average).
__device__ void assemble_record(const uint8_t* __restrict__ recs, const DecodeParams& p, const int32_t* X, const int32_t* Y,
                                const int32_t* Z, uint32_t id, uint64_t col, bool has_col, uint8_t* dst) {
	const uint8_t* r = recs + (int64_t)id * p.rec_len;
	st<int32_t>(dst + 0, X[id]);
	st<int32_t>(dst + 4, Y[id]);
	st<int32_t>(dst + 8, Z[id]);
	if (p.off_intensity >= 0) { dst[p.off_intensity] = r[12]; dst[p.off_intensity + 1] = r[13]; }
	if (p.off_retnum >= 0) dst[p.off_retnum] = r[14] & 7;
	if (p.off_nret >= 0) dst[p.off_nret] = (r[14] >> 3) & 7;
	if (p.off_class >= 0) dst[p.off_class] = r[15] & 31;
	if (p.off_sar >= 0) dst[p.off_sar] = r[16];
	if (p.off_user >= 0) dst[p.off_user] = r[17];
	if (p.off_psid >= 0) { dst[p.off_psid] = r[18]; dst[p.off_psid + 1] = r[19]; }
	if (p.off_gps >= 0)
		for (int k = 0; k < 8; k++) dst[p.off_gps + k] = r[p.src_gps + k];
	if (p.off_rgb >= 0) {
		if (has_col) {
			st<uint16_t>(dst + p.off_rgb, (uint16_t)(col & 0xffff));
			st<uint16_t>(dst + p.off_rgb + 2, (uint16_t)((col >> 16) & 0xffff));
			st<uint16_t>(dst + p.off_rgb + 4, (uint16_t)((col >> 32) & 0xffff));
		} else {
			for (int k = 0; k < 6; k++) dst[p.off_rgb + k] = r[p.src_rgb + k];
		}
	}
	for (int e = 0; e < p.n_extra; e++) {
		const ExtraDesc& d = p.extra[e];
		for (int k = 0; k < d.size; k++) dst[d.dst_off + k] = r[d.src_off + k];
	}
}

constexpr int kOutThreads = 256;

// One CTA per payload; records are staged in shared memory so the global
// writes of a CTA are one contiguous, coalesced span.
__global__ void __launch_bounds__(kOutThreads) write_payloads_kernel(const uint8_t* __restrict__ recs, DecodeParams p, const int32_t* X,
                                                                    const int32_t* Y, const int32_t* Z, const PayloadItem* __restrict__ items,
                                                                    uint8_t* __restrict__ out) {
	extern __shared__ uint8_t stage[];
	const PayloadItem it = items[blockIdx.x];
	const int bpp = p.bpp;
	uint8_t* dst_base = out + it.out_offset * bpp;
	for (int64_t t0 = 0; t0 < it.count; t0 += kOutThreads) {
		int64_t t = t0 + threadIdx.x;
		int64_t nthis = it.count - t0 < kOutThreads ? it.count - t0 : kOutThreads;
		if (t < it.count) {
			uint64_t col = it.cols ? it.cols[t] : 0ull;
			assemble_record(recs, p, X, Y, Z, it.ids[t], col, it.cols != nullptr, stage + threadIdx.x * bpp);
		}
		__syncthreads();
		int64_t bytes = nthis * bpp;
		uint8_t* dst = dst_base + t0 * bpp;
		for (int64_t b = threadIdx.x; b < bytes; b += kOutThreads) dst[b] = stage[b];
		__syncthreads();
	}
}

__global__ void fill_colors_kernel(const uint8_t* __restrict__ recs, int rec_len, int src_rgb, const uint32_t* __restrict__ ids, int64_t n,
                                   uint64_t* __restrict__ cols) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint8_t* r = recs + (int64_t)ids[i] * rec_len + src_rgb;
	uint64_t red = (uint64_t)r[0] | ((uint64_t)r[1] << 8);
	uint64_t green = (uint64_t)r[2] | ((uint64_t)r[3] << 8);
	uint64_t blue = (uint64_t)r[4] | ((uint64_t)r[5] << 8);
	cols[i] = red | (green << 16) | (blue << 32);
}

__global__ void gather_u32_kernel(const uint32_t* __restrict__ src, const int64_t* __restrict__ idx, int64_t n, uint32_t* __restrict__ dst) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) dst[i] = src[idx[i]];
}

__global__ void flags_to_u32_kernel(const uint8_t* __restrict__ f, int64_t n, uint32_t* __restrict__ o) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) o[i] = f[i];
}

__global__ void split_kernel(const uint8_t* __restrict__ accepted, const uint32_t* __restrict__ pre, int64_t n, const uint32_t* __restrict__ ids,
                             const uint64_t* __restrict__ cols, uint32_t* __restrict__ acc_ids, uint64_t* __restrict__ acc_cols,
                             uint32_t* __restrict__ rej_ids) {
	int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= n) return;
	uint32_t a = pre[j];
	if (accepted[j]) {
		acc_ids[a] = ids[j];
		if (acc_cols) acc_cols[a] = cols[j];
	} else if (rej_ids) {
		rej_ids[j - a] = ids[j];
	}
}

}  // namespace

void launch_write_payloads(const uint8_t* d_recs, const DecodeParams& p, const int32_t* X, const int32_t* Y, const int32_t* Z,
                           const PayloadItem* items, int num_items, uint8_t* out, DeviceMem& mem) {
	if (num_items == 0) return;
	size_t smem = (size_t)kOutThreads * p.bpp;
	if (smem > 48 * 1024) PCG_CUDA(cudaFuncSetAttribute(write_payloads_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	write_payloads_kernel<<<num_items, kOutThreads, smem, mem.stream()>>>(d_recs, p, X, Y, Z, items, out);
	PCG_LAUNCHED();
}

void launch_fill_colors(const uint8_t* d_recs, int rec_len, int src_rgb, const uint32_t* ids, int64_t n, uint64_t* cols, DeviceMem& mem) {
	if (n == 0) return;
	fill_colors_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(d_recs, rec_len, src_rgb, ids, n, cols);
	PCG_LAUNCHED();
}

void launch_gather_u32(const uint32_t* src, const int64_t* idx, int64_t n, uint32_t* dst, DeviceMem& mem) {
	if (n == 0) return;
	gather_u32_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(src, idx, n, dst);
	PCG_LAUNCHED();
}

void launch_split(const uint8_t* accepted, int64_t n, const uint32_t* ids, const uint64_t* cols, uint32_t* pre, uint32_t* acc_ids,
                  uint64_t* acc_cols, uint32_t* rej_ids, DeviceMem& mem) {
	if (n == 0) return;
	uint32_t* f = mem.alloc<uint32_t>(n);
	flags_to_u32_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(accepted, n, f);
	PCG_LAUNCHED();
	exclusive_scan_u32(f, pre, n, true, mem);
	mem.free(f);
	split_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(accepted, pre, n, ids, cols, acc_ids, acc_cols, rej_ids);
	PCG_LAUNCHED();
}

}  // namespace pcg
