// Output stage: node payloads are written into the octree.bin image in
// completion order (Writer::writeAndUnload, indexer.cpp:1453-1516). Every
// point record is assembled from its LAS record exactly like the chunker's
// attribute handlers build it (chunker_countsort_laszip.cpp:380-658,
// 770-803), so the sampling stages only move 4-byte point ids.

#include "devutil.cuh"
#include "output.h"

namespace pcg {

namespace {

template <class T> __device__ __forceinline__ void st(uint8_t* p, T v) { memcpy(p, &v, sizeof(T)); }

// Output record of a point from its LAS record r, as the chunker's handlers
// build it: bytes no handler of the source writes stay zero (the batch
// buffer is cleared, :729-732), the standard attributes go to their output
// offsets, then the extra bytes to theirs (a kept extra can land on another
// attribute's bytes, :565-653). has_col then overrides rgb with col, as
// poisson_average rewrites the colour of the chunk records
// (sampler_poisson_average.h:437-446).
__device__ void assemble_record(const uint8_t* r, const DecodeParams& p, const SourceDesc& sd, uint64_t col, bool has_col, uint8_t* dst) {
	if (sd.zero_fill)
		for (int k = 12; k < p.bpp; k++) dst[k] = 0;
	double x, y, z;
	int32_t X, Y, Z;
	quantize_record(p, sd, r, x, y, z, X, Y, Z);
	st<int32_t>(dst + 0, X);
	st<int32_t>(dst + 4, Y);
	st<int32_t>(dst + 8, Z);
	if (p.off_intensity >= 0) { dst[p.off_intensity] = r[12]; dst[p.off_intensity + 1] = r[13]; }
	if (p.off_retnum >= 0) dst[p.off_retnum] = r[14] & 7;
	if (p.off_nret >= 0) dst[p.off_nret] = (r[14] >> 3) & 7;
	if (p.off_class >= 0) dst[p.off_class] = r[15] & 31;
	if (p.off_sar >= 0) dst[p.off_sar] = r[16];
	if (p.off_user >= 0) dst[p.off_user] = r[17];
	if (p.off_psid >= 0) { dst[p.off_psid] = r[18]; dst[p.off_psid + 1] = r[19]; }
	if (p.off_gps >= 0 && sd.src_gps >= 0)
		for (int k = 0; k < 8; k++) dst[p.off_gps + k] = r[sd.src_gps + k];
	if (p.off_rgb >= 0 && sd.src_rgb >= 0)
		for (int k = 0; k < 6; k++) dst[p.off_rgb + k] = r[sd.src_rgb + k];
	for (int e = 0; e < sd.n_extra; e++) {
		const ExtraDesc& d = sd.extra[e];
		for (int k = 0; k < d.size; k++) dst[d.dst_off + k] = r[d.src_off + k];
	}
	if (has_col) {
		st<uint16_t>(dst + p.off_rgb, (uint16_t)(col & 0xffff));
		st<uint16_t>(dst + p.off_rgb + 2, (uint16_t)((col >> 16) & 0xffff));
		st<uint16_t>(dst + p.off_rgb + 4, (uint16_t)((col >> 32) & 0xffff));
	}
}

// The six rgb bytes of a point's output record (before any colour
// averaging): the source's colour, or zeros, with the bytes of kept extras
// that land on them.
__device__ __forceinline__ uint64_t record_rgb(const uint8_t* r, const DecodeParams& p, const SourceDesc& sd) {
	uint64_t c = 0;  // the six bytes, little endian: r | g << 16 | b << 32
	if (sd.src_rgb >= 0)
		for (int k = 0; k < 6; k++) c |= (uint64_t)r[sd.src_rgb + k] << (8 * k);
	for (int e = 0; e < sd.n_extra; e++) {
		const ExtraDesc& d = sd.extra[e];
		for (int k = 0; k < d.size; k++) {
			const int o = d.dst_off + k - p.off_rgb;
			if (o >= 0 && o < 6) c = (c & ~(0xffull << (8 * o))) | ((uint64_t)r[d.src_off + k] << (8 * o));
		}
	}
	return c;
}

constexpr int kOutThreads = 256;

// words of shared scratch per thread for one LAS record (4-byte aligned
// cover of rec_len bytes at any offset)
__host__ __device__ __forceinline__ int rec_words(int rec_len) { return (rec_len + 3) / 4 + 1; }

// 256 output points per CTA over the whole octree.bin image (payloads are
// contiguous in completion order, so a CTA spans one or a few payloads).
// Each thread copies its LAS record into shared memory with aligned 4-byte
// loads (byte loads for the last records, whose cover would reach past the
// source's records), assembles the output record there -- requantizing the
// record's own coordinates -- and the CTA writes its span with 4-byte
// stores.
template <bool kMulti>
__global__ void __launch_bounds__(kOutThreads) write_payloads_kernel(DecodeParams p, const PayloadItem* __restrict__ items,
                                                                    const int32_t* __restrict__ chunk_item, int64_t total,
                                                                    uint8_t* __restrict__ out) {
	extern __shared__ uint32_t smem_words[];
	const int bpp = p.bpp, rw = rec_words(p.max_rec_len);
	uint32_t* scratch = smem_words + threadIdx.x * rw;
	uint8_t* stage = reinterpret_cast<uint8_t*>(smem_words + kOutThreads * rw);
	const int64_t q0 = (int64_t)blockIdx.x * kOutThreads, q = q0 + threadIdx.x;
	const int64_t nthis = total - q0 < kOutThreads ? total - q0 : kOutThreads;
	if (q < total) {
		int k = chunk_item[blockIdx.x];
		while (items[k].out_offset + items[k].count <= q) k++;
		const PayloadItem& it = items[k];
		const int64_t t = q - it.out_offset;
		const uint32_t id = it.ids[t];
		with_source<kMulti>(p, id, [&](const SourceDesc& sd) {
			const int rl = sd.rec_len;
			const uint8_t* recs = sd.recs;
			const int64_t start = ((int64_t)id - sd.first) * rl;
			const int64_t w0 = start >> 2, w1 = (start + rl + 3) >> 2;
			const bool aligned = (reinterpret_cast<uintptr_t>(recs) & 3) == 0;
			const uint8_t* r;
			if (aligned && w1 * 4 <= sd.count * rl) {
				const uint32_t* src = reinterpret_cast<const uint32_t*>(recs) + w0;
				for (int w = 0; w < (int)(w1 - w0); w++) scratch[w] = src[w];
				r = reinterpret_cast<const uint8_t*>(scratch) + (start & 3);
			} else {
				uint8_t* sb = reinterpret_cast<uint8_t*>(scratch);
				for (int w = 0; w < rl; w++) sb[w] = recs[start + w];
				r = sb;
			}
			assemble_record(r, p, sd, it.cols ? it.cols[t] : 0ull, it.cols != nullptr, stage + threadIdx.x * bpp);
		});
	}
	__syncthreads();
	const int64_t bytes = nthis * bpp;
	uint8_t* dst = out + q0 * bpp;
	// head bytes up to a 4-byte boundary, whole words, tail bytes
	int64_t head = (int64_t)((4 - (reinterpret_cast<uintptr_t>(dst) & 3)) & 3);
	if (head > bytes) head = bytes;
	const int64_t words = (bytes - head) >> 2;
	if (threadIdx.x < head) dst[threadIdx.x] = stage[threadIdx.x];
	uint32_t* dw = reinterpret_cast<uint32_t*>(dst + head);
	for (int64_t w = threadIdx.x; w < words; w += kOutThreads) {
		const uint8_t* sp = stage + head + 4 * w;
		dw[w] = (uint32_t)sp[0] | ((uint32_t)sp[1] << 8) | ((uint32_t)sp[2] << 16) | ((uint32_t)sp[3] << 24);
	}
	for (int64_t b = head + 4 * words + threadIdx.x; b < bytes; b += kOutThreads) dst[b] = stage[b];
}

template <bool kMulti>
__global__ void fill_colors_kernel(DecodeParams p, const uint32_t* __restrict__ ids, int64_t n, uint64_t* __restrict__ cols) {
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint32_t id = ids[i];
	with_source<kMulti>(p, id, [&](const SourceDesc& sd) { cols[i] = record_rgb(sd.recs + ((int64_t)id - sd.first) * sd.rec_len, p, sd); });
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
                             const uint64_t* __restrict__ cols, const int4* __restrict__ rec, uint32_t* __restrict__ acc_ids,
                             uint64_t* __restrict__ acc_cols, int4* __restrict__ acc_rec, uint32_t* __restrict__ rej_ids) {
	int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= n) return;
	uint32_t a = pre[j];
	if (accepted[j]) {
		acc_ids[a] = ids[j];
		if (acc_cols) acc_cols[a] = cols[j];
		if (acc_rec) acc_rec[a] = rec[j];
	} else if (rej_ids) {
		rej_ids[j - a] = ids[j];
	}
}

}  // namespace

void launch_write_payloads(const DecodeParams& p, const std::vector<PayloadItem>& items, const PayloadItem* d_items, uint8_t* out,
                           DeviceMem& mem) {
	if (items.empty()) return;
	const int64_t total = items.back().out_offset + items.back().count;
	if (total == 0) return;
	size_t smem = (size_t)kOutThreads * (rec_words(p.max_rec_len) * 4 + p.bpp);
	if (smem > 200 * 1024) throw PcgError(1, "point records too long for the payload writer (record + output > 800 bytes)");
	auto kernel = p.nsrc > 1 ? write_payloads_kernel<true> : write_payloads_kernel<false>;
	if (smem > 48 * 1024) PCG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	// the payload holding the first point of every 256-point chunk
	const int64_t chunks = ceil_div(total, kOutThreads);
	std::vector<int32_t> chunk_item(chunks);
	size_t k = 0;
	for (int64_t c = 0; c < chunks; c++) {
		const int64_t q = c * kOutThreads;
		while (items[k].out_offset + items[k].count <= q) k++;
		chunk_item[c] = (int32_t)k;
	}
	int32_t* d_ci = mem.alloc<int32_t>(chunks);
	PCG_CUDA(cudaMemcpyAsync(d_ci, chunk_item.data(), chunks * sizeof(int32_t), cudaMemcpyHostToDevice, mem.stream()));
	kernel<<<(unsigned)chunks, kOutThreads, smem, mem.stream()>>>(p, d_items, d_ci, total, out);
	PCG_LAUNCHED();
	mem.free(d_ci);
}

void launch_fill_colors(const DecodeParams& p, const uint32_t* ids, int64_t n, uint64_t* cols, DeviceMem& mem) {
	if (n == 0) return;
	if (p.nsrc > 1) fill_colors_kernel<true><<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(p, ids, n, cols);
	else fill_colors_kernel<false><<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(p, ids, n, cols);
	PCG_LAUNCHED();
}

void launch_gather_u32(const uint32_t* src, const int64_t* idx, int64_t n, uint32_t* dst, DeviceMem& mem) {
	if (n == 0) return;
	gather_u32_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(src, idx, n, dst);
	PCG_LAUNCHED();
}

void launch_split(const uint8_t* accepted, int64_t n, const uint32_t* ids, const uint64_t* cols, const int4* rec, uint32_t* pre,
                  uint32_t* acc_ids, uint64_t* acc_cols, int4* acc_rec, uint32_t* rej_ids, DeviceMem& mem) {
	if (n == 0) return;
	uint32_t* f = mem.alloc<uint32_t>(n);
	flags_to_u32_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(accepted, n, f);
	PCG_LAUNCHED();
	exclusive_scan_u32(f, pre, n, true, mem);
	mem.free(f);
	split_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, mem.stream()>>>(accepted, pre, n, ids, cols, rec, acc_ids, acc_cols, acc_rec,
	                                                                 rej_ids);
	PCG_LAUNCHED();
}

}  // namespace pcg
