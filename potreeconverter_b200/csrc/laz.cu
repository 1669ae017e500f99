// LAZ decode on the device: one LASzip chunk per block (its lane 0 runs the
// chunk's arithmetic decoder, laz.cuh), all chunks of a source at once, each
// with its models in the block's shared memory as far as they fit and the
// rest in its own slice of a global arena; the decoded point records land
// where the LAS path keeps a source's records, so the rest of the pipeline
// is unchanged.
// The reference decodes the same chunks sequentially per file, twice
// (countPointsInCells and distributePoints, chunker_countsort_laszip.cpp:
// 194-203, 750-772).

#include "kernels.h"
#include "laz.cuh"

namespace pcg {

namespace {

// words of shared memory the decoder state takes (16-byte multiple)
constexpr uint32_t kStateWords = (uint32_t)((sizeof(laz::ChunkState) + 15) / 16 * 4);

// models go to the block's shared memory first (fast_words of it, after the
// decoder state), then to the chunk's slice of the global arena
__global__ void __launch_bounds__(32) laz_decode_kernel(const uint8_t* __restrict__ bytes, uint64_t base, const laz::Chunk* __restrict__ chunks,
                                                        int c0, int n, laz::Layout L, uint32_t fast_words, uint32_t* __restrict__ arena,
                                                        uint32_t words, uint8_t* __restrict__ out, int* __restrict__ bad) {
	// the decoder's state first, then its fast model region
	extern __shared__ __align__(16) uint32_t smem[];
	if (threadIdx.x != 0 || (int)blockIdx.x >= n) return;
	laz::ChunkState& S = *reinterpret_cast<laz::ChunkState*>(smem);
	uint32_t* fast = smem + kStateWords;
	const int c = c0 + (int)blockIdx.x;
	const laz::Chunk ch = chunks[c];
	const bool ok = laz::decode_chunk(bytes + (ch.start - base), bytes + (ch.end - base), ch.count, L, S, fast_words ? fast : nullptr, fast_words,
	                                  arena + (size_t)blockIdx.x * words, words, out + ch.first * (int64_t)L.rec_len);
	if (!ok) atomicCAS(bad, 0, c + 1);
}

}  // namespace

void launch_laz_decode(const uint8_t* d_bytes, uint64_t base, const std::vector<laz::Chunk>& chunks, const laz::Layout& L, uint8_t* d_out,
                       DeviceMem& mem) {
	if (chunks.empty()) return;
	const uint64_t end = chunks.back().end;
	for (const auto& c : chunks)
		if (c.start < base || c.end > end || c.start >= c.end) throw PcgError(1, "malformed LAZ chunk table");
	laz::Chunk* d_chunks = mem.alloc<laz::Chunk>(chunks.size());
	PCG_CUDA(cudaMemcpyAsync(d_chunks, chunks.data(), chunks.size() * sizeof(laz::Chunk), cudaMemcpyHostToDevice, mem.stream()));
	const uint32_t words = laz::arena_words(L);
	// chunks decoded at once: all, or as many as about 4 GiB of model arenas hold
	const int64_t fit = std::max<int64_t>(1, (int64_t(4) << 30) / ((int64_t)words * 4));
	const int wave = (int)std::min<int64_t>((int64_t)chunks.size(), fit);
	uint32_t* arena = mem.alloc<uint32_t>((size_t)wave * words);
	int* d_bad = mem.alloc<int>(1);
	PCG_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), mem.stream()));
	// shared memory per block: as much as keeps every block of a wave
	// resident at once, within the per-block limit
	int dev = 0, sms = 0, per_sm = 0, per_block = 0;
	PCG_CUDA(cudaGetDevice(&dev));
	PCG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
	PCG_CUDA(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
	PCG_CUDA(cudaDeviceGetAttribute(&per_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
	const int blocks_per_sm = std::max(1, (wave + sms - 1) / sms);
	size_t smem_bytes = std::min<size_t>((size_t)per_block, (size_t)per_sm / blocks_per_sm);
	smem_bytes = smem_bytes > 1024 ? ((smem_bytes - 1024) & ~size_t(15)) : 0;
	const size_t state_bytes = (size_t)kStateWords * 4;
	if (smem_bytes < state_bytes) smem_bytes = state_bytes;
	const uint32_t fast_words = (uint32_t)((smem_bytes - state_bytes) / 4);
	if (smem_bytes > 48 * 1024) PCG_CUDA(cudaFuncSetAttribute(laz_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes));
	for (int c0 = 0; c0 < (int)chunks.size(); c0 += wave) {
		const int n = std::min<int>(wave, (int)chunks.size() - c0);
		laz_decode_kernel<<<(unsigned)n, 32, smem_bytes, mem.stream()>>>(d_bytes, base, d_chunks, c0, n, L, fast_words, arena, words, d_out,
		                                                                  d_bad);
		PCG_LAUNCHED();
	}
	int bad = 0;
	PCG_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, mem.stream()));
	PCG_CUDA(cudaStreamSynchronize(mem.stream()));
	mem.free(d_bad);
	mem.free(arena);
	mem.free(d_chunks);
	if (bad) throw PcgError(1, "malformed LAZ data in chunk " + std::to_string(bad - 1));
}

}  // namespace pcg
