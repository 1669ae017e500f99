// Host-callable launchers of the pipeline kernels (one per CUDA unit).
#pragma once

#include "dev.h"

namespace pcg {

// ------------------------------------------------------------- chunking.cu
struct ChunkCell {      // one chunk found by the LUT merge
	int32_t level, x, y, z;
	int64_t count;
};

struct ChunkingOut {
	int32_t* X; int32_t* Y; int32_t* Z;     // quantized positions, input order
	uint32_t* cell;                          // count-grid cell per point
	AttrStatsDev* stats;                     // per attribute
	unsigned long long* histogram;           // 256 bins (classification)
	int64_t* error;                          // [0] = first failing point + 1 (out of box), [1] = lookup failure
};

// ------------------------------------------------------------------ laz.cu
// Decodes the LASzip chunks of one LAZ source into its point records
// (chunks' byte offsets are file offsets; d_bytes holds the file from
// `base` to the end of the last chunk). Throws on malformed data.
void launch_laz_decode(const uint8_t* d_bytes, uint64_t base, const std::vector<laz::Chunk>& chunks, const laz::Layout& L, uint8_t* d_out,
                       DeviceMem& mem);

// Decodes the records of every source (DecodeParams::src0 / srcs).
void launch_decode_count(const DecodeParams& p, uint32_t* grid, ChunkingOut& out, DeviceMem& mem);
// Pyramid merge of the count grid (createLUT, chunker_countsort_laszip.cpp:1074-1204).
void launch_lut_merge(const uint32_t* grid, int grid_size, int64_t max_points_per_chunk, ChunkCell* chunks,
                      int32_t* num_chunks, int capacity, DeviceMem& mem);
// Fills the LUT: chunk k owns cells of chunks[k] (already in chunk order).
void launch_lut_fill(const ChunkCell* chunks, int num_chunks, int grid_size, int32_t* lut, DeviceMem& mem);
// chunk_of[i] = lut[cell[i]] - chunk_base, ids[i] = i; a cell without a
// chunk, or one below chunk_base, sets error[1]
void launch_assign_chunks(const uint32_t* cell, const int32_t* lut, int64_t n, int chunk_base, uint32_t* chunk_of, uint32_t* ids,
                          int64_t* error, DeviceMem& mem);
// Appends the records among recs[0..n) (one source, p.src0's layout) whose
// count-grid cell lies in chunks k0 .. k1 - 1 to out, in input order, at
// record index *fill onwards; *fill (device) advances by their count.
void launch_select_part(const DecodeParams& p, const uint8_t* recs, int64_t n, const int32_t* lut, int k0, int k1, int64_t* fill,
                        uint8_t* out, DeviceMem& mem);
// out_recs[i] = recs[ids[i]] (rec_len bytes each), oX/oY/oZ[i] = X/Y/Z[ids[i]]
void launch_gather_points(const uint32_t* ids, int64_t n, const uint8_t* recs, int rec_len, const int32_t* X, const int32_t* Y,
                          const int32_t* Z, uint8_t* out_recs, int32_t* oX, int32_t* oY, int32_t* oZ, DeviceMem& mem);
// out[i] = i, i < n
void launch_iota(uint32_t* out, int64_t n, DeviceMem& mem);
// starts[k] = first index of key k in ascending keys[0..n), k = 0..num_keys
// (starts[num_keys] = n; keys < num_keys)
void launch_segment_starts(const uint32_t* keys, int64_t n, int num_keys, int64_t* starts, DeviceMem& mem);

// --------------------------------------------------------------- octree.cu
struct SegmentDesc {        // one node to split with a 32^3 counting sort
	int64_t start;           // range in the working id array
	int64_t count;
	int64_t coff;            // offset in the compacted round array
	double min[3], size[3];  // node box (min, max - min)
};

struct NodeCand {           // createNodes output (indexer.cpp:732-817)
	int32_t seg;
	int32_t level;           // 0..5 below the segment node
	int32_t path;            // 3 bits per level, first level in the high bits
	int32_t pad;
	int64_t start;           // relative to the segment start
	int64_t count;
};

struct PosParams {
	double scale[3], offset[3];
};

void launch_octree_round(uint32_t* ids, const int32_t* X, const int32_t* Y, const int32_t* Z, const PosParams& pp,
                         const SegmentDesc* d_segs, int num_segs, int64_t total, NodeCand* cands, int32_t* num_cands,
                         int64_t cand_capacity, DeviceMem& mem);
// number of distinct (X, Y, Z) among ids[0..n)
int64_t count_unique_positions(const uint32_t* ids, int64_t n, const int32_t* X, const int32_t* Y, const int32_t* Z, DeviceMem& mem);

}  // namespace pcg
