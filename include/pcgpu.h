/*
 * pcgpu.h -- C ABI of the B200-native octree LOD builder (libpcgpu.so).
 *
 * The library converts LAS or LAZ file images into the three files
 * PotreeConverter 2.0 writes (octree.bin, hierarchy.bin, metadata.json),
 * byte-identical to a determinism-pinned reference build, with every stage of
 * the build running as CUDA kernels for sm_100a on one GPU.
 *
 * Reference interfaces replaced (paths relative to the PotreeConverter
 * source tree):
 *   pcg_convert      main.cpp:345-393 chunking() + indexing(), i.e.
 *                    chunker_countsort_laszip::doChunking
 *                    (include/chunker_countsort_laszip.h:19) followed by
 *                    indexer::doIndexing (include/indexer.h:379) with the
 *                    Sampler chosen by -m (main.cpp:377-392).
 *   pcg_method       the three Sampler plug-ins (include/structures.h:152-164):
 *                    SamplerPoisson, SamplerPoissonAverage, SamplerRandom.
 *   pcg_submit/poll  no counterpart: request loop for conversion jobs.
 *   pcg_kernel_*     single-kernel entry points used by the parity tests; each
 *                    names the reference code it reproduces.
 *
 * Conventions: every call returns a pcg_status (the reference calls exit()).
 * The caller owns all host memory it passes in; buffers in a pcg_result are
 * owned by the library until pcg_result_free. The context owns all device
 * memory; all device work runs on the context's stream. A context is
 * internally locked, so it may be shared between host threads.
 */
#ifndef PCGPU_H
#define PCGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pcg_status {
	PCG_OK = 0,
	PCG_BAD_INPUT = 1,    /* malformed or unsupported LAS input            */
	PCG_OUT_OF_BOX = 2,   /* point outside the header bounding box (the
	                         reference's exit(123), chunker_countsort_laszip.cpp:236-251) */
	PCG_OOM = 3,          /* device or host allocation failed             */
	PCG_TIMEOUT = 4,      /* a bounded device wait gave up                */
	PCG_INTERNAL = 5,     /* inconsistent device result                   */
	PCG_CUDA = 6,         /* CUDA runtime error                           */
	PCG_NOT_FOUND = 7     /* unknown job id                               */
} pcg_status;

typedef enum pcg_method {
	PCG_POISSON = 0,          /* sampler_poisson.h        */
	PCG_POISSON_AVERAGE = 1,  /* sampler_poisson_average.h */
	PCG_RANDOM = 2            /* sampler_random.h          */
} pcg_method;

typedef enum pcg_form {
	PCG_FORM_BATCHED = 0, /* one launch per octree level over all nodes, FP32
	                         neighbour tests with an FP64 guard band          */
	PCG_FORM_PLAIN = 1    /* one launch per node, every neighbour test FP64  */
} pcg_form;

/* Where the point records of a conversion in parts live (pcg_opts.records). */
typedef enum pcg_records {
	PCG_RECORDS_AUTO = 0,      /* resident on the device when they fit beside
	                              one part's working set, else streamed      */
	PCG_RECORDS_RESIDENT = 1,  /* copied to the device once (the first pass)  */
	PCG_RECORDS_STREAMED = 2   /* streamed from host memory again for every
	                              part                                        */
} pcg_records;

typedef struct pcg_opts {
	int32_t device;        /* CUDA device ordinal                            */
	uint32_t random_seed;  /* seed of the random sampler's leaf shuffle; the
	                          pinned reference uses 1592614637               */
	int32_t form;          /* pcg_form                                        */
	int32_t records;       /* pcg_records: record placement of conversions in
	                          parts                                           */
	void* stream;          /* cudaStream_t for all device work, or NULL for a
	                          stream owned by the context                     */
	/* Conversion in parts (clouds beyond the device's working set, the
	   reference's out-of-core chunking + indexing, chunker_countsort_laszip.
	   cpp:1206-1261, indexer.cpp:181-281): a job of one uncompressed LAS
	   source with more points than group_points is indexed in parts of
	   consecutive chunks of at most group_points points (a chunk larger than
	   that is a part by itself). 0 = parts only when the whole cloud would
	   not fit the device, sized from its free memory and at most 100M
	   points each. */
	int64_t group_points;
} pcg_opts;

enum {
	PCG_JOB_OCTREE_ON_DEVICE = 1  /* leave octree.bin in device memory:
	                                 pcg_result.octree is then a device pointer */
};

/* One input file of a job with several sources (the reference's source
   list after curateSources, main.cpp:146-200). */
typedef struct pcg_source {
	const void* las;       /* LAS or LAZ file image (host memory); with
	                          device_records set, only its header and VLRs
	                          are read                                        */
	uint64_t las_size;
	const void* device_records; /* its point records in device memory, or NULL */
} pcg_source;

typedef struct pcg_job {
	const void* las;       /* LAS or LAZ file image (host memory); with
	                          device_records set, only its header and VLRs
	                          are read                                        */
	uint64_t las_size;
	int32_t method;        /* pcg_method                                      */
	int32_t flags;         /* PCG_JOB_* bits                                  */
	const char* name;      /* metadata.json "name" (the reference uses the
	                          first input's stem, main.cpp:171-173)           */
	const char* projection;/* metadata.json "projection" (may be NULL)       */
	const void* device_records; /* point records already in device memory
	                          (record_length * point count bytes), or NULL    */
	/* Several input files converted as one point cloud
	   (computeOutputAttributes(sources, ...), PotreeConverter.h:195-276, and
	   doChunking(sources, ...), chunker_countsort_laszip.cpp:1206): with
	   num_sources > 0, sources[0 .. num_sources) are the input, in this
	   order, and las / las_size / device_records are ignored.             */
	int32_t num_sources;
	/* --attributes (main.cpp:108): keep "position" and these attributes, in
	   this order (names not found are skipped); 0 keeps every attribute.  */
	int32_t num_attributes;
	const pcg_source* sources;
	const char* const* attributes;
} pcg_job;

typedef struct pcg_stats {
	int64_t num_points;           /* points in the LAS file                 */
	int64_t num_chunks;
	int64_t num_nodes;            /* hierarchy records written              */
	int64_t output_points;
	int64_t octree_depth;
	int64_t escalated_pairs;      /* FP32 tests re-decided in FP64          */
	int64_t heapsort_fallbacks;   /* introsort depth-limit hits             */
	double ms_total;              /* wall time of pcg_convert               */
	double ms_h2d, ms_chunking, ms_octree, ms_sampling, ms_output, ms_d2h, ms_host_writers;
	int64_t gpu_launches;         /* kernels launched for this job          */
	double ms_sort, ms_greedy;    /* device time of the sampler sort / acceptance kernels */
	int64_t sampled_nodes;        /* inner nodes sampled                    */
	int64_t candidates;           /* candidate points over all sampled nodes */
	int64_t replayed_nodes;       /* nodes with equal keys, sorted by the
	                                 element-for-element introsort replay   */
	int64_t replayed_candidates;  /* their candidates                       */
	double ms_lists;              /* device time of the conflict-list builds
	                                 (part of ms_greedy)                     */
	int64_t list_entries;         /* conflict-list entries over all levels  */
	int64_t cluster_nodes;        /* nodes accepted by a cluster of CTAs    */
	double ms_decode;             /* LAZ decode of the job's .laz sources   */
	int64_t laz_chunks;           /* LASzip chunks decoded                  */
	int64_t device_peak_bytes;    /* high-water mark of the job's device
	                                 allocations                            */
	int64_t parts;                /* parts of a conversion in parts, else 0 */
	int64_t survivors;            /* chunk-root points carried from the
	                                 parts to the levels above them          */
	int64_t records_resident;     /* 1: the records stayed on the device
	                                 between the passes of a conversion in
	                                 parts                                   */
	int64_t device_estimate_bytes; /* the request loop's admission estimate
	                                 of this job's device memory (a job in
	                                 one piece)                              */
} pcg_stats;

/* One completed node: what the reference's hierarchy flusher records for it
   (indexer.h:146-162, Writer::writeAndUnload indexer.cpp:1453-1516). */
typedef struct pcg_node {
	const char* name;      /* "r" + child digits, NUL terminated (owned by the result) */
	int64_t num_points;
	uint64_t byte_offset;  /* of its payload in octree.bin; 0 without points */
	uint64_t byte_size;
} pcg_node;

/* One piece of octree.bin: the file is its pieces back to back. */
typedef struct pcg_octree_part {
	const uint8_t* data;   /* host memory (owned by the result)             */
	uint64_t size;
} pcg_octree_part;

typedef struct pcg_result {
	uint8_t* octree;       uint64_t octree_size;     /* host memory unless the
	                                                    job asked for device;
	                                                    NULL for a conversion
	                                                    in parts, whose
	                                                    octree.bin is
	                                                    octree_parts[] (size
	                                                    still the total)     */
	uint8_t* hierarchy;    uint64_t hierarchy_size;
	char* metadata;        uint64_t metadata_size;   /* NUL terminated */
	pcg_stats stats;
	pcg_node* nodes;       /* every node in completion order (the order of
	                          the payloads in octree.bin); NULL if the host had
	                          no memory for the list */
	uint64_t num_nodes;
	pcg_octree_part* octree_parts; /* octree.bin in pieces, in file order: one
	                          piece (octree itself) for a conversion in one
	                          piece, one per part plus one for the levels
	                          above the parts otherwise                      */
	uint64_t num_octree_parts;
} pcg_result;

typedef struct pcg_ctx pcg_ctx;

/* Context lifecycle. opts may be NULL (device 0, pinned seed, batched). */
pcg_status pcg_create(pcg_ctx** ctx, const pcg_opts* opts);
void pcg_destroy(pcg_ctx* ctx);
const char* pcg_last_error(const pcg_ctx* ctx);
const char* pcg_status_string(pcg_status s);

/* Synchronous conversion (replaces chunking() + indexing(), main.cpp:345-393). */
pcg_status pcg_convert(pcg_ctx* ctx, const pcg_job* job, pcg_result* out);
void pcg_result_free(pcg_result* r);

/* Writes out->{octree,hierarchy,metadata} as <dir>/octree.bin etc. */
pcg_status pcg_write_files(const pcg_result* r, const char* dir);

/* Request loop: jobs are admitted by device-memory footprint and run as
 * device work interleaves; pcg_wait blocks until the job finished. */
pcg_status pcg_submit(pcg_ctx* ctx, const pcg_job* job, uint64_t* job_id);
pcg_status pcg_poll(pcg_ctx* ctx, uint64_t job_id, int32_t* done);
pcg_status pcg_wait(pcg_ctx* ctx, uint64_t job_id, pcg_result* out);

/* ---- single-kernel entry points (device-agnostic host buffers) ---------- */

/* Sorts n keys ascending with the exact element order std::sort (libstdc++
 * introsort: median-of-3 pivot, threshold 16, heapsort at the depth limit)
 * produces for the comparator "a < b" -- the sort the samplers call
 * (sampler_poisson.h:183-203). perm_out[i] = input index of the i-th element. */
pcg_status pcg_kernel_sort_keys(pcg_ctx* ctx, const double* keys, int64_t n, int32_t* perm_out);

/* perm_out[i] = index that std::shuffle(0..n-1, std::default_random_engine(seed))
 * leaves at position i (sampler_random.h:97-104). */
pcg_status pcg_kernel_shuffle(pcg_ctx* ctx, int64_t n, uint32_t seed, int32_t* perm_out);

/* The counting pass of one LAS or LAZ file image (countPointsInCells,
   chunker_countsort_laszip.cpp:131-361, with the decode and quantization of
   :749-803): every point's quantized X, Y, Z and count-grid cell
   (ix + iy G + iz G^2; X, Y, Z, cell hold the point count), and the grid of
   G^3 counts, G (128, 256 or 512 by point count, chunker :1214-1220)
   returned in *grid_size. X, Y, Z and cell hold point_capacity elements; a
   file with more points (by its header) is refused with PCG_BAD_INPUT
   before anything is written. Points outside the header box:
   PCG_OUT_OF_BOX. */
pcg_status pcg_kernel_decode_count(pcg_ctx* ctx, const void* las, uint64_t size, int32_t* X, int32_t* Y, int32_t* Z, uint32_t* cell,
                                   int64_t point_capacity, uint32_t* grid, int64_t grid_capacity, int32_t* grid_size);

/* One chunk of the chunker's LUT (createLUT, chunker_countsort_laszip.cpp:
   1074-1204): its file name without ".bin" (toNodeID, :82-115: "r" + one
   octant digit per level), its cell at its own level and its point count. */
typedef struct pcg_chunk {
	char id[16];
	int32_t level, x, y, z;
	int64_t count;
} pcg_chunk;

/* The LUT merge (createLUT, chunker_countsort_laszip.cpp:1074-1204) of a
   count grid of G^3 cells (G a power of two up to 512, cell index ix + iy G +
   iz G^2): 2x2x2 blocks merge bottom-up while no child is split and the sum
   stays <= max_points_per_chunk. chunks_out receives the chunks in chunk
   file-name order (the order the indexer visits them, indexer.cpp:149 with
   sorted directory iteration), lut_out (G^3 entries) every cell's index in
   that list, -1 for cells no chunk covers. More chunks than chunk_capacity:
   PCG_BAD_INPUT, with *num_chunks set to the count needed. */
pcg_status pcg_kernel_lut(pcg_ctx* ctx, const uint32_t* grid, int32_t grid_size, int64_t max_points_per_chunk, int32_t* lut_out,
                          pcg_chunk* chunks_out, int64_t chunk_capacity, int32_t* num_chunks);

/* The distribution of points to chunks (distributePoints,
   chunker_countsort_laszip.cpp:837-904, with one chunker thread): ids_out
   lists the point indices 0..n-1 grouped by chunk (chunk 0 first), input
   order inside each chunk, and chunk_start[k] (num_chunks + 1 entries) is
   where chunk k starts in ids_out. cell: every point's count-grid cell
   (pcg_kernel_decode_count), lut: G^3 entries (pcg_kernel_lut). A cell no
   chunk covers: PCG_INTERNAL. */
pcg_status pcg_kernel_scatter(pcg_ctx* ctx, const uint32_t* cell, int64_t n, const int32_t* lut, int32_t grid_size, int32_t num_chunks,
                              uint32_t* ids_out, int64_t* chunk_start);

/* One node of a chunk's octree (buildHierarchy, indexer.cpp:823-1109). */
typedef struct pcg_octree_node {
	char name[32];         /* root_name + octant digits                       */
	int64_t start;         /* its points: order_out[start .. start + count)    */
	int64_t count;         /* 0 for inner nodes                                */
	int32_t is_leaf;
	int32_t pad;
} pcg_octree_node;

/* The per-chunk octree of one chunk (buildHierarchy, indexer.cpp:823-1109:
   32^3 counting sort in Morton order, sum pyramid, createNodes :732-817 with
   the 10,000-point split threshold, recursion into over-full nodes and the
   duplicate rule of :1002-1099). X, Y, Z: the chunk's quantized points (n,
   in chunk order); scale / offset: the output position transform
   (x = X * scale + offset); box_min / box_max: the chunk's cube;
   root_name: the chunk's id. order_out (n entries) receives the points'
   indices in the order the reference leaves them, nodes_out every node of
   the chunk's subtree below and including the root, sorted by name;
   *octree_depth the deepest level created (the reference's octreeDepth).
   More nodes than node_capacity: PCG_BAD_INPUT, *num_nodes = count needed. */
pcg_status pcg_kernel_octree(pcg_ctx* ctx, const int32_t* X, const int32_t* Y, const int32_t* Z, int64_t n, const double* scale,
                             const double* offset, const double* box_min, const double* box_max, const char* root_name,
                             uint32_t* order_out, pcg_octree_node* nodes_out, int64_t node_capacity, int64_t* num_nodes,
                             int64_t* octree_depth);

/* The sampler's decision for one inner node (method = pcg_method):
   SamplerPoisson (sampler_poisson.h:127-203: std::sort by squared distance
   to the node centre, greedy acceptance with the early-exit bound and the
   10,001-check cap), SamplerPoissonAverage (sampler_poisson_average.h:
   184-445: pure greedy in a 16^3 grid window, order-dependent colour sums)
   or SamplerRandom (sampler_random.h:123-182: children under 100 points, or
   the first point of a 128^3 cell within 0.7 sqrt(3) of its centre; a fresh
   cell grid, as for the first node a thread samples). The candidates are the
   children's points in gather order: child[] (n entries) is non-decreasing
   in 0..7, X, Y, Z are quantized positions, rgb (3 x uint16 per point) the
   colours (poisson_average only, else may be NULL). box_min / box_max: the
   node's cube, spacing: the node's spacing (baseSpacing / 2^level).
   accepted_out[i] = 1 when candidate i moves to the parent; for
   poisson_average rgb_out (3 x n, may be NULL otherwise) receives the
   averaged colour written into every candidate (:440-445). */
pcg_status pcg_kernel_accept(pcg_ctx* ctx, int32_t method, const int32_t* X, const int32_t* Y, const int32_t* Z, const uint8_t* child,
                             const uint16_t* rgb, int64_t n, const double* scale, const double* offset, const double* box_min,
                             const double* box_max, double spacing, uint8_t* accepted_out, uint16_t* rgb_out);

/* LASzip decode of every point of a LAZ file image (point formats 0-3,
   LASzip's chunked point-wise coding: lasreadpoint.cpp:405-497 with the v2
   item readers of lasreaditemcompressed_v2.cpp) into records_out
   (point count x record length bytes), exactly the records the reference
   reads through laszip_read_point. */
pcg_status pcg_kernel_laz_decode(pcg_ctx* ctx, const void* laz_file, uint64_t size, void* records_out, uint64_t out_size);

/* ---- the same sort for callers that cannot allocate ---------------------
 * No counterpart in the reference. pcg_kernel_sort_keys_noalloc is
 * pcg_kernel_sort_keys for code that must not allocate device memory, e.g. a
 * plugin inside a host framework that owns every device allocation and
 * hands its plugins only the buffers it made (a cudaMalloc of the plugin's
 * own would bypass that framework's memory accounting and can fail once the
 * framework has reserved the device). Keys (n doubles) and the output
 * permutation (n int32) are device buffers the caller provides; all scratch
 * lives in a static device array of 28 * PCG_NOALLOC_SORT_MAX + 256 bytes
 * that every GPU loading the library holds until the process exits. No
 * cudaMalloc/cudaFree is called.
 *  - n > PCG_NOALLOC_SORT_MAX returns PCG_BAD_INPUT and does nothing;
 *  - the first call on a device looks up the array's device address (set-up
 *    per device). The address is kept for the life of the process: do not
 *    call this entry point again on a device after cudaDeviceReset;
 *  - work runs on `stream` (a cudaStream_t, NULL = legacy default) and the
 *    call waits for it to finish (it reads back a small error word), so it
 *    cannot be part of a stream capture;
 *  - a CUDA error left pending by earlier work is reported as PCG_CUDA
 *    before anything is launched, and left pending for the caller;
 *  - all calls share the one array: calls that overlap on the GPU (other
 *    streams or host threads) race and must be serialized by the caller. */
#define PCG_NOALLOC_SORT_MAX 262144
pcg_status pcg_kernel_sort_keys_noalloc(const double* d_keys, int64_t n, int32_t* d_perm, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PCGPU_H */
