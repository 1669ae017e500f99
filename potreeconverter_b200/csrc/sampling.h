// Sampler kernels (one octree level across all its nodes per launch).
#pragma once

#include <vector>

#include "dev.h"

namespace pcg {

struct LevelNode {          // one inner node sampled at this level
	int64_t cand_off;        // first candidate (gather order: child 0..7, index order)
	int64_t count;
	int64_t hash_off;        // first slot of the node's hash table
	int64_t hash_cap;        // power of two
	double min[3], max[3];   // node box
	double spacing;          // baseSpacing / 2^level
	int32_t level;
	int32_t pad;
};

struct GatherItem {         // copy `count` ids (and colours, records) of one child buffer
	const uint32_t* src_ids;
	const uint64_t* src_cols; // packed r | g << 16 | b << 32, or null
	const int4* src_rec;      // (X, Y, Z, -) per id, or null
	int64_t dst_off;
	int64_t count;
	int32_t child;
	int32_t node;
};
// the gather launch takes the items cut into pieces of at most this many
// ids, one CTA each, so a large child buffer does not keep one CTA busy
constexpr int64_t kGatherPiece = 4096;

struct LevelBuffers {
	int64_t M = 0;                 // candidates at this level
	int K = 0;                     // nodes at this level
	uint32_t* ids = nullptr;       // [M] candidate point ids
	uint64_t* cols = nullptr;      // [M] packed colours (poisson_average)
	uint8_t* child = nullptr;      // [M] child index
	int32_t* node_of = nullptr;    // [M] node index
	int32_t* count_in_child = nullptr; // [M] size of the candidate's child buffer (random)
	double* keys = nullptr;        // [M] FP64 squared distance to the node centre
	int32_t* perm = nullptr;       // [M] sorted position t -> local candidate index
	int32_t* pos = nullptr;        // [M] local candidate index -> sorted position
	uint8_t* accepted = nullptr;   // [M]
	int32_t* acc_rank = nullptr;   // [M] acceptance rank for accepted candidates
	int4* cq = nullptr;            // [M] sorted position -> (X, Y, Z, local index)
	int4* rec = nullptr;           // [M] candidate (gather order) -> (X, Y, Z, -), copied with the ids
};

struct SortSeg {            // a std::sort segment [f, l) with its depth budget
	int64_t f, l;
	int32_t d;
	int32_t pad;
};

struct PosParamsS {
	double scale[3], offset[3];
};

struct SampleStats {
	unsigned long long escalated;  // FP32 decisions re-made in FP64
	unsigned long long heapsorts;  // introsort depth-limit fallbacks
	unsigned long long timeouts;   // bounded loops that gave up
	unsigned long long rounds;     // CTA greedy rounds
	unsigned long long passes;     // parallel decision passes over all rounds
	unsigned long long serial;     // rounds that needed the in-order decision warp
	unsigned long long list_entries; // conflict-list entries written
	unsigned long long cluster_nodes; // nodes accepted by a CTA cluster
	unsigned long long cycles[7];  // CTA greedy: SM cycles of thread 0 in phases A, B, C1, C2, D; cells read past 3 and 7 points
};

void launch_gather(const std::vector<GatherItem>& h_items, const GatherItem* items, LevelBuffers& lb, DeviceMem& mem);
// keys from the gathered records lb.rec
void launch_keys(const LevelNode* nodes, const PosParamsS& pp, LevelBuffers& lb, DeviceMem& mem);
// records (X, Y, Z, -) of ids[0..n)
// n_src > 0: X, Y, Z hold n_src points and ids are spread over all of them
// (packed first when there are many)
void launch_gather_records(const uint32_t* ids, int64_t n, const int32_t* X, const int32_t* Y, const int32_t* Z, int4* rec, DeviceMem& mem,
                           int64_t n_src = 0);
// std::sort emulation per node; `order` lists node indices, largest first.
// Nodes order[0..num_big) (the largest) get one CTA each, the rest one warp.
// Which kernel shape samples which node of a level: nodes of at least
// cta_min candidates get a CTA each (small_level_cta_min on levels with
// fewer nodes than 2 x SMs), those of at least cluster_min a cluster of
// CTAs, the rest a warp each, pulled from a device work queue by
// warp_blocks_per_sm resident blocks per SM. The compiled-in values come from
// the autotuner's table (tuned_schedule.h, written by
// potreeconverter_b200/autotune.py); PCG_SCHEDULE="cta_min,small_level_cta_min,
// cluster_min,warp_blocks_per_sm" in the environment overrides them (read at
// every level, for the autotuner's sweep).
struct LevelSchedule {
	int64_t cta_min;
	int64_t small_level_cta_min;
	int64_t cluster_min;
	int warp_blocks_per_sm;
};
LevelSchedule level_schedule();
void launch_node_sort(const LevelNode* nodes, const int32_t* order, int K, LevelBuffers& lb, SampleStats* st, DeviceMem& mem,
                      int node_begin = 0, int node_end = -1, int num_big = 0);
// Exact ascending sort of every node's keys (segmented LSD radix sort of the
// key bits). Nodes whose keys are pairwise distinct end sorted in lb.keys,
// lb.perm and lb.pos, which is std::sort's unique result for them; nodes with
// equal keys are left as they were and flagged in tie[k] for the replay.
// Stable sort of every node's (key, value) pairs by key bits [begin_bit, end_bit) into
// (keys_out, vals_out), each node within its own range [cand_off,
// cand_off + count). vals_in == nullptr means value = index in the node.
// keys_in must not alias keys_out.
void segmented_sort_pairs(const std::vector<LevelNode>& ln, int64_t M, const uint64_t* keys_in, const uint32_t* vals_in,
                          uint64_t* keys_out, uint32_t* vals_out, int begin_bit, int end_bit, DeviceMem& mem);
// The radix-sorted keys of a level, kept for the replay of the nodes with
// equal keys. A segment of the replay whose keys are pairwise distinct ends
// in ascending order whatever its partitions do (the unique sorted order of
// its elements), so the replay writes it from here instead of partitioning
// it further: its smallest and largest element (which may equal keys
// outside the segment) at the ends, between them the sorted elements whose
// keys lie strictly between those two -- exactly the segment's other
// elements, since a partition keeps every key strictly between its pivots
// on one side.
struct SortedLevel {
	const uint64_t* sk = nullptr;     // [M] key bits, ascending within each node
	const uint32_t* sv = nullptr;     // [M] candidate index in its node
	const int32_t* ties = nullptr;    // [M] adjacent equal keys within the node up to each position (inclusive count)
	const int32_t* node_of = nullptr; // [M] node of each level position
	const LevelNode* nodes = nullptr;
	void* owned[3] = {nullptr, nullptr, nullptr};
};
// keep != nullptr: when some node has equal keys, the sorted keys stay
// allocated in *keep for the replay (release with free_sorted_level)
void sort_level_distinct(const LevelNode* d_nodes, const std::vector<LevelNode>& ln, LevelBuffers& lb, DeviceMem& mem,
                         std::vector<uint8_t>& tie, SortedLevel* keep = nullptr);
void free_sorted_level(SortedLevel& keep, DeviceMem& mem);
// the same for keys >= +0 (bit patterns) of nodes `ln`, sorted on all 64 bits
void build_sorted_level(const LevelNode* d_nodes, const std::vector<LevelNode>& ln, const int32_t* node_of, const uint64_t* keys, int64_t M,
                        SortedLevel& out, DeviceMem& mem);
// std::sort replayed on every segment [f, l) of key/val independently, each
// with depth budget d (2 * floor(log2(l - f)) for a whole node). With
// `sorted`, segments whose keys are pairwise distinct are written from it.
void replay_segments(double* key, int32_t* val, int64_t M, const std::vector<SortSeg>& segs, SampleStats* st, DeviceMem& mem,
                     const SortedLevel* sorted = nullptr);
int sort_depth_budget(int64_t n);
// lb.pos of the nodes k with pick[k] != 0, from their sorted lb.perm
void launch_node_pos(const LevelNode* nodes, const std::vector<uint8_t>& pick, LevelBuffers& lb, DeviceMem& mem);
// Earlier candidates of the same node that would reject a candidate if
// accepted (within the spacing and, for poisson, not before the early-exit
// bound), by sorted position; built for the nodes flagged in `use`.
// A list holds at most kListCap entries: the first kListInline in the
// candidate's own 16-byte slot, the rest in a pool shared by the level
// (lists average about one entry, so a fixed row per candidate would be
// mostly empty).
constexpr int kListCap = 32;
constexpr int kListInline = 4;
constexpr uint8_t kListDense = 255;
struct ConflictLists {
	int4* inl = nullptr;            // [M] first entries (node-local sorted positions)
	int32_t* ovf_off = nullptr;     // [M] where entries kListInline.. start in pool
	int32_t* pool = nullptr;        // [pool_cap] the longer lists' remaining entries
	unsigned long long* pool_used = nullptr;  // entries handed out of pool
	int64_t pool_cap = 0;
	uint8_t* count = nullptr;       // [M] by sorted position: entries, or kListDense past kListCap
	uint8_t* node_dense = nullptr;  // [K] some candidate has more than kListCap
};

// entries 4w .. 4w + 3 of the list of candidate slot `idx` (nl entries);
// positions past the list read as 0
__device__ __forceinline__ int4 list_quad(const ConflictLists& cl, int64_t idx, int nl, int w) {
	if (w == 0) return cl.inl[idx];
	const int32_t* p = cl.pool + cl.ovf_off[idx] + 4 * (w - 1);
	const int e = 4 * w;
	return make_int4(e < nl ? p[0] : 0, e + 1 < nl ? p[1] : 0, e + 2 < nl ? p[2] : 0, e + 3 < nl ? p[3] : 0);
}
void build_conflict_lists(int mode, const LevelNode* d_nodes, const std::vector<LevelNode>& ln, const std::vector<uint8_t>& use,
                          const PosParamsS& pp, LevelBuffers& lb, ConflictLists& cl, std::vector<uint8_t>& dense, SampleStats* st,
                          DeviceMem& mem);
void free_conflict_lists(ConflictLists& cl, DeviceMem& mem);
// sorted candidate records lb.cq from lb.perm
void launch_cand_records(const LevelNode* nodes, const int32_t* X, const int32_t* Y, const int32_t* Z, LevelBuffers& lb, DeviceMem& mem);
// Acceptance grids of the CTA-per-node greedy, one per resident CTA. They
// are cleared once when allocated and left empty by every node, so a job
// keeps one set for all of its levels.
struct GreedyArena {
	void* cells = nullptr;
	int32_t* ovf = nullptr;
	int slots = 0;
};
void greedy_arena_reserve(GreedyArena& a, int slots, DeviceMem& mem);
// mode 0 = poisson (early exit + 10,001-check window), 1 = poisson_average (pure greedy)
void launch_greedy(int mode, bool fp32_guard, const LevelNode* nodes, const int32_t* order, int K, const int32_t* X, const int32_t* Y,
                   const int32_t* Z, const PosParamsS& pp, LevelBuffers& lb, uint64_t* hash_keys, int32_t* hash_heads,
                   double* acc_xyz, double* acc_key, int32_t* acc_next, int32_t* acc_pos, SampleStats* st, DeviceMem& mem,
                   GreedyArena* grid, int node_begin = 0, int node_end = -1, int num_big = 0);
// acceptance from conflict lists: cta_nodes (largest first) get a cluster of
// CTAs each when they hold at least 65,536 candidates, else one CTA;
// warp_nodes a warp each
void launch_greedy_lists(int mode, const LevelNode* nodes, const std::vector<int32_t>& cta_nodes, const std::vector<int32_t>& warp_nodes,
                         const PosParamsS& pp, LevelBuffers& lb, uint64_t* hash_keys, int32_t* hash_heads, double* acc_xyz,
                         double* acc_key, int32_t* acc_next, int32_t* acc_pos, const ConflictLists& cl, SampleStats* st, DeviceMem& mem,
                         const std::vector<LevelNode>& ln);
// poisson_average colour sums: new packed colour per accepted candidate
void launch_average_colors(const LevelNode* nodes, const int32_t* X, const int32_t* Y, const int32_t* Z, const PosParamsS& pp,
                           LevelBuffers& lb, const uint64_t* hash_keys, const int32_t* hash_heads, const double* acc_xyz,
                           const int32_t* acc_next, const int32_t* acc_pos, const int64_t* acc_base, long long* sums,
                           DeviceMem& mem);
void launch_random_accept_sized(const LevelNode* nodes, const int32_t* X, const int32_t* Y, const int32_t* Z, const PosParamsS& pp,
                                LevelBuffers& lb, uint64_t* hash_keys, int32_t* hash_vals, int64_t hash_total, SampleStats* st,
                                DeviceMem& mem);
// leaf shuffle of the random sampler; leaves given as (offset, count) ranges of ids
void launch_shuffle_leaves(const int64_t* leaf_off, const int64_t* leaf_cnt, int num_leaves, const uint32_t* ids_in,
                           uint32_t* ids_out, int32_t* scratch, uint32_t seed, DeviceMem& mem);
// stand-alone entry points for the parity tests
void launch_sort_keys_single(double* keys, int32_t* vals, int64_t n, DeviceMem& mem, SampleStats* st, const SortedLevel* sorted = nullptr);
void launch_shuffle_single(int64_t n, uint32_t seed, int32_t* perm, DeviceMem& mem);

}  // namespace pcg
