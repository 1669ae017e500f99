// Host orchestration of one conversion job and the C ABI (include/pcgpu.h).
//
// Stage map (reference files relative to the PotreeConverter source tree):
//   decode + count grid   chunking.cu   chunker_countsort_laszip.cpp:131-361, 749-803
//   LUT merge             chunking.cu   chunker_countsort_laszip.cpp:1074-1204
//   stable scatter        radix.cu      chunker_countsort_laszip.cpp:837-904
//   per-chunk octree      octree.cu     indexer.cpp:691-1109
//   samplers              sampling.cu   sampler_poisson.h, sampler_poisson_average.h, sampler_random.h
//   completion order      here          indexer.cpp:1581-1745 (chunks, chunk-root tasks, root)
//   octree.bin            output.cu     indexer.cpp:1453-1516
//   hierarchy/metadata    writers.cpp   indexer.h:120-244, HierarchyBuilder.h, indexer.cpp:354-524
//
// The reference hands chunks to the indexer through files; here every
// intermediate stays in device memory and only point ids move between
// stages. Sampling runs level by level (deepest first) over all nodes of the
// level at once; the reference's node completion order, which fixes the
// octree.bin layout, is recomputed on the host from the final tree.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <unistd.h>

#include "../../include/pcgpu.h"
#include "kernels.h"
#include "output.h"
#include "sampling.h"
#include "writers.h"

namespace pcg {

namespace {

using Clock = std::chrono::steady_clock;
double ms_since(Clock::time_point t) { return std::chrono::duration<double, std::milli>(Clock::now() - t).count(); }

// error word of the counting pass: the first point outside the header's
// box (index + 1), or -1 when a record copy into shared memory did not
// complete within its bounded wait
void check_counting_pass(int64_t e) {
	if (e < 0) throw PcgError(PCG_TIMEOUT, "a record copy of the counting pass did not complete");
	if (e > 0) throw PcgError(PCG_OUT_OF_BOX, "point " + std::to_string(e - 1) + " lies outside the header bounding box");
}

constexpr int64_t kMaxNodePoints = 10'000;          // indexer.h:47
constexpr int kChunkRootMergeThreshold = 5'000'000; // indexer.cpp:241

struct TNode {
	std::string name;
	int parent = -1;
	int child[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
	Vec3d min, max;
	int depth = 0;
	int chunk = -1;             // chunk whose subtree holds the node; -1 above chunk roots
	bool chunk_root = false;
	// leaf payload from the octree build: range of the working id array
	int64_t leaf_start = 0, leaf_count = 0;
	// current buffer (what the parent's sampler sees)
	const uint32_t* buf_ids = nullptr;
	const uint64_t* buf_cols = nullptr;
	const int4* buf_rec = nullptr;   // (X, Y, Z, -) per buffered id (poisson samplers)
	int64_t buf_count = 0;
	// state after the parent's sampling
	const uint32_t* fin_ids = nullptr;
	const uint64_t* fin_cols = nullptr;
	int64_t fin_count = 0;
	bool completed = false;     // gets a hierarchy record
	bool unlinked = false;      // removed from the parent's child list
	bool has_children() const {
		for (int c : child) if (c >= 0) return true;
		return false;
	}
};

struct Tree {
	std::vector<TNode> nodes;
	int add(const std::string& name, int parent, const Vec3d& mn, const Vec3d& mx) {
		TNode n;
		n.name = name;
		n.parent = parent;
		n.min = mn;
		n.max = mx;
		n.depth = (int)name.size() - 1;
		nodes.push_back(n);
		return (int)nodes.size() - 1;
	}
	int child_of(int p, int idx, int chunk) {
		if (nodes[p].child[idx] >= 0) return nodes[p].child[idx];
		Vec3d mn, mx;
		child_box(nodes[p].min, nodes[p].max, idx, mn, mx);
		int c = add(nodes[p].name + char('0' + idx), p, mn, mx);
		nodes[c].chunk = chunk;
		nodes[p].child[idx] = c;
		return c;
	}
};

// toNodeID(level, gridSize, x, y, z), chunker_countsort_laszip.cpp:82-115,
// called with the grid size of the chunk's own level (:1162)
std::string chunk_id(const ChunkCell& c) {
	std::string id = "r";
	int cur = 1 << c.level;
	int lx = c.x, ly = c.y, lz = c.z;
	for (int i = 0; i < c.level; i++) {
		int index = 0;
		if (lx >= cur / 2) { index += 4; lx -= cur / 2; }
		if (ly >= cur / 2) { index += 2; ly -= cur / 2; }
		if (lz >= cur / 2) { index += 1; lz -= cur / 2; }
		id += char('0' + index);
		cur /= 2;
	}
	return id;
}

double decode_ordered(unsigned long long k) {
	unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
	double d;
	memcpy(&d, &b, 8);
	return d;
}

template <class T>
T* upload(const std::vector<T>& v, DeviceMem& mem) {
	T* d = mem.alloc<T>(v.size() ? v.size() : 1);
	if (!v.empty()) PCG_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, mem.stream()));
	return d;
}

template <class T>
std::vector<T> download(const T* d, size_t n, cudaStream_t s) {
	std::vector<T> v(n);
	if (n) PCG_CUDA(cudaMemcpyAsync(v.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
	PCG_CUDA(cudaStreamSynchronize(s));
	return v;
}

// Pinned host buffers for octree.bin images, recycled between jobs so the
// device-to-host copy runs at link speed instead of paying for page locking
// every time. Buffers handed out in a pcg_result come back in pcg_result_free.
class PinnedPool {
public:
	uint8_t* take(size_t n) {
		std::lock_guard<std::mutex> lk(m_);
		if (n == 0) n = 1;
		auto it = free_.lower_bound(n);
		if (it != free_.end() && it->first <= 2 * n + (size_t(64) << 20)) {
			void* p = it->second;
			cached_ -= it->first;
			in_use_ += it->first;
			free_.erase(it);
			age_.erase(p);
			return static_cast<uint8_t*>(p);
		}
		// a new buffer first frees cached ones (longest unused first) while
		// cached plus handed-out memory would pass half the host's memory
		while (!free_.empty() && cached_ + in_use_ + n > max_total()) drop_oldest();
		void* p = nullptr;
		if (cudaMallocHost(&p, n) != cudaSuccess) {
			cudaGetLastError();
			return nullptr;
		}
		owned_[p] = n;
		in_use_ += n;
		return static_cast<uint8_t*>(p);
	}
	bool give(void* p) {
		std::lock_guard<std::mutex> lk(m_);
		auto it = owned_.find(p);
		if (it == owned_.end()) return false;
		free_.insert({it->second, p});
		age_[p] = ++clock_;
		cached_ += it->second;
		in_use_ -= it->second;
		while (cached_ > max_cached() && !free_.empty()) drop_oldest();
		return true;
	}

private:
	// frees the cached buffer given back longest ago; returns its size
	size_t drop_oldest() {
		void* old = nullptr;
		uint64_t oldest = UINT64_MAX;
		for (const auto& a : age_)
			if (a.second < oldest) { oldest = a.second; old = a.first; }
		if (!old) return 0;
		const size_t sz = owned_[old];
		for (auto f = free_.lower_bound(sz); f != free_.end() && f->first == sz; ++f)
			if (f->second == old) { free_.erase(f); break; }
		age_.erase(old);
		cached_ -= sz;
		owned_.erase(old);
		cudaFreeHost(old);
		return sz;
	}
	static size_t phys() {
		const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGE_SIZE);
		return pages > 0 && page > 0 ? (size_t)pages * (size_t)page : (size_t(32) << 30);
	}
	// pinned memory kept for reuse: a third of the host's memory, at most
	// 64 GiB (the pieces of a large conversion are reused by the next one)
	static size_t max_cached() {
		static const size_t m = std::max(size_t(8) << 30, std::min(size_t(64) << 30, phys() / 3));
		return m;
	}
	// cached plus handed-out pinned memory before new buffers free cached ones
	static size_t max_total() {
		static const size_t m = std::max(size_t(8) << 30, phys() / 2);
		return m;
	}
	std::mutex m_;
	std::multimap<size_t, void*> free_;
	std::unordered_map<void*, size_t> owned_;
	std::unordered_map<void*, uint64_t> age_;  // cached buffer -> when it was given back
	uint64_t clock_ = 0;
	size_t cached_ = 0, in_use_ = 0;
};

PinnedPool g_pinned;

// octree.bin images left in device memory (PCG_JOB_OCTREE_ON_DEVICE)
std::mutex g_dev_mtx;
std::unordered_map<void*, int> g_dev_results;  // pointer -> device

void release_octree(void* p) {
	if (!p) return;
	int dev = -1;
	{
		std::lock_guard<std::mutex> lk(g_dev_mtx);
		auto it = g_dev_results.find(p);
		if (it != g_dev_results.end()) { dev = it->second; g_dev_results.erase(it); }
	}
	if (dev >= 0) {
		int cur = 0;
		cudaGetDevice(&cur);
		cudaSetDevice(dev);
		cudaFree(p);
		cudaSetDevice(cur);
	} else if (!g_pinned.give(p)) {
		cudaFreeHost(p);
	}
}

struct JobResult {
	std::vector<uint8_t> hierarchy;
	std::string metadata;
	uint8_t* octree = nullptr;  // pinned host memory, or device memory
	uint64_t octree_size = 0;
	bool octree_on_device = false;
	// a conversion in parts: octree.bin in pieces (pinned host memory, from
	// g_pinned), octree stays null
	std::vector<std::pair<uint8_t*, uint64_t>> parts;
	pcg_stats stats{};
	std::vector<HierRecord> nodes;  // completion order
	void release_parts() {
		for (auto& pt : parts)
			if (pt.first && !g_pinned.give(pt.first)) cudaFreeHost(pt.first);
		parts.clear();
	}
};

// Streams the records of one host source to the device in tiles of
// `tile_points` points on a side stream, ahead of the kernels that read
// them on the compute stream. Page-locked source memory is copied directly;
// other memory goes through two pinned staging buffers that host threads
// fill. With `resident` set, tile t lands in resident + t * tile bytes (the
// records stay on the device); else in one of two device buffers that
// alternate between tiles.
class TileFeeder {
public:
	TileFeeder(const uint8_t* host, int64_t n, int rec_len, int64_t tile_points, cudaStream_t compute, uint8_t* resident, DeviceMem& mem)
	    : host_(host), n_(n), rec_(rec_len), tile_(tile_points), compute_(compute), resident_(resident) {
		tiles_ = n == 0 ? 0 : (n + tile_ - 1) / tile_;
		cudaPointerAttributes a{};
		pinned_ = cudaPointerGetAttributes(&a, host) == cudaSuccess && a.type == cudaMemoryTypeHost;
		cudaGetLastError();
		PCG_CUDA(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
		const size_t tile_bytes = (size_t)tile_ * rec_;
		for (int b = 0; b < 2; b++) {
			PCG_CUDA(cudaEventCreateWithFlags(&copied_[b], cudaEventDisableTiming));
			PCG_CUDA(cudaEventCreateWithFlags(&consumed_[b], cudaEventDisableTiming));
			PCG_CUDA(cudaEventCreateWithFlags(&staged_[b], cudaEventDisableTiming));
			if (!resident_ && tiles_ > 0) dev_[b] = mem.alloc<uint8_t>(tile_bytes);
			if (!pinned_ && tiles_ > 0) {
				stage_[b] = g_pinned.take(tile_bytes);
				if (!stage_[b]) throw PcgError(PCG_OOM, "no pinned staging memory");
			}
		}
	}
	~TileFeeder() {
		cudaStreamSynchronize(copy_);
		for (int b = 0; b < 2; b++) {
			cudaEventDestroy(copied_[b]);
			cudaEventDestroy(consumed_[b]);
			cudaEventDestroy(staged_[b]);
			if (stage_[b]) g_pinned.give(stage_[b]);
		}
		cudaStreamDestroy(copy_);
	}
	int64_t tiles() const { return tiles_; }
	int64_t tile_points() const { return tile_; }
	// Device records of tile t (points first .. first + count); the compute
	// stream waits for their copy. Tiles are taken in order.
	const uint8_t* acquire(int64_t t, int64_t& first, int64_t& count) {
		if (issued_ <= t) issue(t);
		first = t * tile_;
		count = std::min<int64_t>(tile_, n_ - first);
		PCG_CUDA(cudaStreamWaitEvent(compute_, copied_[t & 1], 0));
		return buffer(t);
	}
	// The compute stream's work on tile t is enqueued: its buffer may be
	// refilled once that work is done; the copy of tile t + 1 starts.
	void release(int64_t t) {
		PCG_CUDA(cudaEventRecord(consumed_[t & 1], compute_));
		if (t + 1 < tiles_ && issued_ <= t + 1) issue(t + 1);
	}

private:
	uint8_t* buffer(int64_t t) const { return resident_ ? resident_ + (size_t)t * tile_ * rec_ : dev_[t & 1]; }
	void issue(int64_t t) {
		const int b = (int)(t & 1);
		const int64_t first = t * tile_;
		const size_t bytes = (size_t)std::min<int64_t>(tile_, n_ - first) * rec_;
		const uint8_t* src = host_ + (size_t)first * rec_;
		if (!resident_ && t >= 2) PCG_CUDA(cudaStreamWaitEvent(copy_, consumed_[b], 0));
		if (!pinned_) {
			// the staging buffer's previous copy must have left it
			if (t >= 2) PCG_CUDA(cudaEventSynchronize(staged_[b]));
			parallel_copy(stage_[b], src, bytes);
			src = stage_[b];
		}
		PCG_CUDA(cudaMemcpyAsync(buffer(t), src, bytes, cudaMemcpyHostToDevice, copy_));
		if (!pinned_) PCG_CUDA(cudaEventRecord(staged_[b], copy_));
		PCG_CUDA(cudaEventRecord(copied_[b], copy_));
		issued_ = t + 1;
	}
	static void parallel_copy(uint8_t* dst, const uint8_t* src, size_t bytes) {
		const int nt = (int)std::min<size_t>(8, std::max<size_t>(1, bytes >> 26));
		if (nt == 1) {
			std::memcpy(dst, src, bytes);
			return;
		}
		std::vector<std::thread> th;
		const size_t per = (bytes + nt - 1) / nt;
		for (int k = 0; k < nt; k++) {
			const size_t o = k * per;
			if (o >= bytes) break;
			th.emplace_back([=] { std::memcpy(dst + o, src + o, std::min(per, bytes - o)); });
		}
		for (auto& x : th) x.join();
	}

	const uint8_t* host_;
	int64_t n_;
	int rec_;
	int64_t tile_, tiles_ = 0, issued_ = 0;
	cudaStream_t compute_, copy_ = nullptr;
	uint8_t* resident_;
	bool pinned_ = false;
	uint8_t* dev_[2] = {nullptr, nullptr};
	uint8_t* stage_[2] = {nullptr, nullptr};
	cudaEvent_t copied_[2], consumed_[2], staged_[2];
};

// PCG_TRACE_LEVELS=1 prints one line per sampled octree level to stderr
static bool trace_levels() {
	static const bool on = [] {
		const char* e = std::getenv("PCG_TRACE_LEVELS");
		return e && e[0] == '1';
	}();
	return on;
}

// The completion order of the single-threaded reference (doIndexing,
// indexer.cpp:1639-1745), built in two steps so a conversion in parts can
// place each part's nodes as soon as the part is sampled: chunk(cr) appends
// the nodes completed while chunk cr is sampled (post-order, :1639-1671);
// finish() appends the merged chunk-root tasks (processChunkRoots, :202-281)
// in pre-order and then the root.
struct CompletionOrder {
	Tree& tree;
	int method;
	std::vector<int> order;
	std::vector<char> sampled, cleared;  // cleared: children.clear() was called

	CompletionOrder(Tree& t, int m) : tree(t), method(m) {}

	void grow() {
		if (sampled.size() < tree.nodes.size()) {
			sampled.resize(tree.nodes.size(), 0);
			cleared.resize(tree.nodes.size(), 0);
		}
	}
	void complete_children(int ni) {
		const TNode& n = tree.nodes[ni];
		for (int c = 0; c < 8; c++) {
			int ci = n.child[c];
			if (ci < 0) continue;
			const TNode& ch = tree.nodes[ci];
			if (method == PCG_POISSON_AVERAGE && ch.unlinked) continue;
			order.push_back(ci);
		}
	}
	void post(int ni) {
		if (!cleared[ni]) {
			for (int c = 0; c < 8; c++) {
				int ci = tree.nodes[ni].child[c];
				if (ci >= 0 && !sampled[ci]) post(ci);
			}
		}
		sampled[ni] = 1;
		if (!cleared[ni] && tree.nodes[ni].has_children()) complete_children(ni);
	}
	void chunk(int cr) {
		grow();
		post(cr);
		cleared[cr] = 1;
	}
	void finish(const std::vector<int>& chunk_roots) {
		grow();
		struct CR { int node; std::vector<int> kids; std::vector<int> fcrs; int64_t num_points = 0; };
		std::vector<CR> crs;
		std::unordered_map<int, int> cr_of;
		std::function<void(int)> build = [&](int ni) {
			int me = (int)crs.size();
			crs.push_back(CR{ni, {}, {}, 0});
			cr_of[ni] = me;
			if (cleared[ni]) return;
			for (int c = 0; c < 8; c++) {
				int ci = tree.nodes[ni].child[c];
				if (ci >= 0) {
					build(ci);
					crs[me].kids.push_back(cr_of[ci]);
				}
			}
		};
		build(0);
		for (int cr : chunk_roots) {
			auto it = cr_of.find(cr);
			if (it == cr_of.end()) continue;
			crs[it->second].fcrs.push_back(cr);
			// numPoints of the chunk root after its chunk was sampled
			crs[it->second].num_points += tree.nodes[cr].buf_count;
		}
		std::function<void(int)> merge = [&](int ci) {
			CR& c = crs[ci];
			for (int k : c.kids) merge(k);
			if (c.kids.empty()) return;
			int64_t np = 0;
			for (int k : crs[ci].kids) np += crs[k].num_points;
			crs[ci].num_points = np;
			if (np < kChunkRootMergeThreshold) {
				std::vector<int> f = crs[ci].fcrs;
				for (int k : crs[ci].kids) f.insert(f.end(), crs[k].fcrs.begin(), crs[k].fcrs.end());
				crs[ci].fcrs = f;
				crs[ci].kids.clear();
			}
		};
		merge(0);
		std::vector<int> tasks;
		std::function<void(int)> pre = [&](int ci) {
			if (!crs[ci].fcrs.empty()) tasks.push_back(crs[ci].node);
			for (int k : crs[ci].kids) pre(k);
		};
		pre(0);
		for (int t : tasks) {
			post(t);
			cleared[t] = 1;
		}
		if (!sampled[0]) post(0);
		order.push_back(0);
	}
};

// Device memory this process can allocate now: what the driver reports free
// plus what the stream-ordered allocator's default pool holds without using
// it (the library keeps freed memory in the pool, so the driver counts it
// as taken).
inline size_t device_available(int device) {
	size_t free_b = 0, total_b = 0;
	PCG_CUDA(cudaMemGetInfo(&free_b, &total_b));
	cudaMemPool_t pool;
	uint64_t reserved = 0, used = 0;
	if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess &&
	    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
	    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
		free_b += (size_t)(reserved - used);
	cudaGetLastError();
	return free_b;
}

// Device memory a job of `points` points and `record_bytes` bytes of point
// records is expected to hold at its peak (the request loop's admission
// figure): the records, a per-point working set and the count grid and LUT.
// Checked against pcg_stats.device_peak_bytes by the request-loop tests.
constexpr int64_t kJobBytesPerPoint = 400;
inline size_t estimate_footprint(int64_t points, int64_t record_bytes) {
	return (size_t)(record_bytes + points * kJobBytesPerPoint) + (size_t(256) << 20);
}

struct Converter {
	int device = 0;
	cudaStream_t stream = nullptr;
	uint32_t seed = 1592614637u;
	int form = PCG_FORM_BATCHED;
	PinnedPool* host_buffers = &g_pinned;
	std::shared_ptr<DeviceArena> arena;  // device memory kept between jobs on `stream`

	void run(const pcg_job& job, JobResult& res) {
		auto t0 = Clock::now();
		g_launch_count = 0;
		PCG_CUDA(cudaSetDevice(device));
		std::string err;
		// the job's sources, in order, and the --attributes list
		std::vector<pcg_source> sources;
		if (job.num_sources > 0) {
			if (!job.sources) throw PcgError(PCG_BAD_INPUT, "num_sources is set but sources is NULL");
			sources.assign(job.sources, job.sources + job.num_sources);
		} else {
			sources.push_back({job.las, job.las_size, job.device_records});
		}
		std::vector<std::string> requested;
		if (job.num_attributes > 0) {
			if (!job.attributes) throw PcgError(PCG_BAD_INPUT, "num_attributes is set but attributes is NULL");
			for (int32_t i = 0; i < job.num_attributes; i++) {
				if (!job.attributes[i]) throw PcgError(PCG_BAD_INPUT, "NULL attribute name");
				requested.push_back(job.attributes[i]);
			}
		}
		std::vector<LasInfo> infos(sources.size());
		for (size_t k = 0; k < sources.size(); k++) {
			const uint8_t* las = static_cast<const uint8_t*>(sources[k].las);
			if (!las || !parse_las(las, sources[k].las_size, infos[k], err, sources[k].device_records != nullptr)) {
				std::string what = err.empty() ? "no input" : err;
				throw PcgError(PCG_BAD_INPUT, sources.size() > 1 ? "source " + std::to_string(k) + ": " + what : what);
			}
		}
		Setup s;
		if (!make_setup(infos, requested, s, err)) throw PcgError(PCG_BAD_INPUT, err);
		if (job.method < 0 || job.method > 2) throw PcgError(PCG_BAD_INPUT, "unknown sampling method");
		if (s.total_points < 2) throw PcgError(PCG_BAD_INPUT, "need at least two points");
		// one uncompressed file in host memory may convert in parts
		if (sources.size() == 1 && !infos[0].compressed && !sources[0].device_records && !(job.flags & PCG_JOB_OCTREE_ON_DEVICE)) {
			bool resident = true;
			const int64_t gp = part_plan(s.total_points, infos[0].record_length, resident);
			if (gp > 0) {
				pcg_job one = job;
				one.las = sources[0].las;
				one.las_size = sources[0].las_size;
				run_streamed(one, s, infos[0], static_cast<const uint8_t*>(sources[0].las), gp, resident, res);
				return;
			}
		}
		if (s.total_points >= (int64_t(1) << 31)) throw PcgError(PCG_BAD_INPUT, "more than 2^31 points per job");
		const int64_t N = s.total_points;
		const int method = job.method;
		DeviceMem mem(stream, arena.get());
		if (arena) arena->reset_peak();
		res.stats.num_points = N;
		{
			int64_t rb = 0;
			for (auto& L : infos) rb += L.num_points * (int64_t)L.record_length;
			res.stats.device_estimate_bytes = (int64_t)estimate_footprint(N, rb);
		}

		// ---------------------------------------------------------- input
		// host sources are copied back to back (16-byte aligned) into one
		// device buffer, one copy each; device-resident ones stay in place
		auto t_h2d = Clock::now();
		std::vector<const uint8_t*> src_recs(sources.size(), nullptr);
		std::vector<int64_t> src_base(sources.size(), -1);
		int64_t host_bytes = 0;
		for (size_t k = 0; k < sources.size(); k++) {
			if (sources[k].device_records) {
				src_recs[k] = static_cast<const uint8_t*>(sources[k].device_records);
				continue;
			}
			src_base[k] = host_bytes;
			host_bytes += (infos[k].num_points * (int64_t)infos[k].record_length + 15) & ~int64_t(15);
		}
		double ms_decode = 0.0;
		if (host_bytes > 0) {
			uint8_t* d_host = mem.alloc<uint8_t>(host_bytes);
			for (size_t k = 0; k < sources.size(); k++) {
				if (src_base[k] < 0 || infos[k].compressed) continue;
				const int64_t bytes = infos[k].num_points * (int64_t)infos[k].record_length;
				src_recs[k] = d_host + src_base[k];
				if (bytes > 0)
					PCG_CUDA(cudaMemcpyAsync(d_host + src_base[k], static_cast<const uint8_t*>(sources[k].las) + infos[k].offset_to_points,
					                         bytes, cudaMemcpyHostToDevice, stream));
			}
			// LAZ sources: the compressed chunks go to the device and are
			// decoded there into the source's records
			for (size_t k = 0; k < sources.size(); k++) {
				if (src_base[k] < 0 || !infos[k].compressed) continue;
				src_recs[k] = d_host + src_base[k];
				const auto& chunks = infos[k].laz_chunks;
				if (chunks.empty()) continue;
				const uint64_t base = chunks.front().start, nbytes = chunks.back().end - base;
				uint8_t* d_laz = mem.alloc<uint8_t>(nbytes);
				PCG_CUDA(cudaMemcpyAsync(d_laz, static_cast<const uint8_t*>(sources[k].las) + base, nbytes, cudaMemcpyHostToDevice, stream));
				const auto t_dec = Clock::now();
				launch_laz_decode(d_laz, base, chunks, infos[k].laz_layout, d_host + src_base[k], mem);
				ms_decode += ms_since(t_dec);
				mem.free(d_laz);
				res.stats.laz_chunks += (int64_t)chunks.size();
			}
			PCG_CUDA(cudaStreamSynchronize(stream));
		}
		res.stats.ms_h2d = ms_since(t_h2d) - ms_decode;
		res.stats.ms_decode = ms_decode;

		// ------------------------------------------------------- chunking
		auto t_chunk = Clock::now();
		std::vector<SourceDesc> descs;
		std::vector<int64_t> firsts;
		DecodeParams p = decode_params(s, src_recs, descs, firsts);
		if (p.nsrc > 1) {
			p.srcs = upload(descs, mem);
			p.src_first = upload(firsts, mem);
		}
		const int G = s.grid_size;
		const int64_t cells = (int64_t)G * G * G;
		uint32_t* grid = mem.alloc<uint32_t>(cells);
		PCG_CUDA(cudaMemsetAsync(grid, 0, cells * sizeof(uint32_t), stream));
		ChunkingOut co;
		co.X = mem.alloc<int32_t>(N);
		co.Y = mem.alloc<int32_t>(N);
		co.Z = mem.alloc<int32_t>(N);
		co.cell = mem.alloc<uint32_t>(N);
		std::vector<AttrStatsDev> st_init(MAX_ATTRS);
		for (auto& a : st_init) for (int c = 0; c < 3; c++) { a.mn[c] = ~0ull; a.mx[c] = 0ull; }
		co.stats = upload(st_init, mem);
		co.histogram = mem.alloc<unsigned long long>(256);
		PCG_CUDA(cudaMemsetAsync(co.histogram, 0, 256 * 8, stream));
		co.error = mem.alloc<int64_t>(2);
		PCG_CUDA(cudaMemsetAsync(co.error, 0, 16, stream));
		launch_decode_count(p, grid, co, mem);

		auto errs = download(co.error, 2, stream);
		check_counting_pass(errs[0]);
		int32_t* lut = mem.alloc<int32_t>(cells);
		const std::vector<std::pair<std::string, ChunkCell>> chunks = make_chunks(grid, G, s.max_points_per_chunk, lut, mem);
		const int nchunks = (int)chunks.size();
		uint32_t* ids = mem.alloc<uint32_t>(N);
		scatter_chunks(co.cell, lut, N, nchunks, 0, ids, co.error, mem);
		errs = download(co.error, 2, stream);
		if (errs[1]) throw PcgError(PCG_INTERNAL, "point to chunk lookup failed");
		mem.free(lut);
		mem.free(grid);
		mem.free(co.cell);
		res.stats.num_chunks = nchunks;
		res.stats.ms_chunking = ms_since(t_chunk);

		// ---------------------------------------------------- octree build
		auto t_oct = Clock::now();
		Tree tree;
		const Vec3d rmin = s.cube_min, rmax = s.root_max;
		tree.add("r", -1, rmin, rmax);
		std::vector<int> chunk_roots;
		int64_t off = 0;
		for (int k = 0; k < nchunks; k++) {
			const std::string& id = chunks[k].first;
			int cur = 0;
			for (size_t i = 1; i < id.size(); i++) cur = tree.child_of(cur, id[i] - '0', i + 1 == id.size() ? k : -1);
			TNode& cr = tree.nodes[cur];
			cr.chunk = k;
			cr.chunk_root = true;
			cr.leaf_start = off;
			cr.leaf_count = chunks[k].second.count;
			off += cr.leaf_count;
			chunk_roots.push_back(cur);
		}
		if (off != N) throw PcgError(PCG_INTERNAL, "chunk counts do not add up");
		PosParams pp;
		for (int a = 0; a < 3; a++) { pp.scale[a] = (&s.pos_scale.x)[a]; pp.offset[a] = (&s.pos_offset.x)[a]; }
		const int64_t octree_depth = refine_octree(tree, chunk_roots, ids, co.X, co.Y, co.Z, pp, mem);
		res.stats.octree_depth = octree_depth;
		res.stats.ms_octree = ms_since(t_oct);
		// --------------------------------------------------------- sampling
		auto t_samp = Clock::now();
		SampleStats* d_st = mem.alloc<SampleStats>(1);
		PCG_CUDA(cudaMemsetAsync(d_st, 0, sizeof(SampleStats), stream));
		GreedyArena grid_arena;
		PosParamsS pps;
		for (int a = 0; a < 3; a++) { pps.scale[a] = pp.scale[a]; pps.offset[a] = pp.offset[a]; }
		const double base_spacing = (rmax - rmin).x / 128.0;  // indexer.cpp:1603
		const uint32_t* leaf_ids = ids;
		uint64_t* leaf_cols = nullptr;
		if (method == PCG_RANDOM) {
			// every leaf is shuffled when the sampler visits it (sampler_random.h:89-121)
			std::vector<int64_t> loff, lcnt;
			for (auto& n : tree.nodes)
				if (!n.has_children() && n.leaf_count > 0) { loff.push_back(n.leaf_start); lcnt.push_back(n.leaf_count); }
			uint32_t* shuffled = mem.alloc<uint32_t>(N);
			int32_t* scratch = mem.alloc<int32_t>(N);
			int64_t* d_off = upload(loff, mem);
			int64_t* d_cnt = upload(lcnt, mem);
			launch_shuffle_leaves(d_off, d_cnt, (int)loff.size(), ids, shuffled, scratch, seed, mem);
			leaf_ids = shuffled;
		}
		if (method == PCG_POISSON_AVERAGE) {
			if (p.off_rgb < 0) throw PcgError(PCG_BAD_INPUT, "poisson_average needs an rgb attribute");
			leaf_cols = mem.alloc<uint64_t>(N);
			launch_fill_colors(p, ids, N, leaf_cols, mem);
		}
		int4* leaf_rec = nullptr;
		if (method != PCG_RANDOM) {
			// coordinates travel with the ids from here on
			leaf_rec = mem.alloc<int4>(N);
			launch_gather_records(leaf_ids, N, co.X, co.Y, co.Z, leaf_rec, mem, N);
		}
		for (auto& n : tree.nodes) {
			if (!n.has_children()) {
				n.buf_ids = leaf_ids + n.leaf_start;
				n.buf_cols = leaf_cols ? leaf_cols + n.leaf_start : nullptr;
				n.buf_rec = leaf_rec ? leaf_rec + n.leaf_start : nullptr;
				n.buf_count = n.leaf_count;
			}
		}
		int max_depth = 0;
		for (auto& n : tree.nodes) max_depth = std::max(max_depth, n.depth);
		for (int d = max_depth - 1; d >= 0; d--) {
			// the chunk roots one level down are final once their level ran
			if (method == PCG_RANDOM) reshuffle_chunk_root_tasks(tree, chunk_roots, d + 1, mem);
			std::vector<int> level_nodes;
			for (int i = 0; i < (int)tree.nodes.size(); i++)
				if (tree.nodes[i].depth == d && tree.nodes[i].has_children()) level_nodes.push_back(i);
			if (level_nodes.empty()) continue;
			sample_level(tree, level_nodes, method, base_spacing, pps, co, d_st, grid_arena, mem, res);
		}
		// the root's final payload is its accepted buffer
		TNode& root = tree.nodes[0];
		root.fin_ids = root.buf_ids;
		root.fin_cols = root.buf_cols;
		root.fin_count = root.buf_count;
		auto hst = download(d_st, 1, stream)[0];
		if (hst.timeouts) throw PcgError(PCG_TIMEOUT, "a bounded device loop gave up");
		res.stats.escalated_pairs = (int64_t)hst.escalated;
		res.stats.heapsort_fallbacks = (int64_t)hst.heapsorts;
		res.stats.list_entries = (int64_t)hst.list_entries;
		res.stats.cluster_nodes = (int64_t)hst.cluster_nodes;
		res.stats.ms_sampling = ms_since(t_samp);

		// ------------------------------------------------ completion order
		auto t_out = Clock::now();
		std::vector<int> order = completion_order(tree, chunk_roots, method);
		std::vector<HierRecord> recs;
		std::vector<PayloadItem> items;
		int64_t out_points = 0;
		for (int ni : order) {
			TNode& n = tree.nodes[ni];
			HierRecord r;
			r.name = n.name;
			r.num_points = n.fin_count;
			if (n.fin_count > 0) {
				r.byte_offset = out_points * s.bpp;
				r.byte_size = n.fin_count * s.bpp;
				items.push_back({n.fin_ids, n.fin_cols, n.fin_count, out_points});
				out_points += n.fin_count;
			}
			recs.push_back(r);
		}
		const bool keep_on_device = (job.flags & PCG_JOB_OCTREE_ON_DEVICE) != 0;
		res.octree_size = (uint64_t)(out_points * s.bpp);
		uint8_t* d_out = nullptr;
		if (keep_on_device) {
			// outlives the job's allocations; released by pcg_result_free
			PCG_CUDA(cudaMallocAsync((void**)&d_out, res.octree_size ? res.octree_size : 1, stream));
			res.octree = d_out;
			res.octree_on_device = true;
		} else {
			d_out = mem.alloc<uint8_t>(res.octree_size);
		}
		// the attribute statistics (final since the counting pass) first;
		// then the payloads are written and octree.bin copied out while the
		// host writes hierarchy.bin and metadata.json
		auto stats_dev = download(co.stats, MAX_ATTRS, stream);
		auto hist = download(co.histogram, 256, stream);
		PayloadItem* d_items = upload(items, mem);
		cudaEvent_t ev_out[2];
		for (auto& e : ev_out) PCG_CUDA(cudaEventCreate(&e));
		PCG_CUDA(cudaEventRecord(ev_out[0], stream));
		launch_write_payloads(p, items, d_items, d_out, mem);
		PCG_CUDA(cudaEventRecord(ev_out[1], stream));
		const double ms_out_host = ms_since(t_out);
		auto t_d2h = Clock::now();
		if (!keep_on_device) {
			res.octree = host_buffers ? host_buffers->take(res.octree_size) : nullptr;
			if (!res.octree) PCG_CUDA(cudaMallocHost((void**)&res.octree, res.octree_size ? res.octree_size : 1));
			if (res.octree_size) PCG_CUDA(cudaMemcpyAsync(res.octree, d_out, res.octree_size, cudaMemcpyDeviceToHost, stream));
		}

		// ---------------------------------------------------- host writers
		auto t_w = Clock::now();
		const int64_t num_nodes = (int64_t)recs.size();
		finish_writers(job, s, N, recs, stats_dev, hist, octree_depth, base_spacing, res);
		res.stats.ms_host_writers = ms_since(t_w);
		PCG_CUDA(cudaStreamSynchronize(stream));
		res.stats.ms_d2h = ms_since(t_d2h);  // payloads and copy, overlapped with the host writers
		float ms_payloads = 0.f;
		PCG_CUDA(cudaEventElapsedTime(&ms_payloads, ev_out[0], ev_out[1]));
		for (auto& e : ev_out) cudaEventDestroy(e);
		res.stats.ms_output = ms_out_host + ms_payloads;  // order and records on the host, then the payload kernel
		res.stats.num_nodes = num_nodes;
		res.stats.output_points = out_points;
		res.stats.gpu_launches = g_launch_count;
		if (arena) res.stats.device_peak_bytes = (int64_t)arena->peak_bytes();
		res.stats.ms_total = ms_since(t0);
	}

	// The per-chunk octrees (buildHierarchy, indexer.cpp:823-1109): every
	// node of `roots` holding at least 10,000 points is split by 32^3
	// counting-sort rounds, all pending nodes of the tree per round, until
	// no node is over-full. ids[leaf_start .. leaf_start + leaf_count) are a
	// node's points; they are reordered in place. Returns the deepest level
	// created (the reference's octreeDepth, updated only here, :984-991).
	int64_t refine_octree(Tree& tree, const std::vector<int>& roots, uint32_t* ids, const int32_t* X, const int32_t* Y, const int32_t* Z,
	                      const PosParams& pp, DeviceMem& mem) {
		int64_t octree_depth = 0;
		// nodes to split this round: (node, count of the parent call for the
		// duplicate test, indexer.cpp:1002)
		struct Pending { int node; int64_t parent_count; };
		std::vector<Pending> pending;
		for (int cr : roots)
			if (tree.nodes[cr].leaf_count >= kMaxNodePoints) pending.push_back({cr, -1});
		NodeCand* d_cands = nullptr;
		int32_t* d_ncands = mem.alloc<int32_t>(1);
		int64_t cand_cap = 0;
		while (!pending.empty()) {
			std::vector<SegmentDesc> segs;
			int64_t total = 0;
			for (auto& pd : pending) {
				TNode& n = tree.nodes[pd.node];
				SegmentDesc d;
				d.start = n.leaf_start;
				d.count = n.leaf_count;
				d.coff = total;
				Vec3d size = n.max - n.min;
				d.min[0] = n.min.x; d.min[1] = n.min.y; d.min[2] = n.min.z;
				d.size[0] = size.x; d.size[1] = size.y; d.size[2] = size.z;
				segs.push_back(d);
				total += d.count;
			}
			if (total > cand_cap) {
				if (d_cands) mem.free(d_cands);
				cand_cap = total;
				d_cands = mem.alloc<NodeCand>(cand_cap);
			}
			SegmentDesc* d_segs = upload(segs, mem);
			PCG_CUDA(cudaMemsetAsync(d_ncands, 0, 4, stream));
			launch_octree_round(ids, X, Y, Z, pp, d_segs, (int)segs.size(), total, d_cands, d_ncands, cand_cap, mem);
			int ncand = download(d_ncands, 1, stream)[0];
			if (ncand > cand_cap) throw PcgError(PCG_INTERNAL, "octree round overflow");
			auto cands = download(d_cands, (size_t)ncand, stream);
			mem.free(d_segs);
			// deterministic handling order: by segment, then path
			std::sort(cands.begin(), cands.end(), [](const NodeCand& a, const NodeCand& b) {
				if (a.seg != b.seg) return a.seg < b.seg;
				if (a.level != b.level) return a.level < b.level;
				return a.path < b.path;
			});
			std::vector<Pending> next;
			std::vector<int64_t> seg_depth(segs.size(), 0);
			for (auto& c : cands) {
				int sn = pending[c.seg].node;
				int cur = sn;
				for (int l = 0; l < c.level; l++) {
					int digit = (c.path >> (3 * (c.level - 1 - l))) & 7;
					cur = tree.child_of(cur, digit, tree.nodes[sn].chunk);
				}
				TNode& rn = tree.nodes[cur];
				rn.leaf_start = tree.nodes[sn].leaf_start + c.start;
				rn.leaf_count = c.count;
				octree_depth = std::max<int64_t>(octree_depth, rn.depth);
				if (rn.leaf_count > kMaxNodePoints) next.push_back({cur, tree.nodes[sn].leaf_count});
			}
			// the split node's own points now live in its children (or in the
			// node itself when createNodes kept it whole)
			for (auto& pd : pending) {
				TNode& n = tree.nodes[pd.node];
				if (n.has_children()) n.leaf_count = 0;
			}
			// duplicate handling for nodes that did not split
			std::vector<Pending> refined;
			for (auto& nx : next) {
				TNode& sub = tree.nodes[nx.node];
				if (sub.leaf_count == nx.parent_count) {
					int64_t uniq = count_unique_positions(ids + sub.leaf_start, sub.leaf_count, X, Y, Z, mem);
					int64_t dups = sub.leaf_count - uniq;
					if (dups >= kMaxNodePoints / 2) {
						// the reference keeps the first `uniq` records (indexer.cpp:1088-1090)
						sub.leaf_count = uniq;
					}
				}
				if (sub.leaf_count >= kMaxNodePoints) refined.push_back({nx.node, sub.leaf_count});
			}
			pending.swap(refined);
		}
		if (d_cands) mem.free(d_cands);
		mem.free(d_ncands);
		return octree_depth;
	}

	// Chunk list and LUT from a count grid of G^3 cells (createLUT,
	// chunker_countsort_laszip.cpp:1074-1204): the chunks in chunk
	// file-name order (the order of the pinned reference's sorted directory
	// scan, indexer.cpp:149), and lut[cell] = index of the chunk covering
	// the cell in that order, -1 elsewhere (lut: G^3 entries, filled here).
	std::vector<std::pair<std::string, ChunkCell>> make_chunks(const uint32_t* grid, int G, int64_t max_points_per_chunk, int32_t* lut,
	                                                           DeviceMem& mem) {
		const int chunk_cap = 1 << 20;
		const int64_t cells = (int64_t)G * G * G;
		ChunkCell* d_chunks = mem.alloc<ChunkCell>(chunk_cap);
		int32_t* d_nchunks = mem.alloc<int32_t>(1);
		PCG_CUDA(cudaMemsetAsync(d_nchunks, 0, 4, stream));
		launch_lut_merge(grid, G, max_points_per_chunk, d_chunks, d_nchunks, chunk_cap, mem);
		const int nchunks = download(d_nchunks, 1, stream)[0];
		if (nchunks > chunk_cap) throw PcgError(PCG_INTERNAL, "too many chunks");
		auto cells_found = download(d_chunks, (size_t)nchunks, stream);
		std::vector<std::pair<std::string, ChunkCell>> chunks;
		for (auto& c : cells_found) chunks.push_back({chunk_id(c), c});
		std::sort(chunks.begin(), chunks.end(), [](const auto& a, const auto& b) { return a.first + ".bin" < b.first + ".bin"; });
		std::vector<ChunkCell> sorted_cells;
		for (auto& c : chunks) sorted_cells.push_back(c.second);
		ChunkCell* d_sorted = upload(sorted_cells, mem);
		PCG_CUDA(cudaMemsetAsync(lut, 0xff, cells * sizeof(int32_t), stream));
		launch_lut_fill(d_sorted, nchunks, G, lut, mem);
		mem.free(d_sorted);
		mem.free(d_nchunks);
		mem.free(d_chunks);
		return chunks;
	}

	// The distribution of points to chunks (distributePoints,
	// chunker_countsort_laszip.cpp:837-904, one chunker thread): ids[0..n)
	// = point indices grouped by chunk, input order inside a chunk (a
	// stable radix sort by chunk index). chunk_base is subtracted from every
	// looked-up index (a cloud part holding chunks chunk_base .. + nchunks).
	// A cell without a chunk sets error[1].
	// chunk_start (device, nchunks + 1 entries), when given, receives where
	// every chunk starts in ids.
	void scatter_chunks(const uint32_t* cell, const int32_t* lut, int64_t n, int nchunks, int chunk_base, uint32_t* ids, int64_t* error,
	                    DeviceMem& mem, int64_t* chunk_start = nullptr) {
		uint32_t* chunk_of = mem.alloc<uint32_t>(std::max<int64_t>(n, 1));
		launch_assign_chunks(cell, lut, n, chunk_base, chunk_of, ids, error, mem);
		uint32_t* kt = mem.alloc<uint32_t>(std::max<int64_t>(n, 1));
		uint32_t* vt = mem.alloc<uint32_t>(std::max<int64_t>(n, 1));
		radix_sort_pairs(chunk_of, ids, kt, vt, n, 0, std::max(1, bits_for((uint64_t)std::max(nchunks - 1, 0))), mem);
		if (chunk_start) launch_segment_starts(chunk_of, n, nchunks, chunk_start, mem);
		mem.free(kt);
		mem.free(vt);
		mem.free(chunk_of);
	}

	// ------------------------------------------------ conversion in parts
	// Device bytes one point of a part needs beside its record (positions,
	// ids, the level buffers of the sampler, sort and conflict-list scratch;
	// the request loop's figure, calibrated against pcg_stats.device_peak_bytes,
	// plus headroom for the power-of-two tables of the very large levels a
	// part of hundreds of millions of points has), and the tile of the
	// streamed passes.
	static constexpr int64_t kPartBytesPerPoint = kJobBytesPerPoint + 80;
	static constexpr int64_t kTilePoints = int64_t(1) << 24;
	// largest part an automatic plan makes: parts of this size keep the GPU
	// busy, and smaller level buffers fragment the device memory less
	static constexpr int64_t kMaxPartPoints = 100'000'000;
	int records_mode = PCG_RECORDS_AUTO;  // pcg_records
	int64_t group_points = 0;             // pcg_opts.group_points

	// Whether a one-file job converts in parts: the part size in points (0:
	// in one piece) and whether its records stay on the device.
	int64_t part_plan(int64_t N, int rec_len, bool& resident) const {
		const size_t free_b = device_available(device);
		int64_t avail = (int64_t)((double)free_b * 0.85);
		if (arena) avail += (int64_t)(arena->reserved() - arena->live_bytes());
		const int64_t rec_bytes = N * (int64_t)rec_len;
		const int64_t stream_bytes = 2 * std::min<int64_t>(kTilePoints, N) * rec_len;
		int64_t gp = group_points;
		if (gp <= 0) {
			if (N < (int64_t(1) << 31) && rec_bytes + N * kPartBytesPerPoint <= avail) return 0;
			// per point of a part: its working set, and its piece of
			// octree.bin, which stays on the device until the next part has
			// run (the copy to the host overlaps it)
			const int64_t per_point = kPartBytesPerPoint + rec_len;
			const int64_t gp_res = (avail - rec_bytes) / per_point;
			const int64_t gp_str = (avail - stream_bytes) / per_point;
			// resident records when they leave room for parts of a few chunks
			const bool res_ok = records_mode != PCG_RECORDS_STREAMED && gp_res >= 40'000'000;
			gp = std::min<int64_t>(res_ok ? gp_res : gp_str, kMaxPartPoints);
			if (gp < 10'000'000) throw PcgError(PCG_OOM, "not enough device memory for one chunk of the cloud");
			resident = records_mode == PCG_RECORDS_RESIDENT || (records_mode == PCG_RECORDS_AUTO && res_ok);
			return gp;
		}
		if (N <= gp) return 0;
		resident = records_mode == PCG_RECORDS_RESIDENT ||
		           (records_mode == PCG_RECORDS_AUTO && rec_bytes + std::min(gp, N) * kPartBytesPerPoint <= avail);
		return gp;
	}

	// Device images of pieces of octree.bin whose copy to the host runs on
	// the side stream; each is returned to the job's memory once its copy
	// has finished (`done`), one part later, so the copy overlaps the next
	// part's work.
	struct PieceInFlight {
		uint8_t* dev;
		cudaEvent_t done;
	};

	// Hands the device image of a finished piece of octree.bin to the host
	// on the side stream `d2h` (after the compute stream's work so far); the
	// piece joins res.parts.
	void emit_part(uint8_t* d_part, uint64_t bytes, cudaStream_t d2h, std::vector<PieceInFlight>& inflight, JobResult& res) {
		uint8_t* h = host_buffers ? host_buffers->take(bytes) : nullptr;
		if (!h) PCG_CUDA(cudaMallocHost((void**)&h, bytes));
		res.parts.push_back({h, bytes});
		cudaEvent_t ev, done;
		PCG_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
		PCG_CUDA(cudaEventRecord(ev, stream));
		PCG_CUDA(cudaStreamWaitEvent(d2h, ev, 0));
		PCG_CUDA(cudaEventDestroy(ev));
		PCG_CUDA(cudaMemcpyAsync(h, d_part, bytes, cudaMemcpyDeviceToHost, d2h));
		PCG_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
		PCG_CUDA(cudaEventRecord(done, d2h));
		inflight.push_back({d_part, done});
	}

	// Returns the device images of all pieces but the last `keep` to the
	// job's memory, waiting for their copies first.
	static void retire_pieces(std::vector<PieceInFlight>& inflight, size_t keep, DeviceMem& mem) {
		while (inflight.size() > keep) {
			PCG_CUDA(cudaEventSynchronize(inflight.front().done));
			cudaEventDestroy(inflight.front().done);
			mem.free(inflight.front().dev);
			inflight.erase(inflight.begin());
		}
	}

	// Payloads of the nodes order[o0 ..) (completed since the last call) into
	// a new piece of octree.bin; their hierarchy records join `recs`.
	void write_piece(const Tree& tree, const std::vector<int>& order, size_t o0, const DecodeParams& p, const Setup& s,
	                 std::vector<HierRecord>& recs, int64_t& out_points, cudaStream_t d2h, std::vector<PieceInFlight>& inflight,
	                 DeviceMem& piece_mem, DeviceMem& mem, JobResult& res) {
		std::vector<PayloadItem> items;
		int64_t piece = 0;
		for (size_t i = o0; i < order.size(); i++) {
			const TNode& n = tree.nodes[order[i]];
			HierRecord r;
			r.name = n.name;
			r.num_points = n.fin_count;
			if (n.fin_count > 0) {
				r.byte_offset = (out_points + piece) * s.bpp;
				r.byte_size = n.fin_count * s.bpp;
				items.push_back({n.fin_ids, n.fin_cols, n.fin_count, piece});
				piece += n.fin_count;
			}
			recs.push_back(r);
		}
		out_points += piece;
		if (piece == 0) return;
		uint8_t* d_part = piece_mem.alloc<uint8_t>((size_t)piece * s.bpp);
		PayloadItem* d_items = upload(items, mem);
		launch_write_payloads(p, items, d_items, d_part, mem);
		emit_part(d_part, (uint64_t)piece * s.bpp, d2h, inflight, res);
		mem.free(d_items);
	}

	// Sampler-ready leaves: buffers of every leaf of `nodes` (chunk-local
	// ids into the part's arrays), shuffled for random, with colours for
	// poisson_average and coordinates for the poisson samplers.
	void prepare_leaves(Tree& tree, const std::vector<int>& nodes, int method, const DecodeParams& p, const uint32_t* ids, int64_t n,
	                    const ChunkingOut& co, DeviceMem& mem) {
		const uint32_t* leaf_ids = ids;
		uint64_t* leaf_cols = nullptr;
		if (method == PCG_RANDOM) {
			std::vector<int64_t> loff, lcnt;
			for (int ni : nodes) {
				const TNode& t = tree.nodes[ni];
				if (!t.has_children() && t.leaf_count > 0) { loff.push_back(t.leaf_start); lcnt.push_back(t.leaf_count); }
			}
			uint32_t* shuffled = mem.alloc<uint32_t>(std::max<int64_t>(n, 1));
			int32_t* scratch = mem.alloc<int32_t>(std::max<int64_t>(n, 1));
			int64_t* d_off = upload(loff, mem);
			int64_t* d_cnt = upload(lcnt, mem);
			launch_shuffle_leaves(d_off, d_cnt, (int)loff.size(), ids, shuffled, scratch, seed, mem);
			mem.free(scratch);
			leaf_ids = shuffled;
		}
		if (method == PCG_POISSON_AVERAGE) {
			if (p.off_rgb < 0) throw PcgError(PCG_BAD_INPUT, "poisson_average needs an rgb attribute");
			leaf_cols = mem.alloc<uint64_t>(std::max<int64_t>(n, 1));
			launch_fill_colors(p, ids, n, leaf_cols, mem);
		}
		int4* leaf_rec = nullptr;
		if (method != PCG_RANDOM) {
			leaf_rec = mem.alloc<int4>(std::max<int64_t>(n, 1));
			launch_gather_records(leaf_ids, n, co.X, co.Y, co.Z, leaf_rec, mem, n);
		}
		for (int ni : nodes) {
			TNode& t = tree.nodes[ni];
			if (t.has_children()) continue;
			t.buf_ids = leaf_ids + t.leaf_start;
			t.buf_cols = leaf_cols ? leaf_cols + t.leaf_start : nullptr;
			t.buf_rec = leaf_rec ? leaf_rec + t.leaf_start : nullptr;
			t.buf_count = t.leaf_count;
		}
	}

	// Samples, deepest level first, the inner nodes among `nodes`.
	// processChunkRoots (indexer.cpp:202-281) merges the chunk roots below a
	// node into one task when they hold fewer than 5M points after their
	// chunks were sampled; a chunk root whose parent is not merged stays a
	// task of its own, and sampling that task (indexer.cpp:1717-1730) runs the
	// sampler's callback on the chunk root once more. Its children were
	// cleared after its chunk (:1675), so it is a leaf by then: the random
	// sampler shuffles its points again with the same seed
	// (sampler_random.h:89-121), the poisson samplers return at a leaf. Called
	// for the chunk roots at `depth` (all of them for depth < 0) once the
	// chunk roots below their parents have all been sampled.
	void reshuffle_chunk_root_tasks(Tree& tree, const std::vector<int>& chunk_roots, int depth, DeviceMem& mem) {
		if (chunk_roots.size() < 2) return;  // one chunk: its root is the octree's root
		std::vector<int64_t> below(tree.nodes.size(), 0);  // CRNode::numPoints
		for (int cr : chunk_roots)
			for (int a = tree.nodes[cr].parent; a >= 0; a = tree.nodes[a].parent) below[a] += tree.nodes[cr].buf_count;
		std::vector<int> sel;
		std::vector<int64_t> off, cnt;
		int64_t total = 0;
		for (int cr : chunk_roots) {
			const TNode& n = tree.nodes[cr];
			if ((depth >= 0 && n.depth != depth) || n.parent < 0 || n.buf_count < 2) continue;
			if (below[n.parent] < kChunkRootMergeThreshold) continue;  // merged into an ancestor's task
			sel.push_back(cr);
			off.push_back(total);
			cnt.push_back(n.buf_count);
			total += n.buf_count;
		}
		if (sel.empty()) return;
		const cudaStream_t stream = mem.stream();
		uint32_t* in = mem.alloc<uint32_t>(total);
		uint32_t* out = mem.alloc<uint32_t>(total);
		int32_t* scratch = mem.alloc<int32_t>(total);
		for (size_t i = 0; i < sel.size(); i++)
			PCG_CUDA(cudaMemcpyAsync(in + off[i], tree.nodes[sel[i]].buf_ids, cnt[i] * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream));
		int64_t* d_off = upload(off, mem);
		int64_t* d_cnt = upload(cnt, mem);
		launch_shuffle_leaves(d_off, d_cnt, (int)sel.size(), in, out, scratch, seed, mem);
		for (size_t i = 0; i < sel.size(); i++) tree.nodes[sel[i]].buf_ids = out + off[i];
		mem.free(d_cnt);
		mem.free(d_off);
		mem.free(scratch);
		mem.free(in);
	}

	void sample_nodes(Tree& tree, const std::vector<int>& nodes, int method, double base_spacing, const PosParamsS& pps,
	                  const ChunkingOut& co, SampleStats* d_st, GreedyArena& grid_arena, DeviceMem& mem, JobResult& res) {
		int max_depth = -1;
		for (int ni : nodes)
			if (tree.nodes[ni].has_children()) max_depth = std::max(max_depth, tree.nodes[ni].depth);
		for (int d = max_depth; d >= 0; d--) {
			std::vector<int> level_nodes;
			for (int ni : nodes)
				if (tree.nodes[ni].depth == d && tree.nodes[ni].has_children()) level_nodes.push_back(ni);
			if (!level_nodes.empty()) sample_level(tree, level_nodes, method, base_spacing, pps, co, d_st, grid_arena, mem, res);
		}
	}

	// A one-file cloud converted in parts (the reference's out-of-core
	// path: chunker_countsort_laszip.cpp:1206-1261 counts and distributes
	// in batches through chunk files, indexer.cpp:1581-1745 indexes chunk by
	// chunk and flushes the chunk roots, :181-281). The counting pass streams
	// the records through the device in tiles; the chunks (file-name order)
	// are cut into parts of consecutive chunks of at most part_points
	// points; each part's records are selected from all records (kept on the
	// device, or streamed again), indexed and sampled down to its chunk
	// roots, and its finished nodes' payloads leave for the host while the
	// next part runs. The chunk roots' points survive the part; the levels
	// above them are sampled last. Output bytes equal the one-piece form's.
	void run_streamed(const pcg_job& job, const Setup& s, const LasInfo& info, const uint8_t* las, int64_t part_points, bool resident,
	                  JobResult& res) {
		const auto t0 = Clock::now();
		const int64_t N = s.total_points;
		const int method = job.method;
		const int rec = info.record_length;
		const uint8_t* host_recs = las + info.offset_to_points;
		if (info.offset_to_points + (uint64_t)N * rec > job.las_size) throw PcgError(PCG_BAD_INPUT, "truncated point records");
		DeviceMem mem(stream, arena.get());
		if (arena) arena->reset_peak();
		res.stats.num_points = N;
		res.stats.records_resident = resident ? 1 : 0;
		cudaStream_t d2h = nullptr;
		PCG_CUDA(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking));
		struct StreamGuard {
			cudaStream_t s;
			~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
		} d2h_guard{d2h};

		// ------------------------------------------ counting pass, in tiles
		auto t_chunk = Clock::now();
		std::vector<SourceDesc> descs;
		std::vector<int64_t> firsts;
		const DecodeParams p = decode_params(s, {nullptr}, descs, firsts);
		const int G = s.grid_size;
		const int64_t cells = (int64_t)G * G * G;
		uint32_t* grid = mem.alloc<uint32_t>(cells);
		PCG_CUDA(cudaMemsetAsync(grid, 0, cells * sizeof(uint32_t), stream));
		ChunkingOut co{};
		std::vector<AttrStatsDev> st_init(MAX_ATTRS);
		for (auto& a : st_init) for (int c = 0; c < 3; c++) { a.mn[c] = ~0ull; a.mx[c] = 0ull; }
		co.stats = upload(st_init, mem);
		co.histogram = mem.alloc<unsigned long long>(256);
		PCG_CUDA(cudaMemsetAsync(co.histogram, 0, 256 * 8, stream));
		co.error = mem.alloc<int64_t>(2);
		PCG_CUDA(cudaMemsetAsync(co.error, 0, 16, stream));
		uint8_t* d_all = resident ? mem.alloc<uint8_t>((size_t)N * rec) : nullptr;
		const int64_t T = std::min<int64_t>(kTilePoints, N);
		{
			ChunkingOut ct = co;
			ct.X = mem.alloc<int32_t>(T);
			ct.Y = mem.alloc<int32_t>(T);
			ct.Z = mem.alloc<int32_t>(T);
			ct.cell = mem.alloc<uint32_t>(T);
			TileFeeder feed(host_recs, N, rec, T, stream, d_all, mem);
			for (int64_t t = 0; t < feed.tiles(); t++) {
				int64_t first = 0, count = 0;
				const uint8_t* d = feed.acquire(t, first, count);
				DecodeParams pt = p;
				pt.n = count;
				pt.src0.recs = d;
				pt.src0.first = 0;
				pt.src0.count = count;
				launch_decode_count(pt, grid, ct, mem);
				feed.release(t);
			}
			PCG_CUDA(cudaStreamSynchronize(stream));
			mem.free(ct.X); mem.free(ct.Y); mem.free(ct.Z); mem.free(ct.cell);
		}
		res.stats.ms_h2d = ms_since(t_chunk);
		check_counting_pass(download(co.error, 2, stream)[0]);
		int32_t* lut = mem.alloc<int32_t>(cells);
		const std::vector<std::pair<std::string, ChunkCell>> chunks = make_chunks(grid, G, s.max_points_per_chunk, lut, mem);
		const int nchunks = (int)chunks.size();
		res.stats.num_chunks = nchunks;
		std::vector<std::pair<int, int>> parts;
		{
			int k0 = 0;
			int64_t acc = 0;
			for (int k = 0; k < nchunks; k++) {
				if (k > k0 && acc + chunks[k].second.count > part_points) {
					parts.push_back({k0, k});
					k0 = k;
					acc = 0;
				}
				acc += chunks[k].second.count;
			}
			if (nchunks > k0) parts.push_back({k0, nchunks});
		}
		res.stats.parts = (int64_t)parts.size();
		res.stats.ms_chunking = ms_since(t_chunk);

		// the tree down to the chunk roots
		Tree tree;
		const Vec3d rmin = s.cube_min, rmax = s.root_max;
		tree.add("r", -1, rmin, rmax);
		std::vector<int> chunk_roots;
		for (int k = 0; k < nchunks; k++) {
			const std::string& id = chunks[k].first;
			int cur = 0;
			for (size_t i = 1; i < id.size(); i++) cur = tree.child_of(cur, id[i] - '0', i + 1 == id.size() ? k : -1);
			tree.nodes[cur].chunk = k;
			tree.nodes[cur].chunk_root = true;
			chunk_roots.push_back(cur);
		}
		PosParams pp;
		PosParamsS pps;
		for (int a = 0; a < 3; a++) {
			pp.scale[a] = pps.scale[a] = (&s.pos_scale.x)[a];
			pp.offset[a] = pps.offset[a] = (&s.pos_offset.x)[a];
		}
		const double base_spacing = (rmax - rmin).x / 128.0;  // indexer.cpp:1603
		SampleStats* d_st = mem.alloc<SampleStats>(1);
		PCG_CUDA(cudaMemsetAsync(d_st, 0, sizeof(SampleStats), stream));
		CompletionOrder corder(tree, method);
		std::vector<HierRecord> recs;
		int64_t out_points = 0, octree_depth = 0;

		// survivors: the chunk roots' points after their part, one block of
		// device memory per part
		struct Block {
			std::unique_ptr<DeviceMem> mem;
			uint8_t* recs = nullptr;
			int32_t *X = nullptr, *Y = nullptr, *Z = nullptr;
			uint64_t* cols = nullptr;
			int64_t count = 0;
		};
		std::vector<Block> blocks;
		std::vector<int64_t> surv_off(nchunks, 0);
		int64_t S = 0;
		std::vector<PieceInFlight> inflight;
		struct PiecesGuard {  // on any exit: no piece copy outlives its memory
			std::vector<PieceInFlight>& v;
			~PiecesGuard() {
				for (auto& pc : v) { cudaEventSynchronize(pc.done); cudaEventDestroy(pc.done); }
			}
		} pieces_guard{inflight};

		// ------------------------------------------------------------ parts
		for (const auto& part : parts) {
			const int k0 = part.first, k1 = part.second;
			int64_t n_g = 0;
			for (int k = k0; k < k1; k++) n_g += chunks[k].second.count;
			DeviceMem gm(stream, arena.get());
			auto t_sel = Clock::now();
			uint8_t* g_recs = gm.alloc<uint8_t>((size_t)n_g * rec);
			int64_t* fill = gm.alloc<int64_t>(1);
			PCG_CUDA(cudaMemsetAsync(fill, 0, 8, stream));
			if (resident) {
				launch_select_part(p, d_all, N, lut, k0, k1, fill, g_recs, gm);
			} else {
				TileFeeder feed(host_recs, N, rec, T, stream, nullptr, gm);
				for (int64_t t = 0; t < feed.tiles(); t++) {
					int64_t first = 0, count = 0;
					const uint8_t* d = feed.acquire(t, first, count);
					launch_select_part(p, d, count, lut, k0, k1, fill, g_recs, gm);
					feed.release(t);
				}
			}
			if (download(fill, 1, stream)[0] != n_g) throw PcgError(PCG_INTERNAL, "part selection lost points");
			res.stats.ms_h2d += ms_since(t_sel);
			// the part as a cloud of its own: positions, cells, chunk order
			auto t_oct = Clock::now();
			DecodeParams pg = p;
			pg.n = n_g;
			pg.src0.recs = g_recs;
			pg.src0.first = 0;
			pg.src0.count = n_g;
			ChunkingOut cg{};
			cg.X = gm.alloc<int32_t>(n_g);
			cg.Y = gm.alloc<int32_t>(n_g);
			cg.Z = gm.alloc<int32_t>(n_g);
			cg.cell = gm.alloc<uint32_t>(n_g);
			cg.stats = upload(st_init, gm);
			cg.histogram = gm.alloc<unsigned long long>(256);
			cg.error = gm.alloc<int64_t>(2);
			PCG_CUDA(cudaMemsetAsync(cg.error, 0, 16, stream));
			launch_decode_count(pg, grid, cg, gm);  // the grid is scratch by now
			uint32_t* ids = gm.alloc<uint32_t>(n_g);
			scatter_chunks(cg.cell, lut, n_g, k1 - k0, k0, ids, cg.error, gm);
			if (download(cg.error, 2, stream)[1]) throw PcgError(PCG_INTERNAL, "point to chunk lookup failed");
			gm.free(cg.cell);
			std::vector<int> roots;
			int64_t off = 0;
			for (int k = k0; k < k1; k++) {
				TNode& cr = tree.nodes[chunk_roots[k]];
				cr.leaf_start = off;
				cr.leaf_count = chunks[k].second.count;
				off += cr.leaf_count;
				roots.push_back(chunk_roots[k]);
			}
			octree_depth = std::max(octree_depth, refine_octree(tree, roots, ids, cg.X, cg.Y, cg.Z, pp, gm));
			res.stats.ms_octree += ms_since(t_oct);
			auto t_samp = Clock::now();
			std::vector<int> nodes;
			for (int i = 0; i < (int)tree.nodes.size(); i++)
				if (tree.nodes[i].chunk >= k0 && tree.nodes[i].chunk < k1) nodes.push_back(i);
			prepare_leaves(tree, nodes, method, pg, ids, n_g, cg, gm);
			GreedyArena grid_arena;
			sample_nodes(tree, nodes, method, base_spacing, pps, cg, d_st, grid_arena, gm, res);
			res.stats.ms_sampling += ms_since(t_samp);
			// the part's finished nodes, in completion order
			auto t_out = Clock::now();
			const size_t o0 = corder.order.size();
			for (int cr : roots) corder.chunk(cr);
			retire_pieces(inflight, 1, mem);  // the previous part's piece has been copied meanwhile
			write_piece(tree, corder.order, o0, pg, s, recs, out_points, d2h, inflight, mem, gm, res);
			// the chunk roots' points, carried to the levels above the parts
			Block b;
			for (int cr : roots) b.count += tree.nodes[cr].buf_count;
			b.mem = std::make_unique<DeviceMem>(stream);
			b.recs = b.mem->alloc<uint8_t>((size_t)std::max<int64_t>(b.count, 1) * rec);
			b.X = b.mem->alloc<int32_t>(std::max<int64_t>(b.count, 1));
			b.Y = b.mem->alloc<int32_t>(std::max<int64_t>(b.count, 1));
			b.Z = b.mem->alloc<int32_t>(std::max<int64_t>(b.count, 1));
			if (method == PCG_POISSON_AVERAGE) b.cols = b.mem->alloc<uint64_t>(std::max<int64_t>(b.count, 1));
			int64_t o = 0;
			for (int k = k0; k < k1; k++) {
				const TNode& cr = tree.nodes[chunk_roots[k]];
				surv_off[k] = S + o;
				if (cr.buf_count == 0) continue;
				launch_gather_points(cr.buf_ids, cr.buf_count, g_recs, rec, cg.X, cg.Y, cg.Z, b.recs + (size_t)o * rec, b.X + o, b.Y + o,
				                     b.Z + o, gm);
				if (b.cols)
					PCG_CUDA(cudaMemcpyAsync(b.cols + o, cr.buf_cols, cr.buf_count * sizeof(uint64_t), cudaMemcpyDeviceToDevice, stream));
				o += cr.buf_count;
			}
			S += b.count;
			blocks.push_back(std::move(b));
			// nothing of the part's device memory is referenced any more
			for (int ni : nodes) {
				TNode& t = tree.nodes[ni];
				t.buf_ids = nullptr; t.buf_cols = nullptr; t.buf_rec = nullptr;
				t.fin_ids = nullptr; t.fin_cols = nullptr;
			}
			res.stats.ms_output += ms_since(t_out);
		}
		res.stats.survivors = S;
		res.stats.octree_depth = octree_depth;

		// ---------------------------------- levels above the chunk roots
		auto t_top = Clock::now();
		if (d_all) mem.free(d_all);
		uint8_t* s_recs = mem.alloc<uint8_t>((size_t)std::max<int64_t>(S, 1) * rec);
		ChunkingOut ctop{};
		ctop.X = mem.alloc<int32_t>(std::max<int64_t>(S, 1));
		ctop.Y = mem.alloc<int32_t>(std::max<int64_t>(S, 1));
		ctop.Z = mem.alloc<int32_t>(std::max<int64_t>(S, 1));
		uint64_t* s_cols = method == PCG_POISSON_AVERAGE ? mem.alloc<uint64_t>(std::max<int64_t>(S, 1)) : nullptr;
		{
			int64_t o = 0;
			for (Block& b : blocks) {
				if (b.count) {
					PCG_CUDA(cudaMemcpyAsync(s_recs + (size_t)o * rec, b.recs, (size_t)b.count * rec, cudaMemcpyDeviceToDevice, stream));
					PCG_CUDA(cudaMemcpyAsync(ctop.X + o, b.X, b.count * 4, cudaMemcpyDeviceToDevice, stream));
					PCG_CUDA(cudaMemcpyAsync(ctop.Y + o, b.Y, b.count * 4, cudaMemcpyDeviceToDevice, stream));
					PCG_CUDA(cudaMemcpyAsync(ctop.Z + o, b.Z, b.count * 4, cudaMemcpyDeviceToDevice, stream));
					if (s_cols) PCG_CUDA(cudaMemcpyAsync(s_cols + o, b.cols, b.count * 8, cudaMemcpyDeviceToDevice, stream));
				}
				o += b.count;
				b.mem.reset();
			}
		}
		uint32_t* s_ids = mem.alloc<uint32_t>(std::max<int64_t>(S, 1));
		launch_iota(s_ids, S, mem);
		int4* s_rec4 = nullptr;
		if (method != PCG_RANDOM) {
			s_rec4 = mem.alloc<int4>(std::max<int64_t>(S, 1));
			launch_gather_records(s_ids, S, ctop.X, ctop.Y, ctop.Z, s_rec4, mem);
		}
		for (int k = 0; k < nchunks; k++) {
			TNode& cr = tree.nodes[chunk_roots[k]];
			cr.buf_ids = s_ids + surv_off[k];
			cr.buf_cols = s_cols ? s_cols + surv_off[k] : nullptr;
			cr.buf_rec = s_rec4 ? s_rec4 + surv_off[k] : nullptr;
		}
		DecodeParams ptop = p;
		ptop.n = S;
		ptop.src0.recs = s_recs;
		ptop.src0.first = 0;
		ptop.src0.count = S;
		std::vector<int> upper;
		for (int i = 0; i < (int)tree.nodes.size(); i++)
			if (tree.nodes[i].chunk < 0) upper.push_back(i);
		if (method == PCG_RANDOM) reshuffle_chunk_root_tasks(tree, chunk_roots, -1, mem);
		GreedyArena grid_arena;
		sample_nodes(tree, upper, method, base_spacing, pps, ctop, d_st, grid_arena, mem, res);
		TNode& root = tree.nodes[0];
		root.fin_ids = root.buf_ids;
		root.fin_cols = root.buf_cols;
		root.fin_count = root.buf_count;
		const size_t o0 = corder.order.size();
		corder.finish(chunk_roots);
		write_piece(tree, corder.order, o0, ptop, s, recs, out_points, d2h, inflight, mem, mem, res);
		const auto hst = download(d_st, 1, stream)[0];
		if (hst.timeouts) throw PcgError(PCG_TIMEOUT, "a bounded device loop gave up");
		res.stats.escalated_pairs = (int64_t)hst.escalated;
		res.stats.heapsort_fallbacks = (int64_t)hst.heapsorts;
		res.stats.list_entries = (int64_t)hst.list_entries;
		res.stats.cluster_nodes = (int64_t)hst.cluster_nodes;
		res.stats.ms_sampling += ms_since(t_top);

		// ------------------------------------------------------ host writers
		const auto stats_dev = download(co.stats, MAX_ATTRS, stream);
		const auto hist = download(co.histogram, 256, stream);
		auto t_w = Clock::now();
		finish_writers(job, s, N, recs, stats_dev, hist, octree_depth, base_spacing, res);
		res.stats.ms_host_writers = ms_since(t_w);
		auto t_d2h = Clock::now();
		PCG_CUDA(cudaStreamSynchronize(d2h));
		retire_pieces(inflight, 0, mem);
		res.stats.ms_d2h = ms_since(t_d2h);
		res.octree = nullptr;
		res.octree_size = (uint64_t)(out_points * s.bpp);
		res.stats.output_points = out_points;
		res.stats.num_nodes = (int64_t)res.nodes.size();
		res.stats.gpu_launches = g_launch_count;
		if (arena) res.stats.device_peak_bytes = (int64_t)arena->peak_bytes();
		res.stats.ms_total = ms_since(t0);
	}

	// hierarchy.bin and metadata.json from the completed nodes and the
	// counting pass's attribute statistics; res.nodes takes the records
	void finish_writers(const pcg_job& job, const Setup& s, int64_t N, std::vector<HierRecord>& recs, const std::vector<AttrStatsDev>& stats_dev,
	                    const std::vector<unsigned long long>& hist, int64_t octree_depth, double base_spacing, JobResult& res) {
		std::string err;
		int64_t first_chunk = 0;
		if (!build_hierarchy(recs, res.hierarchy, first_chunk, err)) throw PcgError(PCG_INTERNAL, err);
		std::vector<AttrStats> astats(s.attrs.size());
		for (size_t i = 0; i < s.attrs.size(); i++) {
			const auto& sd = stats_dev[i];
			astats[i].min = {decode_ordered(sd.mn[0]), decode_ordered(sd.mn[1]), decode_ordered(sd.mn[2])};
			astats[i].max = {decode_ordered(sd.mx[0]), decode_ordered(sd.mx[1]), decode_ordered(sd.mx[2])};
			// the reference passes the statistics through the chunks'
			// metadata.json, where a non-finite value (or none at all: an
			// attribute no point carries) comes back as +Infinity
			// (chunker_countsort_laszip.cpp:1005-1070, indexer.cpp:72-130)
			for (int c = 0; c < s.attrs[i].numElements && c < 3; c++) {
				double* mn = &astats[i].min.x + c;
				double* mx = &astats[i].max.x + c;
				if (!std::isfinite(*mn)) *mn = INFINITY;
				if (!std::isfinite(*mx)) *mx = INFINITY;
			}
			astats[i].histogram.assign(256, 0);
			if (s.attrs[i].kind == AK_CLASSIFICATION)
				for (int k = 0; k < 256; k++) astats[i].histogram[k] = (int64_t)hist[k];
		}
		res.metadata = build_metadata(job.name ? job.name : "", job.projection ? job.projection : "", N, first_chunk, octree_depth, s,
		                              astats, base_spacing);
		res.nodes = std::move(recs);
	}

	// Kernel parameters of the decode: the output layout, and per source its
	// records, coordinate transform and handler byte moves (src_recs: device
	// pointer of each source's first record). descs / firsts receive the
	// source table for jobs with several sources.
	static DecodeParams decode_params(const Setup& s, const std::vector<const uint8_t*>& src_recs, std::vector<SourceDesc>& descs,
	                                  std::vector<int64_t>& firsts) {
		DecodeParams p{};
		for (int a = 0; a < 3; a++) {
			p.pos_scale[a] = (&s.pos_scale.x)[a];
			p.pos_offset[a] = (&s.pos_offset.x)[a];
			p.cmin[a] = (&s.cube_min.x)[a];
		}
		p.csize = s.chunk_cube_size;
		p.n = s.total_points;
		p.bpp = s.bpp;
		p.grid = s.grid_size;
		p.off_intensity = p.off_retnum = p.off_nret = p.off_class = p.off_sar = p.off_user = p.off_psid = p.off_gps = p.off_rgb = -1;
		p.stat_intensity = p.stat_retnum = p.stat_nret = p.stat_class = p.stat_sar = p.stat_user = p.stat_psid = p.stat_gps = p.stat_rgb = -1;
		if ((int)s.attrs.size() > MAX_ATTRS) throw PcgError(PCG_BAD_INPUT, "too many attributes");
		for (int i = 0; i < (int)s.attrs.size(); i++) {
			const AttrDesc& a = s.attrs[i];
			switch (a.kind) {
			case AK_POSITION: p.stat_pos = i; break;
			case AK_INTENSITY: p.off_intensity = a.out_offset; p.stat_intensity = i; break;
			case AK_RETURN_NUMBER: p.off_retnum = a.out_offset; p.stat_retnum = i; break;
			case AK_NUMBER_OF_RETURNS: p.off_nret = a.out_offset; p.stat_nret = i; break;
			case AK_CLASSIFICATION: p.off_class = a.out_offset; p.stat_class = i; break;
			case AK_SCAN_ANGLE_RANK: p.off_sar = a.out_offset; p.stat_sar = i; break;
			case AK_USER_DATA: p.off_user = a.out_offset; p.stat_user = i; break;
			case AK_POINT_SOURCE_ID: p.off_psid = a.out_offset; p.stat_psid = i; break;
			case AK_GPS_TIME: p.off_gps = a.out_offset; p.stat_gps = i; break;
			case AK_RGB: p.off_rgb = a.out_offset; p.stat_rgb = i; break;
			default: break;  // extra bytes: per source below
			}
		}
		descs.assign(s.sources.size(), SourceDesc{});
		firsts.clear();
		int64_t first = 0;
		p.max_rec_len = 0;
		for (size_t k = 0; k < s.sources.size(); k++) {
			const SourceSetup& ss = s.sources[k];
			const LasInfo& L = ss.las;
			SourceDesc& d = descs[k];
			for (int a = 0; a < 3; a++) {
				d.in_scale[a] = (&L.scale.x)[a];
				d.in_offset[a] = (&L.offset.x)[a];
			}
			d.recs = src_recs[k];
			d.first = first;
			d.count = L.num_points;
			d.rec_len = L.record_length;
			d.src_gps = (L.pdrf == 1 || L.pdrf == 3) ? 20 : -1;
			d.src_rgb = L.pdrf == 2 ? 20 : (L.pdrf == 3 ? 28 : -1);
			d.zero_fill = ss.zero_fill ? 1 : 0;
			if ((int)ss.extras.size() > MAX_EXTRA) throw PcgError(PCG_BAD_INPUT, "too many extra attributes");
			d.n_extra = (int)ss.extras.size();
			for (int e = 0; e < d.n_extra; e++) {
				const auto& x = ss.extras[e];
				const AttrDesc& oa = s.attrs[x.out_index];
				d.extra[e] = {x.src_off, x.dst_off, x.size, (int)oa.type, oa.numElements, oa.elementSize, x.out_index, 0};
			}
			firsts.push_back(first);
			first += L.num_points;
			p.max_rec_len = std::max(p.max_rec_len, L.record_length);
		}
		p.nsrc = (int)s.sources.size();
		p.src0 = descs[0];
		return p;
	}

	// Samples every node of level_nodes (all at one depth). level_cols, when
	// given, receives the level's packed colours in gather order (every
	// candidate's averaged colour, poisson_average).
	void sample_level(Tree& tree, const std::vector<int>& level_nodes, int method, double base_spacing, const PosParamsS& pps,
	                  const ChunkingOut& co, SampleStats* d_st, GreedyArena& grid_arena, DeviceMem& mem, JobResult& res,
	                  uint64_t** level_cols = nullptr) {
		const auto t_level = Clock::now();
		const double alloc0 = mem.alloc_ms();
		int sms = 148;
		PCG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
		(void)res;
		const int K = (int)level_nodes.size();
		std::vector<LevelNode> ln(K);
		std::vector<GatherItem> items;
		struct ChildSlot { int node; int64_t start, count; };
		std::vector<ChildSlot> child_slots;  // per (node, child) in gather order
		int64_t M = 0, H = 0;
		for (int k = 0; k < K; k++) {
			TNode& n = tree.nodes[level_nodes[k]];
			LevelNode& l = ln[k];
			l.cand_off = M;
			for (int c = 0; c < 8; c++) {
				int ci = n.child[c];
				if (ci < 0) continue;
				TNode& ch = tree.nodes[ci];
				if (ch.buf_count > 0) items.push_back({ch.buf_ids, ch.buf_cols, ch.buf_rec, M, ch.buf_count, c, k});
				child_slots.push_back({ci, M, ch.buf_count});
				M += ch.buf_count;
			}
			l.count = M - l.cand_off;
			int64_t cap = 64;
			while (cap < 2 * l.count) cap <<= 1;
			l.hash_off = H;
			l.hash_cap = cap;
			H += cap;
			l.min[0] = n.min.x; l.min[1] = n.min.y; l.min[2] = n.min.z;
			l.max[0] = n.max.x; l.max[1] = n.max.y; l.max[2] = n.max.z;
			l.level = n.depth;
			l.spacing = base_spacing / std::pow(2.0, (double)n.depth);  // sampler_poisson.h:114
			l.pad = 0;
		}
		res.stats.sampled_nodes += K;
		res.stats.candidates += M;
		cudaStream_t s = stream;
		LevelBuffers lb;
		lb.M = M;
		lb.K = K;
		lb.ids = mem.alloc<uint32_t>(M);
		lb.cols = method == PCG_POISSON_AVERAGE ? mem.alloc<uint64_t>(M) : nullptr;
		lb.child = mem.alloc<uint8_t>(M);
		lb.node_of = mem.alloc<int32_t>(M);
		lb.count_in_child = mem.alloc<int32_t>(M);
		lb.accepted = mem.alloc<uint8_t>(M);
		lb.rec = method == PCG_RANDOM ? nullptr : mem.alloc<int4>(M);
		LevelNode* d_nodes = upload(ln, mem);
		GatherItem* d_items = upload(items, mem);
		launch_gather(items, d_items, lb, mem);
		// node order for the warp-per-node kernels: largest first
		std::vector<int32_t> order(K);
		for (int k = 0; k < K; k++) order[k] = k;
		std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ln[a].count > ln[b].count; });
		int32_t* d_order = upload(order, mem);
		uint64_t* hkeys = mem.alloc<uint64_t>(H);
		int32_t* hvals = mem.alloc<int32_t>(H);
		if (method == PCG_RANDOM) {
			launch_random_accept_sized(d_nodes, co.X, co.Y, co.Z, pps, lb, hkeys, hvals, H, d_st, mem);
		} else {
			lb.keys = mem.alloc<double>(M);
			lb.perm = mem.alloc<int32_t>(M);
			lb.pos = mem.alloc<int32_t>(M);
			lb.acc_rank = mem.alloc<int32_t>(M);
			lb.cq = mem.alloc<int4>(M);
			launch_keys(d_nodes, pps, lb, mem);
			double* axyz = mem.alloc<double>(3 * M);
			double* akey = mem.alloc<double>(M);
			int32_t* anext = mem.alloc<int32_t>(M);
			int32_t* apos = mem.alloc<int32_t>(M);
			const int mode = method == PCG_POISSON ? 0 : 1;
			const bool guard = form == PCG_FORM_BATCHED;
			// large nodes get a CTA each; on levels with few nodes every node
			// of some size does, so the GPU is not left to a handful of warps
			int num_big = 0;
			const LevelSchedule sch = level_schedule();
			const int64_t big_min = K < 2 * sms ? sch.small_level_cta_min : sch.cta_min;
			while (num_big < K && ln[order[num_big]].count >= big_min) num_big++;
			int list_nodes = 0;
			cudaEvent_t ev_lists;
			PCG_CUDA(cudaEventCreate(&ev_lists));
			cudaEvent_t ev[3];
			for (auto& e : ev) PCG_CUDA(cudaEventCreate(&e));
			PCG_CUDA(cudaEventRecord(ev[0], s));
			if (form == PCG_FORM_PLAIN) {
				for (int k = 0; k < K; k++) launch_node_sort(d_nodes, d_order, K, lb, d_st, mem, k, k + 1, num_big);
				launch_cand_records(d_nodes, co.X, co.Y, co.Z, lb, mem);
				PCG_CUDA(cudaEventRecord(ev[1], s));
				for (int k = 0; k < K; k++)
					launch_greedy(mode, false, d_nodes, d_order, K, co.X, co.Y, co.Z, pps, lb, hkeys, hvals, axyz, akey, anext, apos, d_st, mem, &grid_arena, k, k + 1,
					              num_big);
			} else {
				// distinct keys: one exact radix sort of the level; equal keys:
				// the introsort replay, for those nodes only
				std::vector<uint8_t> tie;
				SortedLevel sorted;
				sort_level_distinct(d_nodes, ln, lb, mem, tie, &sorted);
				std::vector<int32_t> tie_nodes;
				std::vector<SortSeg> tie_segs;
				for (int k = 0; k < K; k++) {
					if (!tie[k]) continue;
					tie_nodes.push_back(k);
					tie_segs.push_back({ln[k].cand_off, ln[k].cand_off + ln[k].count, sort_depth_budget(ln[k].count), 0});
					res.stats.replayed_candidates += ln[k].count;
				}
				res.stats.replayed_nodes += (int64_t)tie_nodes.size();
				if (!tie_nodes.empty()) {
					replay_segments(lb.keys, lb.perm, M, tie_segs, d_st, mem, &sorted);
					launch_node_pos(d_nodes, tie, lb, mem);
				}
				free_sorted_level(sorted, mem);
				launch_cand_records(d_nodes, co.X, co.Y, co.Z, lb, mem);
				PCG_CUDA(cudaEventRecord(ev[1], s));
				// conflict lists for every node; a node where some candidate has
				// too many close predecessors keeps the lookup kernels
				ConflictLists cl;
				std::vector<int32_t> cta_list, warp_list, order2;
				{
					std::vector<uint8_t> use(K, 1), dense;
					build_conflict_lists(mode, d_nodes, ln, use, pps, lb, cl, dense, d_st, mem);
					PCG_CUDA(cudaEventRecord(ev_lists, s));
					for (int i = 0; i < num_big; i++) (dense[order[i]] ? order2 : cta_list).push_back(order[i]);
					const int num_grid = (int)order2.size();
					for (int i = num_big; i < K; i++) (dense[order[i]] ? order2 : warp_list).push_back(order[i]);
					list_nodes = (int)(cta_list.size() + warp_list.size());
					launch_greedy_lists(mode, d_nodes, cta_list, warp_list, pps, lb, hkeys, hvals, axyz, akey, anext, apos, cl, d_st, mem, ln);
					if (!order2.empty()) {
						int32_t* d_order2 = upload(order2, mem);
						launch_greedy(mode, guard, d_nodes, d_order2, (int)order2.size(), co.X, co.Y, co.Z, pps, lb, hkeys, hvals, axyz, akey,
						              anext, apos, d_st, mem, &grid_arena, 0, -1, num_grid);
						mem.free(d_order2);
					}
				}
				free_conflict_lists(cl, mem);
			}
			PCG_CUDA(cudaEventRecord(ev[2], s));
			PCG_CUDA(cudaEventSynchronize(ev[2]));
			float t_sort = 0, t_greedy = 0;
			PCG_CUDA(cudaEventElapsedTime(&t_sort, ev[0], ev[1]));
			PCG_CUDA(cudaEventElapsedTime(&t_greedy, ev[1], ev[2]));
			res.stats.ms_sort += t_sort;
			res.stats.ms_greedy += t_greedy;
			float t_lists = 0;
			if (form != PCG_FORM_PLAIN) PCG_CUDA(cudaEventElapsedTime(&t_lists, ev[1], ev_lists));
			res.stats.ms_lists += t_lists;
			cudaEventDestroy(ev_lists);
			if (trace_levels()) {
				int64_t mx = 0;
				for (auto& l : ln) mx = std::max<int64_t>(mx, l.count);
				static thread_local SampleStats prev{};
				SampleStats now = download(d_st, 1, s)[0];
				if (now.rounds < prev.rounds) prev = SampleStats{};
				fprintf(stderr,
				        "[pcg] level %d: nodes %d (cta %d, lists %d), candidates %lld, largest %lld, sort %.3f ms, greedy %.3f ms (lists %.3f), "
				        "host %.3f ms (alloc %.3f), cta rounds %llu, passes %llu, serial rounds %llu, kcycles/round A %.1f C1 %.1f C2 %.1f D %.1f\n",
				        K ? ln[0].level : -1, K, num_big, list_nodes, (long long)M, (long long)mx, t_sort, t_greedy, t_lists, ms_since(t_level), mem.alloc_ms() - alloc0,
				        now.rounds - prev.rounds, now.passes - prev.passes, now.serial - prev.serial,
				        [&](int i) { return (double)(now.cycles[i] - prev.cycles[i]) / 1e3 / std::max(1ull, now.rounds - prev.rounds); }(0),
				        [&](int i) { return (double)(now.cycles[i] - prev.cycles[i]) / 1e3 / std::max(1ull, now.rounds - prev.rounds); }(2),
				        [&](int i) { return (double)(now.cycles[i] - prev.cycles[i]) / 1e3 / std::max(1ull, now.rounds - prev.rounds); }(3),
				        [&](int i) { return (double)(now.cycles[i] - prev.cycles[i]) / 1e3 / std::max(1ull, now.rounds - prev.rounds); }(4));
				prev = now;
			}
			for (auto& e : ev) cudaEventDestroy(e);
			if (method == PCG_POISSON_AVERAGE) {
				long long* sums = mem.alloc<long long>(4 * M);
				launch_average_colors(d_nodes, co.X, co.Y, co.Z, pps, lb, hkeys, hvals, axyz, anext, apos, nullptr, sums, mem);
				mem.free(sums);
			}
			mem.free(axyz); mem.free(akey); mem.free(anext); mem.free(apos);
			mem.free(lb.keys); mem.free(lb.perm); mem.free(lb.pos); mem.free(lb.acc_rank); mem.free(lb.cq);
		}
		mem.free(hkeys);
		mem.free(hvals);
		// split candidates into the parents' buffers and the children's payloads
		uint32_t* pre = mem.alloc<uint32_t>(M + 1);
		uint32_t* acc_ids = mem.alloc<uint32_t>(M);
		uint64_t* acc_cols = lb.cols ? mem.alloc<uint64_t>(M) : nullptr;
		uint32_t* rej_ids = method == PCG_POISSON_AVERAGE ? nullptr : mem.alloc<uint32_t>(M);
		int4* acc_rec = lb.rec ? mem.alloc<int4>(M) : nullptr;
		launch_split(lb.accepted, M, lb.ids, lb.cols, lb.rec, pre, acc_ids, acc_cols, acc_rec, rej_ids, mem);
		// prefix values at node and child boundaries
		std::vector<int64_t> bidx;
		for (int k = 0; k < K; k++) { bidx.push_back(ln[k].cand_off); bidx.push_back(ln[k].cand_off + ln[k].count); }
		for (auto& cs : child_slots) { bidx.push_back(cs.start); bidx.push_back(cs.start + cs.count); }
		int64_t* d_bidx = upload(bidx, mem);
		uint32_t* d_bval = mem.alloc<uint32_t>(bidx.size());
		launch_gather_u32(pre, d_bidx, (int64_t)bidx.size(), d_bval, mem);
		auto bval = download(d_bval, bidx.size(), s);
		// parents
		for (int k = 0; k < K; k++) {
			TNode& n = tree.nodes[level_nodes[k]];
			uint32_t a0 = bval[2 * k], a1 = bval[2 * k + 1];
			n.buf_ids = acc_ids + a0;
			n.buf_cols = acc_cols ? acc_cols + a0 : nullptr;
			n.buf_rec = acc_rec ? acc_rec + a0 : nullptr;
			n.buf_count = (int64_t)(a1 - a0);
		}
		// children (sampler_poisson.h:247-291, sampler_poisson_average.h:418-475, sampler_random.h:184-225)
		size_t base = 2 * (size_t)K;
		for (size_t i = 0; i < child_slots.size(); i++) {
			const ChildSlot& cs = child_slots[i];
			TNode& ch = tree.nodes[cs.node];
			uint32_t a0 = bval[base + 2 * i], a1 = bval[base + 2 * i + 1];
			int64_t accepted = (int64_t)(a1 - a0);
			int64_t rejected = cs.count - accepted;
			if (method == PCG_POISSON_AVERAGE) {
				if (rejected == 0) {
					ch.unlinked = true;  // dropped, never completed (:465-466)
				} else {
					ch.completed = true;
					ch.fin_ids = lb.ids + cs.start;
					ch.fin_cols = lb.cols + cs.start;
					ch.fin_count = cs.count;  // the child keeps all of its points
				}
			} else {
				ch.completed = true;
				if (rejected == 0) {
					if (!ch.has_children()) ch.unlinked = true;
					ch.fin_count = 0;
				} else {
					ch.fin_ids = rej_ids + (cs.start - a0);
					ch.fin_cols = nullptr;
					ch.fin_count = rejected;
				}
			}
		}
		mem.free(d_bidx);
		mem.free(d_bval);
		mem.free(pre);
		mem.free(d_nodes);
		mem.free(d_items);
		mem.free(d_order);
		mem.free(lb.child);
		mem.free(lb.node_of);
		mem.free(lb.count_in_child);
		mem.free(lb.accepted);
		if (lb.rec) mem.free(lb.rec);
		if (method != PCG_POISSON_AVERAGE) mem.free(lb.ids);
		if (level_cols) *level_cols = lb.cols;
	}

	// The single-threaded reference's completion order (doIndexing,
	// indexer.cpp:1639-1745): chunks in file-name order, each sampled in
	// post-order; then the merged chunk-root tasks (processChunkRoots,
	// :202-281) in pre-order; then the root.
	static std::vector<int> completion_order(Tree& tree, const std::vector<int>& chunk_roots, int method) {
		CompletionOrder co(tree, method);
		for (int cr : chunk_roots) co.chunk(cr);
		co.finish(chunk_roots);
		return co.order;
	}
};

}  // namespace

}  // namespace pcg

// ====================================================================== C ABI

struct pcg_ctx {
	pcg::Converter conv;
	std::mutex mtx;
	std::string last_error;
	// request loop
	struct Job {
		uint64_t id;
		// the job's LAS images, copied back to back at submit: into a pinned
		// buffer of the pool when one can be had (the worker's host-to-device
		// copies then run at link speed), else into `las`
		uint8_t* las_pinned = nullptr;
		size_t las_size = 0;
		std::vector<uint8_t> las;
		std::vector<size_t> src_off, src_size;  // every source's image in it
		bool multi = false;                     // given as a source list
		std::vector<std::string> attributes;
		std::string name, projection;
		int32_t method;
		bool done = false;
		pcg_status status = PCG_OK;
		std::string error;
		pcg::JobResult result;
		size_t footprint = 0;
		int bypassed = 0;  // times a later job was admitted before it
	};
	std::mutex qmtx;
	std::condition_variable qcv;
	std::deque<std::shared_ptr<Job>> queue;
	std::unordered_map<uint64_t, std::shared_ptr<Job>> jobs;
	std::vector<std::thread> workers;
	std::vector<cudaStream_t> worker_streams;
	size_t budget = 0, in_use = 0;
	uint64_t next_id = 1;
	bool stopping = false;
	bool own_stream = true;
};

namespace {

pcg_status fail(pcg_ctx* ctx, pcg_status st, const std::string& msg) {
	if (ctx) ctx->last_error = msg;
	return st;
}

template <class F>
pcg_status guarded(pcg_ctx* ctx, F&& f) {
	try {
		f();
		return PCG_OK;
	} catch (const pcg::PcgError& e) {
		return fail(ctx, (pcg_status)e.status, e.what());
	} catch (const pcg::CudaError& e) {
		cudaGetLastError();
		return fail(ctx, e.code == cudaErrorMemoryAllocation ? PCG_OOM : PCG_CUDA, e.what());
	} catch (const std::bad_alloc&) {
		return fail(ctx, PCG_OOM, "host allocation failed");
	} catch (const std::exception& e) {
		return fail(ctx, PCG_INTERNAL, e.what());
	}
}

void move_result(pcg::JobResult& r, pcg_result* out, int device) {
	memset(out, 0, sizeof(*out));
	if (r.octree_on_device && r.octree) {
		std::lock_guard<std::mutex> lk(pcg::g_dev_mtx);
		pcg::g_dev_results[r.octree] = device;
	}
	out->octree = r.octree;
	out->octree_size = r.octree_size;
	r.octree = nullptr;
	out->hierarchy = (uint8_t*)malloc(r.hierarchy.size() + 1);
	if (!r.hierarchy.empty()) memcpy(out->hierarchy, r.hierarchy.data(), r.hierarchy.size());
	out->hierarchy_size = r.hierarchy.size();
	out->metadata = (char*)malloc(r.metadata.size() + 1);
	memcpy(out->metadata, r.metadata.data(), r.metadata.size());
	out->metadata[r.metadata.size()] = 0;
	out->metadata_size = r.metadata.size();
	out->stats = r.stats;
	// octree.bin in pieces: the one image, or the parts (owned by the result)
	const size_t np = r.octree || r.parts.empty() ? 1 : r.parts.size();
	out->octree_parts = (pcg_octree_part*)malloc(sizeof(pcg_octree_part) * np);
	if (out->octree_parts) {
		if (r.octree || r.parts.empty()) {
			out->octree_parts[0] = {out->octree, out->octree_size};
		} else {
			for (size_t i = 0; i < np; i++) out->octree_parts[i] = {r.parts[i].first, r.parts[i].second};
			r.parts.clear();
		}
		out->num_octree_parts = np;
	}
	// node list: the records, then their names, in one block
	size_t chars = 0;
	for (auto& n : r.nodes) chars += n.name.size() + 1;
	char* block = (char*)malloc(sizeof(pcg_node) * r.nodes.size() + chars + 1);
	if (block) {
		pcg_node* nodes = reinterpret_cast<pcg_node*>(block);
		char* name = block + sizeof(pcg_node) * r.nodes.size();
		for (size_t i = 0; i < r.nodes.size(); i++) {
			const auto& n = r.nodes[i];
			memcpy(name, n.name.c_str(), n.name.size() + 1);
			nodes[i] = pcg_node{name, n.num_points, (uint64_t)n.byte_offset, (uint64_t)n.byte_size};
			name += n.name.size() + 1;
		}
		out->nodes = nodes;
		out->num_nodes = r.nodes.size();
	}
}

// Points and bytes of point records a source image stands for: its
// header's point count x record length (a LAZ image is several times
// smaller than the records it decodes to), at least the image size.
size_t record_bytes(const void* image, size_t size, size_t* points = nullptr) {
	if (points) *points = size / 20;
	const uint8_t* h = static_cast<const uint8_t*>(image);
	if (size < 227 || std::memcmp(h, "LASF", 4) != 0) return size;
	uint16_t header_size, rec_len;
	uint32_t legacy;
	std::memcpy(&header_size, h + 94, 2);
	std::memcpy(&rec_len, h + 105, 2);
	std::memcpy(&legacy, h + 107, 4);
	uint64_t count = legacy;
	if (h[25] >= 4 && header_size >= 375 && size >= 255) {
		uint64_t ext;
		std::memcpy(&ext, h + 247, 8);
		if (ext > count) count = ext;
	}
	if (count > (uint64_t(1) << 32)) return size;  // implausible; parsing will refuse it
	if (points) *points = count;
	const uint64_t bytes = count * rec_len;
	return bytes > size ? (size_t)bytes : size;
}


constexpr int kMaxBypass = 16;

void worker_main(pcg_ctx* ctx, int wi) {
	pcg::Converter conv = ctx->conv;
	conv.stream = ctx->worker_streams[wi];
	// jobs of a worker share its arena; it is emptied after each job so the
	// memory admission of the queue sees what the jobs hold
	conv.arena = std::make_shared<pcg::DeviceArena>(conv.stream);
	while (true) {
		std::shared_ptr<pcg_ctx::Job> job;
		{
			std::unique_lock<std::mutex> lk(ctx->qmtx);
			// first fit: the oldest job whose footprint fits the memory left
			// (any job when nothing runs); a job bypassed kMaxBypass times
			// blocks the ones behind it until it fits
			auto pick = [&]() -> std::deque<std::shared_ptr<pcg_ctx::Job>>::iterator {
				for (auto it = ctx->queue.begin(); it != ctx->queue.end(); ++it) {
					if (ctx->in_use == 0 || ctx->in_use + (*it)->footprint <= ctx->budget) return it;
					if ((*it)->bypassed >= kMaxBypass) break;
				}
				return ctx->queue.end();
			};
			ctx->qcv.wait(lk, [&] { return ctx->stopping || pick() != ctx->queue.end(); });
			if (ctx->stopping && ctx->queue.empty()) return;
			auto it = pick();
			if (it == ctx->queue.end()) continue;
			for (auto b = ctx->queue.begin(); b != it; ++b) (*b)->bypassed++;
			job = *it;
			ctx->queue.erase(it);
			ctx->in_use += job->footprint;
		}
		pcg_job pj{};
		const uint8_t* image = job->las_pinned ? job->las_pinned : job->las.data();
		std::vector<pcg_source> srcs;
		for (size_t k = 0; k < job->src_off.size(); k++) srcs.push_back({image + job->src_off[k], job->src_size[k], nullptr});
		std::vector<const char*> names;
		for (auto& a : job->attributes) names.push_back(a.c_str());
		if (job->multi) {
			pj.num_sources = (int32_t)srcs.size();
			pj.sources = srcs.data();
		} else {
			pj.las = image;
			pj.las_size = job->las_size;
		}
		pj.num_attributes = (int32_t)names.size();
		pj.attributes = names.empty() ? nullptr : names.data();
		pj.method = job->method;
		pj.name = job->name.c_str();
		pj.projection = job->projection.c_str();
		std::string err;
		pcg_status st = PCG_OK;
		try {
			conv.run(pj, job->result);
		} catch (const pcg::PcgError& e) {
			st = (pcg_status)e.status; err = e.what();
		} catch (const pcg::CudaError& e) {
			cudaGetLastError(); st = PCG_CUDA; err = e.what();
		} catch (const std::exception& e) {
			st = PCG_INTERNAL; err = e.what();
		}
		if (st != PCG_OK) job->result.release_parts();
		conv.arena->release_all();
		if (job->las_pinned) {
			pcg::g_pinned.give(job->las_pinned);
			job->las_pinned = nullptr;
		}
		std::vector<uint8_t>().swap(job->las);
		{
			std::lock_guard<std::mutex> lk(ctx->qmtx);
			job->status = st;
			job->error = err;
			job->done = true;
			ctx->in_use -= job->footprint;
		}
		ctx->qcv.notify_all();
	}
}

}  // namespace

extern "C" {

const char* pcg_status_string(pcg_status s) {
	switch (s) {
	case PCG_OK: return "ok";
	case PCG_BAD_INPUT: return "bad input";
	case PCG_OUT_OF_BOX: return "point outside bounding box";
	case PCG_OOM: return "out of memory";
	case PCG_TIMEOUT: return "timeout";
	case PCG_INTERNAL: return "internal error";
	case PCG_CUDA: return "cuda error";
	case PCG_NOT_FOUND: return "not found";
	}
	return "unknown";
}

pcg_status pcg_create(pcg_ctx** out, const pcg_opts* opts) {
	if (!out) return PCG_BAD_INPUT;
	*out = nullptr;
	pcg_ctx* ctx = new (std::nothrow) pcg_ctx();
	if (!ctx) return PCG_OOM;
	pcg_status st = guarded(ctx, [&] {
		if (opts) {
			ctx->conv.device = opts->device;
			ctx->conv.seed = opts->random_seed;
			ctx->conv.form = opts->form;
			if (opts->records < PCG_RECORDS_AUTO || opts->records > PCG_RECORDS_STREAMED || opts->group_points < 0)
				throw pcg::PcgError(PCG_BAD_INPUT, "bad records placement or part size");
			ctx->conv.records_mode = opts->records;
			ctx->conv.group_points = opts->group_points;
		}
		int n = 0;
		PCG_CUDA(cudaGetDeviceCount(&n));
		if (ctx->conv.device < 0 || ctx->conv.device >= n) throw pcg::PcgError(PCG_BAD_INPUT, "no such CUDA device");
		PCG_CUDA(cudaSetDevice(ctx->conv.device));
		if (opts && opts->stream) {
			ctx->conv.stream = static_cast<cudaStream_t>(opts->stream);
			ctx->own_stream = false;
		} else {
			PCG_CUDA(cudaStreamCreateWithFlags(&ctx->conv.stream, cudaStreamNonBlocking));
		}
		cudaMemPool_t pool;
		PCG_CUDA(cudaDeviceGetDefaultMemPool(&pool, ctx->conv.device));
		uint64_t threshold = UINT64_MAX;
		PCG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
		ctx->conv.arena = std::make_shared<pcg::DeviceArena>(ctx->conv.stream);
	});
	if (st != PCG_OK) {
		fprintf(stderr, "pcg_create: %s\n", ctx->last_error.c_str());
		delete ctx;
		return st;
	}
	*out = ctx;
	return PCG_OK;
}

void pcg_destroy(pcg_ctx* ctx) {
	if (!ctx) return;
	{
		std::lock_guard<std::mutex> lk(ctx->qmtx);
		ctx->stopping = true;
	}
	ctx->qcv.notify_all();
	for (auto& t : ctx->workers) t.join();
	for (auto& kv : ctx->jobs) {
		if (kv.second->result.octree && !pcg::g_pinned.give(kv.second->result.octree)) cudaFreeHost(kv.second->result.octree);
		kv.second->result.release_parts();
	}
	for (auto& kv : ctx->jobs)
		if (kv.second->las_pinned) pcg::g_pinned.give(kv.second->las_pinned);
	cudaSetDevice(ctx->conv.device);
	for (auto s : ctx->worker_streams) cudaStreamDestroy(s);
	ctx->conv.arena.reset();
	if (ctx->conv.stream) {
		cudaStreamSynchronize(ctx->conv.stream);
		if (ctx->own_stream) cudaStreamDestroy(ctx->conv.stream);
	}
	delete ctx;
}

const char* pcg_last_error(const pcg_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }

pcg_status pcg_convert(pcg_ctx* ctx, const pcg_job* job, pcg_result* out) {
	if (!ctx || !job || !out) return PCG_BAD_INPUT;
	std::lock_guard<std::mutex> lk(ctx->mtx);
	memset(out, 0, sizeof(*out));
	pcg::JobResult r;
	pcg_status st = guarded(ctx, [&] { ctx->conv.run(*job, r); });
	if (st != PCG_OK) {
		if (r.octree_on_device && r.octree) cudaFree(r.octree);
		else if (r.octree && !pcg::g_pinned.give(r.octree)) cudaFreeHost(r.octree);
		r.release_parts();  // their copies ended with the conversion's side stream
		return st;
	}
	move_result(r, out, ctx->conv.device);
	return PCG_OK;
}

void pcg_result_free(pcg_result* r) {
	if (!r) return;
	if (!r->octree && r->octree_parts)  // the pieces of a conversion in parts
		for (uint64_t i = 0; i < r->num_octree_parts; i++) pcg::release_octree(const_cast<uint8_t*>(r->octree_parts[i].data));
	free(r->octree_parts);
	pcg::release_octree(r->octree);
	free(r->hierarchy);
	free(r->metadata);
	free(r->nodes);
	memset(r, 0, sizeof(*r));
}

pcg_status pcg_write_files(const pcg_result* r, const char* dir) {
	if (!r || !dir) return PCG_BAD_INPUT;
	auto wr = [&](const char* name, const void* data, uint64_t size) {
		std::ofstream f(std::string(dir) + "/" + name, std::ios::binary);
		if (!f) return false;
		f.write((const char*)data, (std::streamsize)size);
		return (bool)f;
	};
	if (r->octree || !r->octree_parts) {
		if (!wr("octree.bin", r->octree, r->octree_size)) return PCG_BAD_INPUT;
	} else {
		std::ofstream f(std::string(dir) + "/octree.bin", std::ios::binary);
		for (uint64_t i = 0; f && i < r->num_octree_parts; i++)
			f.write((const char*)r->octree_parts[i].data, (std::streamsize)r->octree_parts[i].size);
		if (!f) return PCG_BAD_INPUT;
	}
	if (!wr("hierarchy.bin", r->hierarchy, r->hierarchy_size)) return PCG_BAD_INPUT;
	if (!wr("metadata.json", r->metadata, r->metadata_size)) return PCG_BAD_INPUT;
	return PCG_OK;
}

pcg_status pcg_submit(pcg_ctx* ctx, const pcg_job* job, uint64_t* job_id) {
	if (!ctx || !job || !job_id) return PCG_BAD_INPUT;
	// the request loop takes host images only; they are copied here
	std::vector<pcg_source> srcs;
	if (job->num_sources > 0) {
		if (!job->sources) return PCG_BAD_INPUT;
		srcs.assign(job->sources, job->sources + job->num_sources);
	} else {
		srcs.push_back({job->las, job->las_size, job->device_records});
	}
	for (auto& src : srcs)
		if (!src.las || src.device_records) return PCG_BAD_INPUT;
	if (job->num_attributes > 0 && !job->attributes) return PCG_BAD_INPUT;
	for (int32_t i = 0; i < job->num_attributes; i++)
		if (!job->attributes[i]) return PCG_BAD_INPUT;
	return guarded(ctx, [&] {
		// the images are copied before the queue is locked, so a large job's
		// copy does not hold up the workers
		auto j = std::make_shared<pcg_ctx::Job>();
		size_t total = 0;
		for (auto& src : srcs) {
			j->src_off.push_back(total);
			j->src_size.push_back(src.las_size);
			total += (src.las_size + 15) & ~size_t(15);
		}
		j->multi = job->num_sources > 0;
		j->las_size = total;
		j->las_pinned = pcg::g_pinned.take(total ? total : 1);
		uint8_t* image = j->las_pinned;
		if (!image) {
			j->las.resize(total);
			image = j->las.data();
		}
		for (size_t k = 0; k < srcs.size(); k++) std::memcpy(image + j->src_off[k], srcs[k].las, srcs[k].las_size);
		if (!j->multi) j->las_size = srcs[0].las_size;
		for (int32_t i = 0; i < job->num_attributes; i++) j->attributes.push_back(job->attributes[i]);
		j->name = job->name ? job->name : "";
		j->projection = job->projection ? job->projection : "";
		j->method = job->method;
		size_t records = 0, points = 0;
		for (auto& src : srcs) {
			size_t np = 0;
			records += record_bytes(src.las, src.las_size, &np);
			points += np;
		}
		j->footprint = pcg::estimate_footprint((int64_t)points, (int64_t)records);
		std::lock_guard<std::mutex> lk(ctx->qmtx);
		if (ctx->workers.empty()) {
			PCG_CUDA(cudaSetDevice(ctx->conv.device));
			const size_t free_b = pcg::device_available(ctx->conv.device);
			ctx->budget = (size_t)(free_b * 0.8);
			const int nworkers = 4;
			for (int i = 0; i < nworkers; i++) {
				cudaStream_t s;
				PCG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
				ctx->worker_streams.push_back(s);
			}
			for (int i = 0; i < nworkers; i++) ctx->workers.emplace_back(worker_main, ctx, i);
		}
		j->id = ctx->next_id++;
		ctx->jobs[j->id] = j;
		ctx->queue.push_back(j);
		*job_id = j->id;
		ctx->qcv.notify_all();
	});
}

pcg_status pcg_poll(pcg_ctx* ctx, uint64_t job_id, int32_t* done) {
	if (!ctx || !done) return PCG_BAD_INPUT;
	std::lock_guard<std::mutex> lk(ctx->qmtx);
	auto it = ctx->jobs.find(job_id);
	if (it == ctx->jobs.end()) return PCG_NOT_FOUND;
	*done = it->second->done ? 1 : 0;
	return PCG_OK;
}

pcg_status pcg_wait(pcg_ctx* ctx, uint64_t job_id, pcg_result* out) {
	if (!ctx || !out) return PCG_BAD_INPUT;
	std::shared_ptr<pcg_ctx::Job> j;
	{
		std::unique_lock<std::mutex> lk(ctx->qmtx);
		auto it = ctx->jobs.find(job_id);
		if (it == ctx->jobs.end()) return PCG_NOT_FOUND;
		j = it->second;
		ctx->qcv.wait(lk, [&] { return j->done; });
		ctx->jobs.erase(job_id);
	}
	memset(out, 0, sizeof(*out));
	if (j->status != PCG_OK) {
		ctx->last_error = j->error;
		return j->status;
	}
	move_result(j->result, out, ctx->conv.device);
	return PCG_OK;
}

pcg_status pcg_kernel_sort_keys(pcg_ctx* ctx, const double* keys, int64_t n, int32_t* perm_out) {
	if (!ctx || (n > 0 && (!keys || !perm_out)) || n < 0 || n >= (int64_t(1) << 31)) return PCG_BAD_INPUT;
	std::lock_guard<std::mutex> lk(ctx->mtx);
	return guarded(ctx, [&] {
		if (n == 0) return;
		PCG_CUDA(cudaSetDevice(ctx->conv.device));
		pcg::DeviceMem mem(ctx->conv.stream, ctx->conv.arena.get());
		double* dk = mem.alloc<double>(n);
		int32_t* dv = mem.alloc<int32_t>(n);
		pcg::SampleStats* st = mem.alloc<pcg::SampleStats>(1);
		PCG_CUDA(cudaMemsetAsync(st, 0, sizeof(pcg::SampleStats), mem.stream()));
		PCG_CUDA(cudaMemcpyAsync(dk, keys, n * sizeof(double), cudaMemcpyHostToDevice, mem.stream()));
		std::vector<int32_t> iota(n);
		for (int64_t i = 0; i < n; i++) iota[i] = (int32_t)i;
		PCG_CUDA(cudaMemcpyAsync(dv, iota.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, mem.stream()));
		// keys >= +0 (the samplers' squared distances): the replay finishes
		// the partitions whose keys are distinct from their radix order
		bool nonneg = true;
		for (int64_t i = 0; i < n && nonneg; i++) nonneg = keys[i] >= 0.0 && !std::signbit(keys[i]);
		pcg::SortedLevel sorted;
		int32_t* d_node_of = nullptr;
		pcg::LevelNode* d_one = nullptr;
		if (nonneg) {
			std::vector<pcg::LevelNode> one(1);
			one[0].cand_off = 0;
			one[0].count = n;
			d_one = pcg::upload(one, mem);
			d_node_of = mem.alloc<int32_t>(n);
			PCG_CUDA(cudaMemsetAsync(d_node_of, 0, n * sizeof(int32_t), mem.stream()));
			pcg::build_sorted_level(d_one, one, d_node_of, reinterpret_cast<const uint64_t*>(dk), n, sorted, mem);
		}
		pcg::launch_sort_keys_single(dk, dv, n, mem, st, nonneg ? &sorted : nullptr);
		pcg::free_sorted_level(sorted, mem);
		if (d_node_of) mem.free(d_node_of);
		if (d_one) mem.free(d_one);
		PCG_CUDA(cudaMemcpyAsync(perm_out, dv, n * sizeof(int32_t), cudaMemcpyDeviceToHost, mem.stream()));
		PCG_CUDA(cudaStreamSynchronize(mem.stream()));
	});
}

pcg_status pcg_kernel_shuffle(pcg_ctx* ctx, int64_t n, uint32_t seed, int32_t* perm_out) {
	if (!ctx || n < 0 || (n > 0 && !perm_out) || n >= (int64_t(1) << 31)) return PCG_BAD_INPUT;
	std::lock_guard<std::mutex> lk(ctx->mtx);
	return guarded(ctx, [&] {
		if (n == 0) return;
		PCG_CUDA(cudaSetDevice(ctx->conv.device));
		pcg::DeviceMem mem(ctx->conv.stream, ctx->conv.arena.get());
		int32_t* dp = mem.alloc<int32_t>(n);
		pcg::launch_shuffle_single(n, seed, dp, mem);
		PCG_CUDA(cudaMemcpyAsync(perm_out, dp, n * sizeof(int32_t), cudaMemcpyDeviceToHost, mem.stream()));
		PCG_CUDA(cudaStreamSynchronize(mem.stream()));
	});
}

pcg_status pcg_kernel_decode_count(pcg_ctx* ctx, const void* las, uint64_t size, int32_t* X, int32_t* Y, int32_t* Z, uint32_t* cell,
                                   int64_t point_capacity, uint32_t* grid, int64_t grid_capacity, int32_t* grid_size) {
	if (!ctx || !las || !grid_size) return PCG_BAD_INPUT;
	std::lock_guard<std::mutex> lk(ctx->mtx);
	return guarded(ctx, [&] {
		pcg::LasInfo info;
		std::string err;
		if (!pcg::parse_las(static_cast<const uint8_t*>(las), size, info, err)) throw pcg::PcgError(PCG_BAD_INPUT, err);
		pcg::Setup s;
		if (!pcg::make_setup(info, s, err)) throw pcg::PcgError(PCG_BAD_INPUT, err);
		const int64_t N = s.total_points;
		const int64_t G = s.grid_size, cells = G * G * G;
		if (N >= (int64_t(1) << 31)) throw pcg::PcgError(PCG_BAD_INPUT, "more than 2^31 points");
		if (!grid || grid_capacity < cells) throw pcg::PcgError(PCG_BAD_INPUT, "grid is smaller than grid_size^3");
		if (N > point_capacity) throw pcg::PcgError(PCG_BAD_INPUT, "the file holds more points than the X/Y/Z/cell buffers");
		if (N > 0 && (!X || !Y || !Z || !cell)) throw pcg::PcgError(PCG_BAD_INPUT, "NULL output");
		*grid_size = (int32_t)G;
		PCG_CUDA(cudaSetDevice(ctx->conv.device));
		cudaStream_t stream = ctx->conv.stream;
		pcg::DeviceMem mem(stream, ctx->conv.arena.get());
		// the records on the device, as the conversion puts them there
		uint8_t* d_recs = mem.alloc<uint8_t>(std::max<int64_t>(1, N * (int64_t)info.record_length));
		if (info.compressed) {
			const auto& chunks = info.laz_chunks;
			if (!chunks.empty()) {
				const uint64_t base = chunks.front().start, nbytes = chunks.back().end - base;
				uint8_t* d_laz = mem.alloc<uint8_t>(nbytes);
				PCG_CUDA(cudaMemcpyAsync(d_laz, static_cast<const uint8_t*>(las) + base, nbytes, cudaMemcpyHostToDevice, stream));
				pcg::launch_laz_decode(d_laz, base, chunks, info.laz_layout, d_recs, mem);
			}
		} else if (N > 0) {
			PCG_CUDA(cudaMemcpyAsync(d_recs, static_cast<const uint8_t*>(las) + info.offset_to_points, N * (int64_t)info.record_length,
			                         cudaMemcpyHostToDevice, stream));
		}
		std::vector<pcg::SourceDesc> descs;
		std::vector<int64_t> firsts;
		pcg::DecodeParams p = pcg::Converter::decode_params(s, {d_recs}, descs, firsts);
		uint32_t* d_grid = mem.alloc<uint32_t>(cells);
		PCG_CUDA(cudaMemsetAsync(d_grid, 0, cells * sizeof(uint32_t), stream));
		pcg::ChunkingOut co;
		co.X = mem.alloc<int32_t>(std::max<int64_t>(1, N));
		co.Y = mem.alloc<int32_t>(std::max<int64_t>(1, N));
		co.Z = mem.alloc<int32_t>(std::max<int64_t>(1, N));
		co.cell = mem.alloc<uint32_t>(std::max<int64_t>(1, N));
		std::vector<pcg::AttrStatsDev> st_init(pcg::MAX_ATTRS);
		for (auto& a : st_init) for (int c = 0; c < 3; c++) { a.mn[c] = ~0ull; a.mx[c] = 0ull; }
		co.stats = pcg::upload(st_init, mem);
		co.histogram = mem.alloc<unsigned long long>(256);
		PCG_CUDA(cudaMemsetAsync(co.histogram, 0, 256 * 8, stream));
		co.error = mem.alloc<int64_t>(2);
		PCG_CUDA(cudaMemsetAsync(co.error, 0, 16, stream));
		pcg::launch_decode_count(p, d_grid, co, mem);
		const auto errs = pcg::download(co.error, 2, stream);
		pcg::check_counting_pass(errs[0]);
		if (N > 0) {
			PCG_CUDA(cudaMemcpyAsync(X, co.X, N * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
			PCG_CUDA(cudaMemcpyAsync(Y, co.Y, N * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
			PCG_CUDA(cudaMemcpyAsync(Z, co.Z, N * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
			PCG_CUDA(cudaMemcpyAsync(cell, co.cell, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
		}
		PCG_CUDA(cudaMemcpyAsync(grid, d_grid, cells * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
		PCG_CUDA(cudaStreamSynchronize(stream));
	});
}

pcg_status pcg_kernel_lut(pcg_ctx* ctx, const uint32_t* grid, int32_t grid_size, int64_t max_points_per_chunk, int32_t* lut_out,
                          pcg_chunk* chunks_out, int64_t chunk_capacity, int32_t* num_chunks) {
	if (!ctx || !grid || !lut_out || !num_chunks) return PCG_BAD_INPUT;
	if (grid_size < 2 || grid_size > 512 || (grid_size & (grid_size - 1)) != 0 || max_points_per_chunk < 0) return PCG_BAD_INPUT;
	std::lock_guard<std::mutex> lk(ctx->mtx);
	return guarded(ctx, [&] {
		PCG_CUDA(cudaSetDevice(ctx->conv.device));
		const cudaStream_t stream = ctx->conv.stream;
		pcg::DeviceMem mem(stream, ctx->conv.arena.get());
		const int64_t cells = (int64_t)grid_size * grid_size * grid_size;
		uint32_t* d_grid = mem.alloc<uint32_t>(cells);
		int32_t* d_lut = mem.alloc<int32_t>(cells);
		PCG_CUDA(cudaMemcpyAsync(d_grid, grid, cells * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
		const auto chunks = ctx->conv.make_chunks(d_grid, grid_size, max_points_per_chunk, d_lut, mem);
		*num_chunks = (int32_t)chunks.size();
		if ((int64_t)chunks.size() > chunk_capacity || (!chunks.empty() && !chunks_out))
			throw pcg::PcgError(PCG_BAD_INPUT, "more chunks than chunk_capacity");
		for (size_t k = 0; k < chunks.size(); k++) {
			pcg_chunk c{};
			std::snprintf(c.id, sizeof(c.id), "%s", chunks[k].first.c_str());
			c.level = chunks[k].second.level;
			c.x = chunks[k].second.x;
			c.y = chunks[k].second.y;
			c.z = chunks[k].second.z;
			c.count = chunks[k].second.count;
			chunks_out[k] = c;
		}
		PCG_CUDA(cudaMemcpyAsync(lut_out, d_lut, cells * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
		PCG_CUDA(cudaStreamSynchronize(stream));
	});
}

pcg_status pcg_kernel_scatter(pcg_ctx* ctx, const uint32_t* cell, int64_t n, const int32_t* lut, int32_t grid_size, int32_t num_chunks,
                              uint32_t* ids_out, int64_t* chunk_start) {
	if (!ctx || !lut || !chunk_start || n < 0 || n >= (int64_t(1) << 31) || num_chunks < 0) return PCG_BAD_INPUT;
	if (n > 0 && (!cell || !ids_out)) return PCG_BAD_INPUT;
	if (grid_size < 2 || grid_size > 512 || (grid_size & (grid_size - 1)) != 0) return PCG_BAD_INPUT;
	std::lock_guard<std::mutex> lk(ctx->mtx);
	return guarded(ctx, [&] {
		PCG_CUDA(cudaSetDevice(ctx->conv.device));
		const cudaStream_t stream = ctx->conv.stream;
		pcg::DeviceMem mem(stream, ctx->conv.arena.get());
		const int64_t cells = (int64_t)grid_size * grid_size * grid_size;
		// cells beyond the grid would index past the LUT
		for (int64_t i = 0; i < n; i++)
			if (cell[i] >= (uint64_t)cells) throw pcg::PcgError(PCG_BAD_INPUT, "cell index outside the grid");
		uint32_t* d_cell = mem.alloc<uint32_t>(std::max<int64_t>(n, 1));
		int32_t* d_lut = mem.alloc<int32_t>(cells);
		uint32_t* d_ids = mem.alloc<uint32_t>(std::max<int64_t>(n, 1));
		int64_t* d_start = mem.alloc<int64_t>((size_t)num_chunks + 1);
		int64_t* d_err = mem.alloc<int64_t>(2);
		PCG_CUDA(cudaMemsetAsync(d_err, 0, 16, stream));
		if (n > 0) PCG_CUDA(cudaMemcpyAsync(d_cell, cell, n * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
		PCG_CUDA(cudaMemcpyAsync(d_lut, lut, cells * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
		ctx->conv.scatter_chunks(d_cell, d_lut, n, num_chunks, 0, d_ids, d_err, mem, d_start);
		if (n == 0) {
			for (int32_t k = 0; k <= num_chunks; k++) chunk_start[k] = 0;
			return;
		}
		const auto err = pcg::download(d_err, 2, stream);
		if (err[1]) throw pcg::PcgError(PCG_INTERNAL, "point " + std::to_string(err[1] - 1) + ": its cell belongs to no chunk");
		PCG_CUDA(cudaMemcpyAsync(ids_out, d_ids, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
		PCG_CUDA(cudaMemcpyAsync(chunk_start, d_start, ((size_t)num_chunks + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
		PCG_CUDA(cudaStreamSynchronize(stream));
	});
}

pcg_status pcg_kernel_octree(pcg_ctx* ctx, const int32_t* X, const int32_t* Y, const int32_t* Z, int64_t n, const double* scale,
                             const double* offset, const double* box_min, const double* box_max, const char* root_name,
                             uint32_t* order_out, pcg_octree_node* nodes_out, int64_t node_capacity, int64_t* num_nodes,
                             int64_t* octree_depth) {
	if (!ctx || !scale || !offset || !box_min || !box_max || !root_name || !num_nodes || !octree_depth) return PCG_BAD_INPUT;
	if (n < 0 || n >= (int64_t(1) << 31) || (n > 0 && (!X || !Y || !Z || !order_out))) return PCG_BAD_INPUT;
	if (root_name[0] != 'r' || std::strlen(root_name) > 24) return PCG_BAD_INPUT;
	std::lock_guard<std::mutex> lk(ctx->mtx);
	return guarded(ctx, [&] {
		PCG_CUDA(cudaSetDevice(ctx->conv.device));
		const cudaStream_t stream = ctx->conv.stream;
		pcg::DeviceMem mem(stream, ctx->conv.arena.get());
		pcg::Tree tree;
		tree.add(root_name, -1, pcg::Vec3d{box_min[0], box_min[1], box_min[2]}, pcg::Vec3d{box_max[0], box_max[1], box_max[2]});
		tree.nodes[0].chunk = 0;
		tree.nodes[0].chunk_root = true;
		tree.nodes[0].leaf_start = 0;
		tree.nodes[0].leaf_count = n;
		const size_t nb = (size_t)std::max<int64_t>(n, 1);
		int32_t* d_X = mem.alloc<int32_t>(nb);
		int32_t* d_Y = mem.alloc<int32_t>(nb);
		int32_t* d_Z = mem.alloc<int32_t>(nb);
		std::vector<uint32_t> iota((size_t)n);
		for (int64_t i = 0; i < n; i++) iota[i] = (uint32_t)i;
		uint32_t* d_ids = pcg::upload(iota, mem);
		if (n > 0) {
			PCG_CUDA(cudaMemcpyAsync(d_X, X, n * 4, cudaMemcpyHostToDevice, stream));
			PCG_CUDA(cudaMemcpyAsync(d_Y, Y, n * 4, cudaMemcpyHostToDevice, stream));
			PCG_CUDA(cudaMemcpyAsync(d_Z, Z, n * 4, cudaMemcpyHostToDevice, stream));
		}
		pcg::PosParams pp;
		for (int a = 0; a < 3; a++) { pp.scale[a] = scale[a]; pp.offset[a] = offset[a]; }
		*octree_depth = ctx->conv.refine_octree(tree, {0}, d_ids, d_X, d_Y, d_Z, pp, mem);
		std::vector<int> order(tree.nodes.size());
		for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
		std::sort(order.begin(), order.end(), [&](int a, int b) { return tree.nodes[a].name < tree.nodes[b].name; });
		*num_nodes = (int64_t)order.size();
		if ((int64_t)order.size() > node_capacity || !nodes_out) throw pcg::PcgError(PCG_BAD_INPUT, "more nodes than node_capacity");
		for (size_t k = 0; k < order.size(); k++) {
			const pcg::TNode& t = tree.nodes[order[k]];
			pcg_octree_node o{};
			std::snprintf(o.name, sizeof(o.name), "%s", t.name.c_str());
			o.is_leaf = t.has_children() ? 0 : 1;
			o.start = o.is_leaf ? t.leaf_start : 0;
			o.count = o.is_leaf ? t.leaf_count : 0;
			nodes_out[k] = o;
		}
		if (n > 0) PCG_CUDA(cudaMemcpyAsync(order_out, d_ids, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
		PCG_CUDA(cudaStreamSynchronize(stream));
	});
}

pcg_status pcg_kernel_accept(pcg_ctx* ctx, int32_t method, const int32_t* X, const int32_t* Y, const int32_t* Z, const uint8_t* child,
                             const uint16_t* rgb, int64_t n, const double* scale, const double* offset, const double* box_min,
                             const double* box_max, double spacing, uint8_t* accepted_out, uint16_t* rgb_out) {
	if (!ctx || !scale || !offset || !box_min || !box_max || method < 0 || method > 2) return PCG_BAD_INPUT;
	if (n < 0 || n >= (int64_t(1) << 31) || (n > 0 && (!X || !Y || !Z || !child || !accepted_out))) return PCG_BAD_INPUT;
	if (method == PCG_POISSON_AVERAGE && n > 0 && !rgb) return PCG_BAD_INPUT;
	if (!(spacing > 0.0)) return PCG_BAD_INPUT;
	for (int64_t i = 0; i < n; i++)
		if (child[i] > 7 || (i > 0 && child[i] < child[i - 1])) return PCG_BAD_INPUT;
	std::lock_guard<std::mutex> lk(ctx->mtx);
	return guarded(ctx, [&] {
		if (n == 0) return;
		PCG_CUDA(cudaSetDevice(ctx->conv.device));
		const cudaStream_t stream = ctx->conv.stream;
		pcg::DeviceMem mem(stream, ctx->conv.arena.get());
		// the node "r" (level 0, so baseSpacing = spacing) with one leaf per
		// child holding that child's candidates
		pcg::Tree tree;
		tree.add("r", -1, pcg::Vec3d{box_min[0], box_min[1], box_min[2]}, pcg::Vec3d{box_max[0], box_max[1], box_max[2]});
		int64_t first = 0;
		for (int64_t i = 1; i <= n; i++) {
			if (i < n && child[i] == child[first]) continue;
			const int c = tree.child_of(0, child[first], 0);
			tree.nodes[c].leaf_start = first;
			tree.nodes[c].leaf_count = i - first;
			first = i;
		}
		pcg::ChunkingOut co{};
		co.X = mem.alloc<int32_t>(n);
		co.Y = mem.alloc<int32_t>(n);
		co.Z = mem.alloc<int32_t>(n);
		PCG_CUDA(cudaMemcpyAsync(co.X, X, n * 4, cudaMemcpyHostToDevice, stream));
		PCG_CUDA(cudaMemcpyAsync(co.Y, Y, n * 4, cudaMemcpyHostToDevice, stream));
		PCG_CUDA(cudaMemcpyAsync(co.Z, Z, n * 4, cudaMemcpyHostToDevice, stream));
		std::vector<uint32_t> iota((size_t)n);
		for (int64_t i = 0; i < n; i++) iota[i] = (uint32_t)i;
		uint32_t* d_ids = pcg::upload(iota, mem);
		uint64_t* d_cols = nullptr;
		if (method == PCG_POISSON_AVERAGE) {
			std::vector<uint64_t> cols((size_t)n);
			for (int64_t i = 0; i < n; i++)
				cols[i] = (uint64_t)rgb[3 * i] | (uint64_t)rgb[3 * i + 1] << 16 | (uint64_t)rgb[3 * i + 2] << 32;
			d_cols = pcg::upload(cols, mem);
		}
		int4* d_rec = nullptr;
		if (method != PCG_RANDOM) {
			d_rec = mem.alloc<int4>(n);
			pcg::launch_gather_records(d_ids, n, co.X, co.Y, co.Z, d_rec, mem);
		}
		for (auto& t : tree.nodes) {
			if (t.has_children()) continue;
			t.buf_ids = d_ids + t.leaf_start;
			t.buf_cols = d_cols ? d_cols + t.leaf_start : nullptr;
			t.buf_rec = d_rec ? d_rec + t.leaf_start : nullptr;
			t.buf_count = t.leaf_count;
		}
		pcg::SampleStats* d_st = mem.alloc<pcg::SampleStats>(1);
		PCG_CUDA(cudaMemsetAsync(d_st, 0, sizeof(pcg::SampleStats), stream));
		pcg::GreedyArena grid_arena;
		pcg::PosParamsS pps;
		for (int a = 0; a < 3; a++) { pps.scale[a] = scale[a]; pps.offset[a] = offset[a]; }
		pcg::JobResult res;
		uint64_t* level_cols = nullptr;
		ctx->conv.sample_level(tree, {0}, method, spacing, pps, co, d_st, grid_arena, mem, res, &level_cols);
		const pcg::TNode& root = tree.nodes[0];
		const auto acc = pcg::download(root.buf_ids, (size_t)root.buf_count, stream);
		if (pcg::download(d_st, 1, stream)[0].timeouts) throw pcg::PcgError(PCG_TIMEOUT, "a bounded device loop gave up");
		std::memset(accepted_out, 0, (size_t)n);
		for (uint32_t id : acc) accepted_out[id] = 1;
		if (method == PCG_POISSON_AVERAGE && rgb_out) {
			const auto cols = pcg::download(level_cols, (size_t)n, stream);
			for (int64_t i = 0; i < n; i++) {
				rgb_out[3 * i] = (uint16_t)(cols[i] & 0xffff);
				rgb_out[3 * i + 1] = (uint16_t)((cols[i] >> 16) & 0xffff);
				rgb_out[3 * i + 2] = (uint16_t)((cols[i] >> 32) & 0xffff);
			}
		}
	});
}

pcg_status pcg_kernel_laz_decode(pcg_ctx* ctx, const void* laz_file, uint64_t size, void* records_out, uint64_t out_size) {
	if (!ctx || !laz_file) return PCG_BAD_INPUT;
	std::lock_guard<std::mutex> lk(ctx->mtx);
	return guarded(ctx, [&] {
		pcg::LasInfo info;
		std::string err;
		if (!pcg::parse_las(static_cast<const uint8_t*>(laz_file), size, info, err)) throw pcg::PcgError(PCG_BAD_INPUT, err);
		if (!info.compressed) throw pcg::PcgError(PCG_BAD_INPUT, "not a LAZ file");
		const uint64_t bytes = (uint64_t)info.num_points * (uint64_t)info.record_length;
		if (out_size < bytes || (bytes && !records_out)) throw pcg::PcgError(PCG_BAD_INPUT, "records_out is too small");
		if (bytes == 0) return;
		PCG_CUDA(cudaSetDevice(ctx->conv.device));
		pcg::DeviceMem mem(ctx->conv.stream, ctx->conv.arena.get());
		const auto& chunks = info.laz_chunks;
		const uint64_t base = chunks.front().start, nbytes = chunks.back().end - base;
		uint8_t* d_laz = mem.alloc<uint8_t>(nbytes);
		uint8_t* d_out = mem.alloc<uint8_t>(bytes);
		PCG_CUDA(cudaMemcpyAsync(d_laz, static_cast<const uint8_t*>(laz_file) + base, nbytes, cudaMemcpyHostToDevice, mem.stream()));
		pcg::launch_laz_decode(d_laz, base, chunks, info.laz_layout, d_out, mem);
		PCG_CUDA(cudaMemcpyAsync(records_out, d_out, bytes, cudaMemcpyDeviceToHost, mem.stream()));
		PCG_CUDA(cudaStreamSynchronize(mem.stream()));
	});
}

}  // extern "C"
