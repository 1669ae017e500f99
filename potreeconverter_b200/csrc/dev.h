// Device-side helpers and host launchers shared by the CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <map>
#include <memory>
#include <unordered_map>
#include <stdexcept>
#include <string>
#include <vector>

#include "pcg_internal.h"

namespace pcg {

// Error raised by host code when a CUDA call fails; converted to a
// pcg_status at the C ABI.
struct CudaError : std::runtime_error {
	cudaError_t code;
	CudaError(cudaError_t c, const std::string& what) : std::runtime_error(what), code(c) {}
};

struct PcgError : std::runtime_error {
	int status;
	PcgError(int s, const std::string& what) : std::runtime_error(what), status(s) {}
};

#define PCG_CUDA(call)                                                                       \
	do {                                                                                     \
		cudaError_t e_ = (call);                                                             \
		if (e_ != cudaSuccess)                                                               \
			throw ::pcg::CudaError(e_, std::string(#call) + ": " + cudaGetErrorString(e_)); \
	} while (0)

// Launch bookkeeping: every kernel launch goes through PCG_LAUNCH so the
// number of launches per job is reported and launch errors surface at once.
extern thread_local int64_t g_launch_count;
#define PCG_LAUNCHED()                                                               \
	do {                                                                             \
		::pcg::g_launch_count++;                                                     \
		cudaError_t e_ = cudaGetLastError();                                          \
		if (e_ != cudaSuccess) throw ::pcg::CudaError(e_, std::string("launch: ") + cudaGetErrorString(e_)); \
	} while (0)

// Device memory cached for one stream across the levels of a job and
// across jobs: chunks of at least kArenaChunk bytes from the stream-ordered
// allocator, carved first-fit on the host. Everything that uses the memory
// runs on the arena's stream (or on a stream joined back to it before the
// memory is released), so a released range can be handed out again at once:
// later work on the stream runs after the work that used it. This keeps the
// driver out of the per-level allocations, whose occasional pool growth
// stalled the host for hundreds of milliseconds.
class DeviceArena {
public:
	static constexpr size_t kArenaChunk = size_t(2) << 30;
	explicit DeviceArena(cudaStream_t s) : stream_(s) {}
	~DeviceArena() {
		release_all();
		for (int k = 0; k < kSides; k++) {
			if (!side_[k]) continue;
			cudaStreamSynchronize(side_[k]);
			cudaStreamDestroy(side_[k]);
			cudaEventDestroy(fork_[k]);
			cudaEventDestroy(join_[k]);
		}
	}

	// Streams for work that runs beside the arena's stream (k < kSides), with
	// the events that fork each from and join it back to the arena's
	// stream; created once (stream creation can stall the host).
	static constexpr int kSides = 2;
	cudaStream_t side_stream(cudaEvent_t& fork, cudaEvent_t& join, int k = 0) {
		if (!side_[k]) {
			cudaError_t e = cudaStreamCreateWithFlags(&side_[k], cudaStreamNonBlocking);
			if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork_[k], cudaEventDisableTiming);
			if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join_[k], cudaEventDisableTiming);
			if (e != cudaSuccess) throw CudaError(e, std::string("side stream: ") + cudaGetErrorString(e));
		}
		fork = fork_[k];
		join = join_[k];
		return side_[k];
	}
	DeviceArena(const DeviceArena&) = delete;
	DeviceArena& operator=(const DeviceArena&) = delete;

	void* alloc(size_t bytes) {
		for (size_t ci = 0; ci < chunks_.size(); ci++) {
			void* p = take(ci, bytes);
			if (p) return p;
		}
		size_t size = bytes > kArenaChunk ? bytes : kArenaChunk;
		void* base = nullptr;
		cudaError_t e = cudaMallocAsync(&base, size, stream_);
		if (e != cudaSuccess && size > bytes) {
			cudaGetLastError();
			size = bytes;
			e = cudaMallocAsync(&base, size, stream_);
		}
		if (e != cudaSuccess) {
			cudaGetLastError();
			// give back chunks nobody uses and try once more
			trim();
			e = cudaMallocAsync(&base, size, stream_);
			if (e != cudaSuccess) {
				cudaGetLastError();
				throw PcgError(3, "device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
			}
		}
		Chunk c;
		c.base = static_cast<char*>(base);
		c.size = size;
		c.free[0] = size;
		chunks_.push_back(std::move(c));
		return take(chunks_.size() - 1, bytes);
	}

	void free(void* p) {
		auto it = live_.find(p);
		if (it == live_.end()) return;
		Chunk& c = chunks_[it->second.first];
		size_t off = static_cast<char*>(p) - c.base, len = it->second.second;
		live_.erase(it);
		live_bytes_ -= len;
		auto nx = c.free.lower_bound(off);
		if (nx != c.free.end() && off + len == nx->first) {  // merge with the next range
			len += nx->second;
			nx = c.free.erase(nx);
		}
		if (nx != c.free.begin()) {  // and with the previous one
			auto pv = std::prev(nx);
			if (pv->first + pv->second == off) {
				pv->second += len;
				return;
			}
		}
		c.free[off] = len;
	}

	// frees the chunks that hold no live range
	void trim() {
		std::vector<Chunk> keep;
		std::vector<size_t> remap(chunks_.size());
		for (size_t i = 0; i < chunks_.size(); i++) {
			Chunk& c = chunks_[i];
			if (c.free.size() == 1 && c.free.begin()->first == 0 && c.free.begin()->second == c.size) {
				cudaFreeAsync(c.base, stream_);
				remap[i] = SIZE_MAX;
			} else {
				remap[i] = keep.size();
				keep.push_back(std::move(c));
			}
		}
		for (auto& kv : live_) kv.second.first = remap[kv.second.first];
		chunks_ = std::move(keep);
	}

	void release_all() {
		for (Chunk& c : chunks_) cudaFreeAsync(c.base, stream_);
		chunks_.clear();
		live_.clear();
		live_bytes_ = 0;
	}

	size_t reserved() const {
		size_t r = 0;
		for (const Chunk& c : chunks_) r += c.size;
		return r;
	}
	// bytes handed out and not yet freed, and their high-water mark since
	// the last reset_peak()
	size_t live_bytes() const { return live_bytes_; }
	size_t peak_bytes() const { return peak_bytes_; }
	void reset_peak() { peak_bytes_ = live_bytes_; }
	cudaStream_t stream() const { return stream_; }

private:
	struct Chunk {
		char* base = nullptr;
		size_t size = 0;
		std::map<size_t, size_t> free;  // offset -> length
	};

	void* take(size_t ci, size_t bytes) {
		Chunk& c = chunks_[ci];
		for (auto it = c.free.begin(); it != c.free.end(); ++it) {
			if (it->second < bytes) continue;
			const size_t off = it->first, len = it->second;
			c.free.erase(it);
			if (len > bytes) c.free[off + bytes] = len - bytes;
			void* p = c.base + off;
			live_[p] = {ci, bytes};
			live_bytes_ += bytes;
			if (live_bytes_ > peak_bytes_) peak_bytes_ = live_bytes_;
			return p;
		}
		return nullptr;
	}

	cudaStream_t stream_;
	cudaStream_t side_[kSides] = {nullptr, nullptr};
	cudaEvent_t fork_[kSides] = {nullptr, nullptr}, join_[kSides] = {nullptr, nullptr};
	std::vector<Chunk> chunks_;
	std::unordered_map<void*, std::pair<size_t, size_t>> live_;  // range -> (chunk, length)
	size_t live_bytes_ = 0, peak_bytes_ = 0;
};

// Stream-ordered device allocations owned by one job, from an arena when the
// job has one, else straight from the stream-ordered allocator.
class DeviceMem {
public:
	explicit DeviceMem(cudaStream_t s, DeviceArena* arena = nullptr) : stream_(s), arena_(arena) {}
	~DeviceMem() { release(); }
	DeviceMem(const DeviceMem&) = delete;
	DeviceMem& operator=(const DeviceMem&) = delete;
	template <class T> T* alloc(size_t count) {
		void* p = nullptr;
		size_t bytes = count * sizeof(T);
		if (bytes == 0) bytes = 16;
		bytes = (bytes + 255) & ~size_t(255);
		const auto t0 = std::chrono::steady_clock::now();
		if (arena_) {
			p = arena_->alloc(bytes);
		} else {
			cudaError_t e = cudaMallocAsync(&p, bytes, stream_);
			if (e != cudaSuccess) {
				cudaGetLastError();
				throw PcgError(3, "device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
			}
		}
		alloc_ms_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
		ptrs_.push_back(p);
		bytes_ += bytes;
		return static_cast<T*>(p);
	}
	void free(void* p) {
		for (size_t i = 0; i < ptrs_.size(); i++) {
			if (ptrs_[i] == p) {
				give_back(p);
				ptrs_[i] = ptrs_.back();
				ptrs_.pop_back();
				return;
			}
		}
	}
	void release() {
		for (void* p : ptrs_) give_back(p);
		ptrs_.clear();
	}
	size_t bytes() const { return bytes_; }
	double alloc_ms() const { return alloc_ms_; }  // host time spent allocating
	cudaStream_t stream() const { return stream_; }
	DeviceArena* arena() const { return arena_; }

private:
	void give_back(void* p) {
		if (arena_) arena_->free(p);
		else cudaFreeAsync(p, stream_);
	}
	cudaStream_t stream_;
	DeviceArena* arena_;
	std::vector<void*> ptrs_;
	size_t bytes_ = 0;
	double alloc_ms_ = 0;
};

// ---------------------------------------------------------------- launchers
// Stable LSD radix sort of (key, value) uint32 pairs on bits [begin_bit,
// end_bit). The sorted pairs end in (keys, vals); tmp buffers are scratch of
// the same length.
void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp, int64_t n,
                      int begin_bit, int end_bit, DeviceMem& mem);

// out[i] = sum(in[0..i)) ; returns nothing, total is out[n] when out has n+1
// elements and write_total is set.
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, bool write_total, DeviceMem& mem);
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, bool write_total, DeviceMem& mem);

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

inline int bits_for(uint64_t v) {  // bits needed to represent values 0..v
	int b = 0;
	while ((v >> b) != 0) b++;
	return b;
}

}  // namespace pcg
