// Device-side helpers and host launchers shared by the CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
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

// Stream-ordered device allocations owned by one job.
class DeviceMem {
public:
	explicit DeviceMem(cudaStream_t s) : stream_(s) {}
	~DeviceMem() { release(); }
	DeviceMem(const DeviceMem&) = delete;
	DeviceMem& operator=(const DeviceMem&) = delete;
	template <class T> T* alloc(size_t count) {
		void* p = nullptr;
		size_t bytes = count * sizeof(T);
		if (bytes == 0) bytes = 16;
		bytes = (bytes + 255) & ~size_t(255);
		cudaError_t e = cudaMallocAsync(&p, bytes, stream_);
		if (e != cudaSuccess) {
			cudaGetLastError();
			throw PcgError(3, "device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
		}
		ptrs_.push_back(p);
		bytes_ += bytes;
		return static_cast<T*>(p);
	}
	void free(void* p) {
		for (size_t i = 0; i < ptrs_.size(); i++) {
			if (ptrs_[i] == p) {
				cudaFreeAsync(p, stream_);
				ptrs_[i] = ptrs_.back();
				ptrs_.pop_back();
				return;
			}
		}
	}
	void release() {
		for (void* p : ptrs_) cudaFreeAsync(p, stream_);
		ptrs_.clear();
	}
	size_t bytes() const { return bytes_; }
	cudaStream_t stream() const { return stream_; }

private:
	cudaStream_t stream_;
	std::vector<void*> ptrs_;
	size_t bytes_ = 0;
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
