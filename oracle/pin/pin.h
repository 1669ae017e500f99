// Determinism pins for the reference build that serves as the parity oracle.
//
// This header is force-included (g++ -include) into every PotreeConverter
// translation unit of the *pinned* oracle binary. It changes no arithmetic of
// the converter; it only removes the run-to-run freedom the stock binary has:
//
//   1. every TaskPool runs exactly one worker, so chunk files are appended in
//      batch order and chunks are indexed one after another
//      (chunker_countsort_laszip.cpp:277,937; indexer.cpp:1638);
//   2. std::thread::hardware_concurrency() reports 1, which pins the chunk
//      writer's flush threads (chunker_countsort_laszip.cpp:44-45);
//   3. directory iteration yields entries sorted by file name, so chunk order
//      (indexer.cpp:149) and hierarchy batch order (HierarchyBuilder.h:302)
//      are pure functions of the input;
//   4. the random sampler's clock seed (sampler_random.h:102) reads a fixed
//      value, PIN_RANDOM_SEED, instead of the wall clock.
//
// The header must be included before any reference header so that the
// standard library is fully parsed before the macros below are defined.
#pragma once

#include <bits/stdc++.h>

// TaskPool.hpp expects std::shared_ptr to be visible unqualified, as the
// reference headers that normally precede it arrange.
using std::shared_ptr;
#include "unsuck/TaskPool.hpp"

#ifndef PIN_RANDOM_SEED
#define PIN_RANDOM_SEED 1592614637ll /* 0x5EED5EED */
#endif

template <class T>
class PinnedSerialTaskPool : public TaskPool<T> {
public:
	PinnedSerialTaskPool(size_t /*requestedThreads*/, typename TaskPool<T>::TaskProcessorType processor)
		: TaskPool<T>(1, processor) {}
};

namespace std::filesystem {
inline std::vector<directory_entry> pin_sorted_directory(const path& dir) {
	std::vector<directory_entry> entries;
	for (directory_iterator it(dir), end; it != end; ++it) {
		entries.push_back(*it);
	}
	std::sort(entries.begin(), entries.end(), [](const directory_entry& a, const directory_entry& b) {
		return a.path().filename().string() < b.path().filename().string();
	});
	return entries;
}
}  // namespace std::filesystem

namespace std::chrono {
struct pin_seed_clock {
	using duration = std::chrono::nanoseconds;
	using rep = duration::rep;
	using period = duration::period;
	using time_point = std::chrono::time_point<pin_seed_clock, duration>;
	static constexpr bool is_steady = false;
	static time_point now() noexcept { return time_point(duration(PIN_RANDOM_SEED)); }
};
}  // namespace std::chrono

#define TaskPool PinnedSerialTaskPool
#define hardware_concurrency() hardware_concurrency() * 0 + 1
#define directory_iterator(p) pin_sorted_directory(p)
#define system_clock pin_seed_clock
