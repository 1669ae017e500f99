// Host writers for hierarchy.bin and metadata.json.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "pcg_internal.h"

namespace pcg {

// One completed node as the reference's HierarchyFlusher records it
// (indexer.h:146-162): name, byte offset/size in octree.bin, point count.
struct HierRecord {
	std::string name;
	int64_t byte_offset = 0;
	int64_t byte_size = 0;
	int64_t num_points = 0;
};

// Serializes hierarchy.bin from records in completion order with the
// batch/chunk layout of HierarchyFlusher (indexer.h:171-243) and
// HierarchyBuilder (HierarchyBuilder.h:82-352). Returns the root batch size
// (metadata "firstChunkSize").
bool build_hierarchy(const std::vector<HierRecord>& completed, std::vector<uint8_t>& out,
                     int64_t& first_chunk_size, std::string& err);

// metadata.json text, Indexer::createMetadata (indexer.cpp:354-524).
struct AttrStats {
	Vec3d min, max;
	std::vector<int64_t> histogram;  // 256 bins, classification only
};

std::string build_metadata(const std::string& name, const std::string& projection, int64_t points_total,
                           int64_t first_chunk_size, int64_t depth, const Setup& s,
                           const std::vector<AttrStats>& stats, double spacing);

}  // namespace pcg
