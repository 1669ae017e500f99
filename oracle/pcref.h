// ORACLE -- test infrastructure only (see pcref.cpp).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace pcref {

struct NodeRecord {
	std::string name;
	int64_t byteOffset, byteSize, numPoints;
};

struct Result {
	std::vector<uint8_t> octree, hierarchy, metadata;
	std::vector<std::string> chunkIds;    // chunk (file-name) order
	std::vector<int64_t> chunkCounts;
	std::vector<NodeRecord> nodes;        // completion order
};

struct SourceImage {
	const uint8_t* las;
	size_t size;
};

// Converts one uncompressed LAS file image; method is "poisson",
// "poisson_average" or "random"; name goes to metadata.json; seed is the
// random sampler's pinned seed.
bool convert(const uint8_t* las, size_t size, const std::string& method, const std::string& name,
             uint32_t seed, Result& res, std::string& err);

// The counting pass alone for one LAS image: quantized X, Y, Z and the
// count-grid cell of every point, and the grid of counts (gridSize^3).
bool decodeCount(const uint8_t* las, size_t size, int32_t* X, int32_t* Y, int32_t* Z, uint32_t* cell, std::vector<int64_t>& grid,
                 int64_t& gridSize, std::string& err);

// Converts several LAS file images as one point cloud (the reference's
// source list, in order), keeping only the named attributes when
// attributes is not empty (--attributes).
bool convert(const std::vector<SourceImage>& sources, const std::vector<std::string>& attributes, const std::string& method,
             const std::string& name, uint32_t seed, Result& res, std::string& err);

}  // namespace pcref
