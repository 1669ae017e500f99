// ORACLE -- test infrastructure only.
//
// A single-threaded, in-memory CPU restatement of PotreeConverter 2.0's
// LAS -> octree LOD build (chunking, indexing, the three samplers and the
// octree.bin / hierarchy.bin / metadata.json writers). It is the checker for
// the CUDA path: only tests, the smoke check and the benchmark's CPU-baseline
// leg may load it. It is pinned against the reference binary built by
// oracle/Makefile (PotreeConverter_pinned) through tests/golden.
//
// Determinism pins, identical to oracle/pin/pin.h: one worker thread, chunks
// and hierarchy batches taken in file-name order, and the random sampler
// seeded with a fixed value instead of the clock.
//
// Every function cites the reference file:line it restates (paths relative
// to the PotreeConverter source tree). std::sort and std::shuffle are called
// exactly as the reference calls them, so tie order and the shuffle sequence
// come from the same libstdc++ the reference links.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <iomanip>
#include <limits>
#include <map>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "pcref.h"

namespace pcref {

using std::function;
using std::make_shared;
using std::shared_ptr;
using std::string;
using std::stringstream;
using std::vector;

static const double Inf = std::numeric_limits<double>::infinity();

// ---------------------------------------------------------------- Vector3.h
struct Vec3 {
	double x = 0.0, y = 0.0, z = 0.0;
	Vec3() {}
	Vec3(double x, double y, double z) : x(x), y(y), z(z) {}
	double max() const { return std::max(std::max(x, y), z); }
	Vec3 operator-(const Vec3& r) const { return Vec3(x - r.x, y - r.y, z - r.z); }
	Vec3 operator+(const Vec3& r) const { return Vec3(x + r.x, y + r.y, z + r.z); }
	Vec3 operator+(double s) const { return Vec3(x + s, y + s, z + s); }
	Vec3 operator*(double s) const { return Vec3(x * s, y * s, z * s); }
};

// ------------------------------------------------------------- Attributes.h
enum class AType { INT8 = 0, INT16 = 1, INT32 = 2, INT64 = 3, UINT8 = 10, UINT16 = 11, UINT32 = 12, UINT64 = 13, FLOAT = 20, DOUBLE = 21, UNDEFINED = 123456 };

static int typeSize(AType t) {  // Attributes.h:33-49
	switch (t) {
	case AType::UINT8: case AType::INT8: return 1;
	case AType::UINT16: case AType::INT16: return 2;
	case AType::UINT32: case AType::INT32: case AType::FLOAT: return 4;
	case AType::UINT64: case AType::INT64: case AType::DOUBLE: return 8;
	default: return 0;
	}
}

static string typeName(AType t) {  // Attributes.h:51-78
	switch (t) {
	case AType::INT8: return "int8"; case AType::INT16: return "int16";
	case AType::INT32: return "int32"; case AType::INT64: return "int64";
	case AType::UINT8: return "uint8"; case AType::UINT16: return "uint16";
	case AType::UINT32: return "uint32"; case AType::UINT64: return "uint64";
	case AType::FLOAT: return "float"; case AType::DOUBLE: return "double";
	case AType::UNDEFINED: return "undefined";
	}
	return "error";
}

struct Attribute {  // Attributes.h:109-139
	string name, description;
	int size = 0, numElements = 0, elementSize = 0;
	AType type = AType::UNDEFINED;
	Vec3 min = {Inf, Inf, Inf};
	Vec3 max = {-Inf, -Inf, -Inf};
	Vec3 scale = {1.0, 1.0, 1.0};
	Vec3 offset = {0.0, 0.0, 0.0};
	vector<int64_t> histogram = vector<int64_t>(256, 0);
	Attribute() {}
	Attribute(string n, int s, int ne, int es, AType t) : name(n), size(s), numElements(ne), elementSize(es), type(t) {}
};

struct Attributes {  // Attributes.h:141-186
	vector<Attribute> list;
	int bytes = 0;
	Vec3 posScale = {1.0, 1.0, 1.0};
	Vec3 posOffset = {0.0, 0.0, 0.0};
	Attributes() {}
	explicit Attributes(vector<Attribute> a) : list(a) { for (auto& x : a) bytes += x.size; }
	int getOffset(const string& name) const {
		int off = 0;
		for (auto& a : list) { if (a.name == name) return off; off += a.size; }
		return -1;
	}
	Attribute* get(const string& name) {
		for (auto& a : list) if (a.name == name) return &a;
		return nullptr;
	}
};

// ------------------------------------------------------------ LAS header
// Raw LAS header fields as LASzip exposes them for uncompressed files
// (LasLoader.cpp:72-128; laszip_dll.cpp header reader).
struct LasHeader {
	Vec3 min, max, scale, offset;
	int64_t numPoints = 0;
	int pointDataFormat = -1;
	int recordLength = 0;
	uint64_t offsetToPoints = 0;
	struct VLR { uint16_t recordID; vector<uint8_t> data; };
	vector<VLR> vlrs;
};

template <class T> static T rd(const uint8_t* p) { T v; memcpy(&v, p, sizeof(T)); return v; }

static bool parseHeader(const uint8_t* las, size_t size, LasHeader& h, string& err) {
	if (size < 227 || memcmp(las, "LASF", 4) != 0) { err = "not a LAS file"; return false; }
	int versionMinor = las[25];
	uint16_t headerSize = rd<uint16_t>(las + 94);
	h.offsetToPoints = rd<uint32_t>(las + 96);
	uint32_t numVlrs = rd<uint32_t>(las + 100);
	h.pointDataFormat = las[104] & 0x3f;
	h.recordLength = rd<uint16_t>(las + 105);
	uint64_t legacyCount = rd<uint32_t>(las + 107);
	h.scale = Vec3(rd<double>(las + 131), rd<double>(las + 139), rd<double>(las + 147));
	h.offset = Vec3(rd<double>(las + 155), rd<double>(las + 163), rd<double>(las + 171));
	h.max.x = rd<double>(las + 179); h.min.x = rd<double>(las + 187);
	h.max.y = rd<double>(las + 195); h.min.y = rd<double>(las + 203);
	h.max.z = rd<double>(las + 211); h.min.z = rd<double>(las + 219);
	uint64_t extCount = 0;
	if (versionMinor >= 4 && headerSize >= 375 && size >= 255) extCount = rd<uint64_t>(las + 247);
	h.numPoints = (int64_t)std::max(extCount, legacyCount);  // LasLoader.cpp:103
	size_t pos = headerSize;
	for (uint32_t i = 0; i < numVlrs; i++) {
		if (pos + 54 > size) { err = "truncated VLR"; return false; }
		LasHeader::VLR v;
		v.recordID = rd<uint16_t>(las + pos + 18);
		uint16_t len = rd<uint16_t>(las + pos + 20);
		if (pos + 54 + len > size) { err = "truncated VLR"; return false; }
		v.data.assign(las + pos + 54, las + pos + 54 + len);
		h.vlrs.push_back(v);
		pos += 54 + len;
	}
	if (h.offsetToPoints + (uint64_t)h.numPoints * h.recordLength > size) { err = "truncated point data"; return false; }
	return true;
}

static void lasTypeInfo(int typeID, AType& type, int& numElements) {  // LasLoader.cpp:7-69
	static const AType base[] = {AType::UNDEFINED, AType::UINT8, AType::INT8, AType::UINT16, AType::INT16, AType::UINT32, AType::INT32, AType::UINT64, AType::INT64, AType::FLOAT, AType::DOUBLE};
	if (typeID == 0) { type = AType::UNDEFINED; numElements = 1; return; }
	int k = (typeID - 1) % 10 + 1;
	type = base[k];
	numElements = typeID <= 10 ? 1 : (typeID <= 20 ? 2 : 3);
}

static vector<Attribute> parseExtraAttributes(const LasHeader& header) {  // PotreeConverter.h:80-133
	vector<Attribute> attributes;
	for (auto& vlr : header.vlrs) {
		if (vlr.recordID != 4) continue;
		int num = (int)vlr.data.size() / 192;
		for (int i = 0; i < num; i++) {
			const uint8_t* r = vlr.data.data() + i * 192;
			uint8_t type = r[2], options = r[3];
			char chrName[33] = {0}; memcpy(chrName, r + 4, 32);
			Vec3 aScale(1, 1, 1), aOffset(0, 0, 0);
			if (options & 0b01000) memcpy(&aScale, r + 112, 24);
			if (options & 0b10000) memcpy(&aOffset, r + 136, 24);
			char chrDesc[33] = {0}; memcpy(chrDesc, r + 160, 32);
			AType t; int ne; lasTypeInfo(type, t, ne);
			int es = typeSize(t);
			Attribute a(string(chrName), ne * es, ne, es, t);
			a.description = string(chrDesc);
			a.scale = aScale; a.offset = aOffset;
			attributes.push_back(a);
		}
	}
	return attributes;
}

static bool outputAttributesOf(const LasHeader& header, vector<Attribute>& list) {  // PotreeConverter.h:136-193
	Attribute xyz("position", 12, 3, 4, AType::INT32);
	Attribute intensity("intensity", 2, 1, 2, AType::UINT16);
	Attribute returnNumber("return number", 1, 1, 1, AType::UINT8);
	Attribute numberOfReturns("number of returns", 1, 1, 1, AType::UINT8);
	Attribute classification("classification", 1, 1, 1, AType::UINT8);
	Attribute scanAngleRank("scan angle rank", 1, 1, 1, AType::UINT8);
	Attribute userData("user data", 1, 1, 1, AType::UINT8);
	Attribute pointSourceId("point source id", 2, 1, 2, AType::UINT16);
	Attribute gpsTime("gps-time", 8, 1, 8, AType::DOUBLE);
	Attribute rgb("rgb", 6, 3, 2, AType::UINT16);
	int f = header.pointDataFormat;
	if (f == 0) list = {xyz, intensity, returnNumber, numberOfReturns, classification, scanAngleRank, userData, pointSourceId};
	else if (f == 1) list = {xyz, intensity, returnNumber, numberOfReturns, classification, scanAngleRank, userData, pointSourceId, gpsTime};
	else if (f == 2) list = {xyz, intensity, returnNumber, numberOfReturns, classification, scanAngleRank, userData, pointSourceId, rgb};
	else if (f == 3) list = {xyz, intensity, returnNumber, numberOfReturns, classification, scanAngleRank, userData, pointSourceId, gpsTime, rgb};
	else return false;  // formats 4-10 are not restated
	auto extra = parseExtraAttributes(header);
	list.insert(list.end(), extra.begin(), extra.end());
	return true;
}

// ------------------------------------------------------------- the job
struct Source {  // one input file (main.cpp:146-200 Source)
	const uint8_t* las = nullptr;
	LasHeader header;
	vector<Attribute> list;  // its own attribute list, PotreeConverter.h:136-193
};

struct Job {
	vector<Source> sources;     // in the order the reference takes them
	vector<string> requested;   // --attributes (empty: all)
	Attributes attributes;      // output attributes incl. scale/offset
	Vec3 min, max;              // cubic box, main.cpp:237-239
	int64_t totalPoints = 0;
	string name;
	string method;
	uint32_t seed = 0;
	string err;
};

static bool setup(Job& job) {
	// computeOutputAttributes(sources, requestedAttributes), PotreeConverter.h:195-276
	Vec3 scaleMin(Inf, Inf, Inf), min(Inf, Inf, Inf), max(-Inf, -Inf, -Inf);
	vector<Attribute> full;
	for (auto& src : job.sources) {
		if (!outputAttributesOf(src.header, src.list)) { job.err = "unsupported point format"; return false; }
		for (auto& a : src.list) {
			bool added = false;
			for (auto& f : full) added = added || f.name == a.name;
			if (!added) full.push_back(a);
		}
		const LasHeader& h = src.header;
		scaleMin.x = std::min(scaleMin.x, h.scale.x); scaleMin.y = std::min(scaleMin.y, h.scale.y); scaleMin.z = std::min(scaleMin.z, h.scale.z);
		min.x = std::min(min.x, h.min.x); min.y = std::min(min.y, h.min.y); min.z = std::min(min.z, h.min.z);
		max.x = std::max(max.x, h.max.x); max.y = std::max(max.y, h.max.y); max.z = std::max(max.z, h.max.z);
		job.totalPoints += h.numPoints;
	}
	// computeScaleOffset, PotreeConverter.h:29-76
	Vec3 size = max - min;
	double msx = size.x / pow(2.0, 30.0), msy = size.y / pow(2.0, 30.0), msz = size.z / pow(2.0, 30.0);
	Vec3 scale(std::max(scaleMin.x, msx), std::max(scaleMin.y, msy), std::max(scaleMin.z, msz));
	// the filter, PotreeConverter.h:252-275: position first, then the
	// requested names found in the full list, in request order
	vector<Attribute> filtered = full;
	if (!job.requested.empty()) {
		vector<string> should = job.requested;
		should.insert(should.begin(), "position");
		filtered.clear();
		for (auto& nm : should)
			for (auto& f : full)
				if (f.name == nm) { filtered.push_back(f); break; }
	}
	job.attributes = Attributes(filtered);
	job.attributes.posScale = scale;
	job.attributes.posOffset = min;
	// computeStats, main.cpp:215-284 (the same header boxes)
	double cubeSize = (max - min).max();
	Vec3 csize(cubeSize, cubeSize, cubeSize);
	job.min = min;
	job.max = min + cubeSize;
	if (csize.x == 0.0 || csize.y == 0.0 || csize.z == 0) { job.err = "invalid bounding box"; return false; }
	return true;
}

// ---------------------------------------------------------------- chunker
struct ChunkNode { string id; int64_t level = 0, x = 0, y = 0, z = 0, size = 0, numPoints = 0; };

static string toNodeID(int level, int gridSize, int64_t x, int64_t y, int64_t z) {  // chunker_countsort_laszip.cpp:82-115
	string id = "r";
	int cur = gridSize;
	int lx = (int)x, ly = (int)y, lz = (int)z;
	for (int i = 0; i < level; i++) {
		int index = 0;
		if (lx >= cur / 2) { index += 0b100; lx -= cur / 2; }
		if (ly >= cur / 2) { index += 0b010; ly -= cur / 2; }
		if (lz >= cur / 2) { index += 0b001; lz -= cur / 2; }
		id += std::to_string(index);
		cur /= 2;
	}
	return id;
}

struct PointCoord { double x, y, z; };

static inline const uint8_t* lasRecord(const Source& src, int64_t i) {
	return src.las + src.header.offsetToPoints + (uint64_t)i * src.header.recordLength;
}

static inline PointCoord lasCoordinates(const Source& src, int64_t i) {  // laszip_dll.cpp:1137-1139
	const uint8_t* r = lasRecord(src, i);
	const LasHeader& h = src.header;
	int32_t X = rd<int32_t>(r), Y = rd<int32_t>(r + 4), Z = rd<int32_t>(r + 8);
	return {h.scale.x * X + h.offset.x, h.scale.y * Y + h.offset.y, h.scale.z * Z + h.offset.z};
}

struct Chunk { string id; Vec3 min, max; vector<uint8_t> data; };

static void createLUT(const vector<int64_t>& grid, int64_t gridSize, int64_t maxPointsPerChunk, vector<ChunkNode>& nodes,
                      vector<int32_t>& lut) {  // chunker_countsort_laszip.cpp:1074-1204
	nodes.clear();
	lut.assign(gridSize * gridSize * gridSize, -1);
	vector<int64_t> gridHigh = grid;
	int64_t levelMax = int64_t(log2(gridSize));
	for (int64_t levelLow = levelMax - 1; levelLow >= 0; levelLow--) {
		int64_t levelHigh = levelLow + 1;
		int64_t gH = int64_t(pow(2, levelHigh)), gL = int64_t(pow(2, levelLow));
		vector<int64_t> gridLow(gL * gL * gL, 0);
		for (int64_t x = 0; x < gL; x++) for (int64_t y = 0; y < gL; y++) for (int64_t z = 0; z < gL; z++) {
			int64_t indexLow = x + y * gL + z * gL * gL;
			int64_t sum = 0; bool unmergeable = false;
			for (int64_t j = 0; j < 8; j++) {
				int64_t nx = 2 * x + ((j & 4) >> 2), ny = 2 * y + ((j & 2) >> 1), nz = 2 * z + (j & 1);
				int64_t v = gridHigh[nx + ny * gH + nz * gH * gH];
				if (v == -1) unmergeable = true; else sum += v;
			}
			if (unmergeable || sum > maxPointsPerChunk) {
				for (int64_t j = 0; j < 8; j++) {
					int64_t nx = 2 * x + ((j & 4) >> 2), ny = 2 * y + ((j & 2) >> 1), nz = 2 * z + (j & 1);
					int64_t v = gridHigh[nx + ny * gH + nz * gH * gH];
					if (v > 0) {
						ChunkNode n;
						n.id = toNodeID((int)levelHigh, (int)gH, nx, ny, nz);
						n.numPoints = v; n.x = nx; n.y = ny; n.z = nz;
						n.size = int64_t(pow(2, levelMax - levelHigh));
						nodes.push_back(n);
					}
				}
				gridLow[indexLow] = -1;
			} else {
				gridLow[indexLow] = sum;
			}
		}
		gridHigh = gridLow;
	}
	for (int i = 0; i < (int)nodes.size(); i++) {
		auto& n = nodes[i];
		for (int64_t ox = 0; ox < n.size; ox++) for (int64_t oy = 0; oy < n.size; oy++) for (int64_t oz = 0; oz < n.size; oz++) {
			int64_t x = n.size * n.x + ox, y = n.size * n.y + oy, z = n.size * n.z + oz;
			lut[x + y * gridSize + z * gridSize * gridSize] = i;
		}
	}
}

static bool doChunking(Job& job, vector<Chunk>& chunksOut, Attributes& attrsOut, Vec3& minOut, Vec3& maxOut) {
	// chunker_countsort_laszip.cpp:1206-1261
	int64_t total = job.totalPoints;
	int64_t tmp = total / 20;
	int maxPointsPerChunk = (int)std::min(tmp, int64_t(10'000'000));
	int64_t gridSize = total < 100'000'000 ? 128 : (total < 500'000'000 ? 256 : 512);
	Attributes& out = job.attributes;
	Vec3 min = job.min, max = job.max;
	Vec3 posScale = out.posScale, posOffset = out.posOffset;

	// countPointsInCells, :131-361
	vector<int64_t> grid(gridSize * gridSize * gridSize, 0);
	{
		double cubeSize = (max - min).max();
		Vec3 size(cubeSize, cubeSize, cubeSize);
		double dG = double(gridSize);
		for (auto& src : job.sources) for (int64_t i = 0; i < src.header.numPoints; i++) {
			PointCoord c = lasCoordinates(src, i);
			int32_t X = int32_t((c.x - posOffset.x) / posScale.x);
			int32_t Y = int32_t((c.y - posOffset.y) / posScale.y);
			int32_t Z = int32_t((c.z - posOffset.z) / posScale.z);
			double ux = (double(X) * posScale.x + posOffset.x - min.x) / size.x;
			double uy = (double(Y) * posScale.y + posOffset.y - min.y) / size.y;
			double uz = (double(Z) * posScale.z + posOffset.z - min.z) / size.z;
			bool inBox = ux >= 0.0 && uy >= 0.0 && uz >= 0.0 && ux <= 1.0 && uy <= 1.0 && uz <= 1.0;
			if (!inBox) { job.err = "point outside bounding box"; return false; }
			int64_t ix = int64_t(std::min(dG * ux, dG - 1.0));
			int64_t iy = int64_t(std::min(dG * uy, dG - 1.0));
			int64_t iz = int64_t(std::min(dG * uz, dG - 1.0));
			grid[ix + iy * gridSize + iz * gridSize * gridSize]++;
		}
	}

	// createLUT, :1074-1204
	vector<ChunkNode> nodes;
	vector<int32_t> lut;
	createLUT(grid, gridSize, maxPointsPerChunk, nodes, lut);

	// distributePoints, :660-1003 (handlers :380-658), one batch thread,
	// sources in order
	int bpp = out.bytes;
	vector<vector<uint8_t>> buckets(nodes.size());
	Attributes stats = out;  // global min/max/histogram accumulator
	for (auto& a : stats.list) { a.min = {Inf, Inf, Inf}; a.max = {-Inf, -Inf, -Inf}; for (auto& h : a.histogram) h = 0; }
	static const char* standard[] = {"rgb", "intensity", "return number", "number of returns", "classification", "scan angle rank",
	                                 "scan angle", "user data", "point source id", "gps-time", "classification flags"};
	for (auto& src : job.sources) {
		int fmt = src.header.pointDataFormat;
		// the handlers of createAttributeHandlers for this source's own
		// attribute list (the input list, :952-983)
		const vector<Attribute>& inList = src.list;
		vector<string> handled;  // standard handlers, in input-list order (:531-545)
		for (auto& ia : inList) {
			if (ia.name == "position") continue;
			bool mapped = false;
			for (const char* sn : standard) mapped = mapped || ia.name == sn;
			if (mapped && out.get(ia.name) != nullptr) handled.push_back(ia.name);
		}
		int firstExtraIndex = (fmt == 0) ? 8 : (fmt == 1 || fmt == 2) ? 9 : 10;  // :551-560 (formats 0-3)
		int stdRecLen = (fmt == 0) ? 20 : (fmt == 1) ? 28 : (fmt == 2) ? 26 : 34;
		struct ExtraHandler { int attributeOffset, sourceOffset, size; string name; };
		vector<ExtraHandler> extraHandlers;  // :579-653: the target offset is counted over the input list
		{
			int attributeOffset = 0;
			for (int k = 0; k < firstExtraIndex && k < (int)inList.size(); k++) attributeOffset += inList[k].size;
			int sourceOffset = 0;
			for (int k = firstExtraIndex; k < (int)inList.size(); k++) {
				const Attribute* oa = out.get(inList[k].name);
				if (oa) {
					if (attributeOffset + inList[k].size > bpp) { job.err = "extra attribute written past the point record (undefined in the reference)"; return false; }
					if (stdRecLen + sourceOffset + oa->numElements * oa->elementSize > src.header.recordLength) { job.err = "extra attribute read past the LAS record (undefined in the reference)"; return false; }
					extraHandlers.push_back({attributeOffset, sourceOffset, inList[k].size, inList[k].name});
					attributeOffset += oa->size;
				}
				sourceOffset += inList[k].size;
			}
		}
		double cubeSize = (max - min).max();
		Vec3 size(cubeSize, cubeSize, cubeSize);
		double dG = double(gridSize);
		vector<uint8_t> rec(bpp);
		for (int64_t i = 0; i < src.header.numPoints; i++) {
			const uint8_t* r = lasRecord(src, i);
			std::fill(rec.begin(), rec.end(), 0);
			PointCoord c = lasCoordinates(src, i);
			int32_t X = int32_t((c.x - posOffset.x) / posScale.x);
			int32_t Y = int32_t((c.y - posOffset.y) / posScale.y);
			int32_t Z = int32_t((c.z - posOffset.z) / posScale.z);
			memcpy(&rec[0], &X, 4); memcpy(&rec[4], &Y, 4); memcpy(&rec[8], &Z, 4);
			Attribute* aPos = stats.get("position");
			aPos->min.x = std::min(aPos->min.x, c.x); aPos->min.y = std::min(aPos->min.y, c.y); aPos->min.z = std::min(aPos->min.z, c.z);
			aPos->max.x = std::max(aPos->max.x, c.x); aPos->max.y = std::max(aPos->max.y, c.y); aPos->max.z = std::max(aPos->max.z, c.z);
			for (const string& nm : handled) {
				int off = out.getOffset(nm);
				Attribute* a = stats.get(nm);
				auto upd = [a](double v) { a->min.x = std::min(a->min.x, v); a->max.x = std::max(a->max.x, v); };
				if (nm == "intensity") { uint16_t v = rd<uint16_t>(r + 12); memcpy(&rec[off], &v, 2); upd(double(v)); }
				else if (nm == "return number") { uint8_t v = r[14] & 7; rec[off] = v; upd(double(v)); }
				else if (nm == "number of returns") { uint8_t v = (r[14] >> 3) & 7; rec[off] = v; upd(double(v)); }
				else if (nm == "classification") { uint8_t v = r[15] & 31; rec[off] = v; a->histogram[v]++; upd(double(v)); }
				else if (nm == "scan angle rank") { int8_t v = (int8_t)r[16]; memcpy(&rec[off], &v, 1); upd(double(v)); }
				else if (nm == "user data") { uint8_t v = r[17]; rec[off] = v; upd(double(v)); }
				else if (nm == "point source id") { uint16_t v = rd<uint16_t>(r + 18); memcpy(&rec[off], &v, 2); upd(double(v)); }
				else if (nm == "gps-time") { double v = rd<double>(r + 20); memcpy(&rec[off], &v, 8); upd(v); }
				else if (nm == "rgb") {
					int ro = (fmt == 2) ? 20 : 28;
					uint16_t c3[3] = {rd<uint16_t>(r + ro), rd<uint16_t>(r + ro + 2), rd<uint16_t>(r + ro + 4)};
					memcpy(&rec[off], c3, 6);
					a->min.x = std::min(a->min.x, double(c3[0])); a->min.y = std::min(a->min.y, double(c3[1])); a->min.z = std::min(a->min.z, double(c3[2]));
					a->max.x = std::max(a->max.x, double(c3[0])); a->max.y = std::max(a->max.y, double(c3[1])); a->max.z = std::max(a->max.z, double(c3[2]));
				}
			}
			const uint8_t* extra = r + stdRecLen;
			for (auto& eh : extraHandlers) {
				Attribute* a = stats.get(eh.name);
				memcpy(&rec[eh.attributeOffset], extra + eh.sourceOffset, eh.size);
				auto f = [a](const uint8_t* p) -> double {
					switch (a->type) {
					case AType::INT8: return double(rd<int8_t>(p)); case AType::INT16: return double(rd<int16_t>(p));
					case AType::INT32: return double(rd<int32_t>(p)); case AType::INT64: return double(rd<int64_t>(p));
					case AType::UINT8: return double(rd<uint8_t>(p)); case AType::UINT16: return double(rd<uint16_t>(p));
					case AType::UINT32: return double(rd<uint32_t>(p)); case AType::UINT64: return double(rd<uint64_t>(p));
					case AType::FLOAT: return double(rd<float>(p)); case AType::DOUBLE: return rd<double>(p);
					default: return 0.0;
					}
				};
				const uint8_t* q = extra + eh.sourceOffset;
				if (a->numElements == 1) { double x = f(q); a->min.x = std::min(a->min.x, x); a->max.x = std::max(a->max.x, x); }
				else if (a->numElements == 2) {
					double x = f(q), y = f(q + a->elementSize);
					a->min.x = std::min(a->min.x, x); a->min.y = std::min(a->min.y, y); a->max.x = std::max(a->max.x, x); a->max.y = std::max(a->max.y, y);
				} else if (a->numElements == 3) {
					double x = f(q), y = f(q + a->elementSize), z = f(q + 2 * a->elementSize);
					a->min.x = std::min(a->min.x, x); a->min.y = std::min(a->min.y, y); a->min.z = std::min(a->min.z, z);
					a->max.x = std::max(a->max.x, x); a->max.y = std::max(a->max.y, y); a->max.z = std::max(a->max.z, z);
				}
			}
			// bucket lookup, :817-904
			double ux = (double(X) * posScale.x + posOffset.x - min.x) / size.x;
			double uy = (double(Y) * posScale.y + posOffset.y - min.y) / size.y;
			double uz = (double(Z) * posScale.z + posOffset.z - min.z) / size.z;
			int64_t ix = int64_t(std::min(dG * ux, dG - 1.0));
			int64_t iy = int64_t(std::min(dG * uy, dG - 1.0));
			int64_t iz = int64_t(std::min(dG * uz, dG - 1.0));
			int32_t nodeIndex = lut[ix + iy * gridSize + iz * gridSize * gridSize];
			if (nodeIndex == -1) { job.err = "point to chunk lookup failed"; return false; }
			buckets[nodeIndex].insert(buckets[nodeIndex].end(), rec.begin(), rec.end());
		}
	}

	// chunk metadata, :1251-1256 (the cube is recomputed once more)
	double cubeSize = (max - min).max();
	max = min + cubeSize;
	minOut = min; maxOut = max;
	attrsOut = stats;
	attrsOut.posScale = out.posScale; attrsOut.posOffset = out.posOffset;
	// the statistics reach the indexer through the chunks' metadata.json
	// (writeMetadata, :1005-1070; read back at indexer.cpp:72-130): a
	// non-finite value is written as null and read back as +Infinity, for
	// min and max alike (an attribute no point of any source carries)
	for (auto& a : attrsOut.list) {
		double* mn[3] = {&a.min.x, &a.min.y, &a.min.z};
		double* mx[3] = {&a.max.x, &a.max.y, &a.max.z};
		for (int c = 0; c < a.numElements && c < 3; c++) {
			if (!std::isfinite(*mn[c])) *mn[c] = Inf;
			if (!std::isfinite(*mx[c])) *mx[c] = Inf;
		}
	}

	// getChunks, indexer.cpp:53-179 -- chunk order pinned to file-name order
	vector<size_t> order(nodes.size());
	for (size_t i = 0; i < order.size(); i++) order[i] = i;
	std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return nodes[a].id + ".bin" < nodes[b].id + ".bin"; });
	for (size_t oi : order) {
		if (buckets[oi].empty()) continue;
		Chunk c;
		c.id = nodes[oi].id;
		Vec3 bmin = min, bmax = max;
		for (size_t k = 1; k < c.id.size(); k++) {
			int index = c.id[k] - '0';
			Vec3 sz = bmax - bmin;
			Vec3 ctr = bmin + sz * 0.5;
			Vec3 nmin, nmax;
			if ((index & 4) == 0) { nmin.x = bmin.x; nmax.x = ctr.x; } else { nmin.x = ctr.x; nmax.x = bmax.x; }
			if ((index & 2) == 0) { nmin.y = bmin.y; nmax.y = ctr.y; } else { nmin.y = ctr.y; nmax.y = bmax.y; }
			if ((index & 1) == 0) { nmin.z = bmin.z; nmax.z = ctr.z; } else { nmin.z = ctr.z; nmax.z = bmax.z; }
			bmin = nmin; bmax = nmax;
		}
		c.min = bmin; c.max = bmax;
		c.data = std::move(buckets[oi]);
		chunksOut.push_back(std::move(c));
	}
	return true;
}

// ----------------------------------------------------------------- octree
struct Node {  // structures.h:27-140
	vector<shared_ptr<Node>> children;
	string name;
	shared_ptr<vector<uint8_t>> points;
	Vec3 min, max;
	int64_t indexStart = 0, byteOffset = 0, byteSize = 0, numPoints = 0;
	bool sampled = false;
	Node() {}
	Node(string n, Vec3 mn, Vec3 mx) : name(n), min(mn), max(mx) { children.resize(8, nullptr); }
	int64_t level() const { return (int64_t)name.size() - 1; }
	bool isLeaf() const { for (auto& c : children) if (c) return false; return true; }
};

static inline uint64_t splitBy3(unsigned int a) {  // converter_utils.h:89-101
	uint64_t x = a & 0x1fffff;
	x = (x | x << 32) & 0x1f00000000ffff;
	x = (x | x << 16) & 0x1f0000ff0000ff;
	x = (x | x << 8) & 0x100f00f00f00f00f;
	x = (x | x << 4) & 0x10c30c30c30c30c3;
	x = (x | x << 2) & 0x1249249249249249;
	return x;
}
static inline uint64_t morton(unsigned x, unsigned y, unsigned z) { return splitBy3(x) | splitBy3(y) << 1 | splitBy3(z) << 2; }

static void childBox(const Vec3& min, const Vec3& max, int index, Vec3& omin, Vec3& omax) {  // converter_utils.h:106-136
	Vec3 size = max - min;
	Vec3 center = min + (size * 0.5);
	if ((index & 0b100) == 0) { omin.x = min.x; omax.x = center.x; } else { omin.x = center.x; omax.x = max.x; }
	if ((index & 0b010) == 0) { omin.y = min.y; omax.y = center.y; } else { omin.y = center.y; omax.y = max.y; }
	if ((index & 0b001) == 0) { omin.z = min.z; omax.z = center.z; } else { omin.z = center.z; omax.z = max.z; }
}

struct Indexer {
	Attributes attributes;
	shared_ptr<Node> root;
	double spacing = 1.0;
	int64_t octreeDepth = 0;
	int64_t byteOffset = 0;
	vector<uint8_t> octree;
	struct HRec { string name; int64_t byteOffset, byteSize, numPoints; };
	vector<HRec> flushed;
	uint32_t seed = 0;

	void onNodeCompleted(Node* node) {  // indexer.cpp:1605-1608, 1453-1516; indexer.h:146-162
		if (node->numPoints != 0) {
			int64_t bs = (int64_t)node->points->size();
			node->byteSize = bs;
			node->byteOffset = byteOffset;
			byteOffset += bs;
			octree.insert(octree.end(), node->points->begin(), node->points->end());
			node->points = nullptr;
		}
		flushed.push_back({node->name, node->byteOffset, node->byteSize, node->numPoints});
	}
};

static const int64_t maxPointsPerNode = 10'000;  // indexer.h:47

struct NodeCandidate { string name; int64_t indexStart = 0, numPoints = 0, level = 0, x = 0, y = 0, z = 0; };

static vector<vector<int64_t>> createSumPyramid(vector<int64_t>& grid, int gridSize) {  // indexer.cpp:691-730
	int maxLevel = (int)std::log2(gridSize);
	int cur = gridSize / 2;
	vector<vector<int64_t>> pyr(maxLevel + 1);
	for (int level = 0; level < maxLevel; level++) pyr[level].resize((size_t)pow(8, level), 0);
	pyr[maxLevel] = grid;
	for (int level = maxLevel - 1; level >= 0; level--) {
		for (int x = 0; x < cur; x++) for (int y = 0; y < cur; y++) for (int z = 0; z < cur; z++) {
			auto index = morton(z, y, x);
			auto p1 = morton(2 * z, 2 * y, 2 * x);
			int64_t sum = 0;
			for (int i = 0; i < 8; i++) sum += pyr[level + 1][p1 + i];
			pyr[level][index] = sum;
		}
		cur /= 2;
	}
	return pyr;
}

static vector<NodeCandidate> createNodes(vector<vector<int64_t>>& pyr) {  // indexer.cpp:732-817
	vector<NodeCandidate> nodes;
	vector<vector<int64_t>> offs;
	for (auto& c : pyr) {
		if (c.size() == 1) { offs.push_back({0}); continue; }
		vector<int64_t> o(c.size(), 0);
		for (size_t i = 1; i < c.size(); i++) o[i] = o[i - 1] + c[i - 1];
		offs.push_back(o);
	}
	size_t maxLevel = pyr.size() - 1;
	NodeCandidate root;
	vector<NodeCandidate> stack = {root};
	while (!stack.empty()) {
		NodeCandidate cand = stack.back(); stack.pop_back();
		auto level = cand.level; auto x = cand.x, y = cand.y, z = cand.z;
		int64_t numPoints = pyr[level][morton(z, y, x)];
		if ((size_t)level == maxLevel) {
			if (numPoints > 0) nodes.push_back(cand);
		} else if (numPoints > maxPointsPerNode) {
			for (int i = 0; i < 8; i++) {
				auto p1 = morton(2 * z, 2 * y, 2 * x) + i;
				auto count = pyr[level + 1][p1];
				if (count > 0) {
					NodeCandidate ch;
					ch.level = level + 1;
					ch.name = cand.name + std::to_string(i);
					ch.indexStart = offs[level + 1][p1];
					ch.numPoints = count;
					ch.x = 2 * x + ((i & 4) >> 2); ch.y = 2 * y + ((i & 2) >> 1); ch.z = 2 * z + (i & 1);
					stack.push_back(ch);
				}
			}
		} else if (numPoints > 0) {
			nodes.push_back(cand);
		}
	}
	return nodes;
}

static void buildHierarchy(Indexer* indexer, Node* node, shared_ptr<vector<uint8_t>> points, int64_t numPoints, int64_t depth = 0) {
	// indexer.cpp:823-1109
	if (numPoints < maxPointsPerNode) {
		node->indexStart = 0; node->numPoints = numPoints; node->points = points;
		return;
	}
	const int64_t G = 32;
	vector<int64_t> counters(G * G * G, 0);
	Vec3 min = node->min, max = node->max, size = max - min;
	int64_t bpp = indexer->attributes.bytes;
	Vec3 scale = indexer->attributes.posScale, offset = indexer->attributes.posOffset;
	auto gridIndexOf = [&](int64_t i) {
		const uint8_t* p = points->data() + i * bpp;
		int32_t X = rd<int32_t>(p), Y = rd<int32_t>(p + 4), Z = rd<int32_t>(p + 8);
		double x = (X * scale.x) + offset.x, y = (Y * scale.y) + offset.y, z = (Z * scale.z) + offset.z;
		int64_t ix = double(G) * (x - min.x) / size.x;
		int64_t iy = double(G) * (y - min.y) / size.y;
		int64_t iz = double(G) * (z - min.z) / size.z;
		ix = std::max(int64_t(0), std::min(ix, G - 1));
		iy = std::max(int64_t(0), std::min(iy, G - 1));
		iz = std::max(int64_t(0), std::min(iz, G - 1));
		return morton((unsigned)iz, (unsigned)iy, (unsigned)ix);
	};
	for (int64_t i = 0; i < numPoints; i++) counters[gridIndexOf(i)]++;
	{
		vector<int64_t> offsets(counters.size(), 0);
		for (size_t i = 1; i < counters.size(); i++) offsets[i] = offsets[i - 1] + counters[i - 1];
		vector<uint8_t> tmp(numPoints * bpp);
		for (int64_t i = 0; i < numPoints; i++) {
			auto t = offsets[gridIndexOf(i)]++;
			memcpy(tmp.data() + t * bpp, points->data() + i * bpp, bpp);
		}
		memcpy(points->data(), tmp.data(), numPoints * bpp);
	}
	auto pyr = createSumPyramid(counters, (int)G);
	auto nodes = createNodes(pyr);
	auto expandTo = [node](NodeCandidate& cand) {
		string full = node->name + cand.name;
		Node* cur = node;
		for (size_t i = node->name.size(); i < full.size(); i++) {
			int index = full[i] - '0';
			if (!cur->children[index]) {
				auto ch = make_shared<Node>();
				childBox(cur->min, cur->max, index, ch->min, ch->max);
				ch->name = cur->name + std::to_string(index);
				ch->children.resize(8);
				cur->children[index] = ch;
				cur = ch.get();
			} else {
				cur = cur->children[index].get();
			}
		}
		return cur;
	};
	vector<Node*> needRefinement;
	int64_t octreeDepth = 0;
	for (auto& cand : nodes) {
		Node* real = expandTo(cand);
		real->indexStart = cand.indexStart;
		real->numPoints = cand.numPoints;
		auto buf = make_shared<vector<uint8_t>>(points->begin() + cand.indexStart * bpp, points->begin() + (cand.indexStart + cand.numPoints) * bpp);
		real->points = buf;
		if (real->numPoints > maxPointsPerNode) needRefinement.push_back(real);
		octreeDepth = std::max(octreeDepth, real->level());
	}
	indexer->octreeDepth = std::max(indexer->octreeDepth, octreeDepth);
	for (int64_t ni = 0; ni < (int64_t)needRefinement.size(); ni++) {
		auto subject = needRefinement[ni];
		auto buffer = subject->points;
		if (subject->numPoints == numPoints) {  // :1002-1099 duplicate handling
			std::unordered_map<string, int> counts;
			for (int64_t i = 0; i < numPoints; i++) {
				const uint8_t* p = buffer->data() + i * bpp;
				stringstream ss; ss << rd<int32_t>(p) << ", " << rd<int32_t>(p + 4) << ", " << rd<int32_t>(p + 8);
				counts[ss.str()]++;
			}
			int64_t numUnique = (int64_t)counts.size();
			int64_t numDuplicates = subject->numPoints - numUnique;
			if (numDuplicates >= maxPointsPerNode / 2) {
				// the reference copies the FIRST numUnique records (:1088-1090)
				auto distinct = make_shared<vector<uint8_t>>(buffer->begin(), buffer->begin() + numUnique * bpp);
				subject->points = distinct;
				subject->numPoints = numUnique;
				ni--;
				continue;
			}
		}
		int64_t next = subject->numPoints;
		subject->points = nullptr;
		subject->numPoints = 0;
		buildHierarchy(indexer, subject, buffer, next, depth + 1);
	}
}

// --------------------------------------------------------------- samplers
using Callback = function<void(Node*)>;

static void traversePost(Node* node, const function<void(Node*)>& cb) {  // sampler_*.h traversePost
	for (auto& c : node->children) if (c && !c->sampled) traversePost(c.get(), cb);
	cb(node);
}

static void samplePoisson(Node* root, Attributes& attributes, double baseSpacing, const Callback& onNodeCompleted) {
	// sampler_poisson.h:14-304
	struct Point { double x, y, z; int32_t pointIndex, childIndex; };
	int64_t bpp = attributes.bytes;
	Vec3 scale = attributes.posScale, offset = attributes.posOffset;
	static thread_local vector<Point> accepted(1'000'000);
	traversePost(root, [&](Node* node) {
		node->sampled = true;
		if (node->isLeaf()) return;
		vector<Point> points;
		vector<vector<int8_t>> flags(8);
		vector<int64_t> numRejectedPerChild(8, 0);
		int64_t numAccepted = 0;
		for (int64_t ci = 0; ci < 8; ci++) {
			auto child = node->children[ci];
			if (!child) continue;
			flags[ci].assign(child->numPoints, 0);
			for (int64_t i = 0; i < child->numPoints; i++) {
				const uint8_t* p = child->points->data() + i * bpp;
				double x = (rd<int32_t>(p) * scale.x) + offset.x;
				double y = (rd<int32_t>(p + 4) * scale.y) + offset.y;
				double z = (rd<int32_t>(p + 8) * scale.z) + offset.z;
				points.push_back({x, y, z, (int32_t)i, (int32_t)ci});
			}
		}
		int64_t numAcc = 0;
		double spacing = baseSpacing / pow(2.0, node->level());
		double squaredSpacing = spacing * spacing;
		Vec3 center = (node->min + node->max) * 0.5;
		auto checkAccept = [&](const Point& cand) {
			double cx = cand.x - center.x, cy = cand.y - center.y, cz = cand.z - center.z;
			double cdd = cx * cx + cy * cy + cz * cz;
			double cd = sqrt(cdd);
			double limit = cd - spacing;
			double limitSquared = limit * limit;
			int64_t j = 0;
			for (int64_t i = numAcc - 1; i >= 0; i--) {
				auto& pt = accepted[i];
				double px = pt.x - center.x, py = pt.y - center.y, pz = pt.z - center.z;
				double pdd = px * px + py * py + pz * pz;
				if (pdd < limitSquared) return true;
				double dx = pt.x - cand.x, dy = pt.y - cand.y, dz = pt.z - cand.z;
				double dd = dx * dx + dy * dy + dz * dz;
				if (dd < squaredSpacing) return false;
				j++;
				if (j > 10'000) return true;
			}
			return true;
		};
		std::sort(points.begin(), points.end(), [center](Point a, Point b) -> bool {
			auto ax = a.x - center.x, ay = a.y - center.y, az = a.z - center.z;
			auto add = ax * ax + ay * ay + az * az;
			auto bx = b.x - center.x, by = b.y - center.y, bz = b.z - center.z;
			auto bdd = bx * bx + by * by + bz * bz;
			return add < bdd;
		});
		for (const Point& pt : points) {
			bool ok = checkAccept(pt);
			if (ok) { accepted[numAcc] = pt; numAcc++; numAccepted++; }
			else numRejectedPerChild[pt.childIndex]++;
			flags[pt.childIndex][pt.pointIndex] = ok ? 1 : 0;
		}
		auto acc = make_shared<vector<uint8_t>>();
		acc->reserve(numAccepted * bpp);
		for (int64_t ci = 0; ci < 8; ci++) {
			auto child = node->children[ci];
			if (!child) continue;
			auto numRejected = numRejectedPerChild[ci];
			auto rej = make_shared<vector<uint8_t>>();
			rej->reserve(numRejected * bpp);
			for (int64_t i = 0; i < child->numPoints; i++) {
				const uint8_t* p = child->points->data() + i * bpp;
				if (flags[ci][i]) acc->insert(acc->end(), p, p + bpp); else rej->insert(rej->end(), p, p + bpp);
			}
			if (numRejected == 0 && child->isLeaf()) {
				node->children[ci] = nullptr;
			}
			if (numRejected > 0) {
				child->points = rej; child->numPoints = numRejected;
				onNodeCompleted(child.get());
			} else if (numRejected == 0) {
				child->points = nullptr; child->numPoints = 0;
				onNodeCompleted(child.get());
			}
		}
		node->points = acc;
		node->numPoints = numAccepted;
	});
}

static void samplePoissonAverage(Node* root, Attributes& attributes, double baseSpacing, const Callback& onNodeCompleted) {
	// sampler_poisson_average.h:14-492
	struct Point { double x, y, z; int32_t pointIndex, childIndex; int64_t r = 0, g = 0, b = 0, w = 0; int64_t mainIndex = 0; bool accepted = false; };
	int64_t bpp = attributes.bytes;
	Vec3 scale = attributes.posScale, offset = attributes.posOffset;
	int offsetRGB = attributes.getOffset("rgb");
	traversePost(root, [&](Node* node) {
		node->sampled = true;
		if (node->isLeaf()) return;
		Vec3 min = node->min, max = node->max, size = max - min;
		vector<Point> points;
		vector<vector<int8_t>> flags(8);
		vector<int64_t> numRejectedPerChild(8, 0);
		int64_t numAccepted = 0;
		for (int ci = 0; ci < 8; ci++) {
			auto child = node->children[ci];
			if (!child) continue;
			flags[ci].assign(child->numPoints, 0);
			for (int i = 0; i < child->numPoints; i++) {
				const uint8_t* p = child->points->data() + (int64_t)i * bpp;
				double x = (rd<int32_t>(p) * scale.x) + offset.x;
				double y = (rd<int32_t>(p + 4) * scale.y) + offset.y;
				double z = (rd<int32_t>(p + 8) * scale.z) + offset.z;
				Point pt; pt.x = x; pt.y = y; pt.z = z; pt.pointIndex = i; pt.childIndex = ci;
				pt.r = rd<uint16_t>(p + offsetRGB); pt.g = rd<uint16_t>(p + offsetRGB + 2); pt.b = rd<uint16_t>(p + offsetRGB + 4); pt.w = 1;
				pt.mainIndex = (int64_t)points.size();
				points.push_back(pt);
			}
		}
		double spacing = baseSpacing / pow(2.0, node->level());
		double squaredSpacing = spacing * spacing;
		Vec3 center = (node->min + node->max) * 0.5;
		const double G = 16;
		vector<vector<Point>> grid((size_t)(G * G * G));
		auto sq = [](const Point& a, const Point& b) { double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z; return dx * dx + dy * dy + dz * dz; };
		struct Win { int ix, iy, iz, x0, y0, z0, x1, y1, z1; };
		auto window = [&](const Point& c) {
			double dx = G * (c.x - min.x) / size.x, dy = G * (c.y - min.y) / size.y, dz = G * (c.z - min.z) / size.z;
			double dx0 = G * (c.x - spacing - min.x) / size.x, dy0 = G * (c.y - spacing - min.y) / size.y, dz0 = G * (c.z - spacing - min.z) / size.z;
			double dx1 = G * (c.x + spacing - min.x) / size.x, dy1 = G * (c.y + spacing - min.y) / size.y, dz1 = G * (c.z + spacing - min.z) / size.z;
			auto cl = [G](double v) { return (int)std::max(std::min(v, G - 1.0), 0.0); };
			return Win{cl(dx), cl(dy), cl(dz), cl(dx0), cl(dy0), cl(dz0), cl(dx1), cl(dy1), cl(dz1)};
		};
		auto checkAccept = [&](const Point& c) {
			Win w = window(c);
			for (int x = w.x0; x <= w.x1; x++) for (int y = w.y0; y <= w.y1; y++) for (int z = w.z0; z <= w.z1; z++) {
				int index = x + y * (int)G + z * (int)G * (int)G;
				for (auto& pt : grid[index]) if (sq(pt, c) < squaredSpacing) return false;
			}
			grid[w.ix + w.iy * (int)G + w.iz * (int)G * (int)G].push_back(c);
			return true;
		};
		std::sort(points.begin(), points.end(), [center](Point a, Point b) -> bool {
			auto ax = a.x - center.x, ay = a.y - center.y, az = a.z - center.z;
			auto add = ax * ax + ay * ay + az * az;
			auto bx = b.x - center.x, by = b.y - center.y, bz = b.z - center.z;
			auto bdd = bx * bx + by * by + bz * bz;
			return add < bdd;
		});
		vector<int32_t> mainToSort(points.size());
		for (size_t i = 0; i < points.size(); i++) mainToSort[points[i].mainIndex] = (int32_t)i;
		for (Point& pt : points) {
			bool ok = checkAccept(pt);
			if (ok) numAccepted++; else numRejectedPerChild[pt.childIndex]++;
			flags[pt.childIndex][pt.pointIndex] = ok ? 1 : 0;
		}
		for (Point& cand : points) {  // :369-415
			Win w = window(cand);
			for (int x = w.x0; x <= w.x1; x++) for (int y = w.y0; y <= w.y1; y++) for (int z = w.z0; z <= w.z1; z++) {
				int index = x + y * (int)G + z * (int)G * (int)G;
				for (auto& pt : grid[index]) {
					if (sq(pt, cand) < squaredSpacing) {
						Point& avg = points[mainToSort[pt.mainIndex]];
						avg.r = avg.r + cand.r; avg.g = avg.g + cand.g; avg.b = avg.b + cand.b; avg.w = avg.w + cand.w;
					}
				}
			}
		}
		auto acc = make_shared<vector<uint8_t>>();
		size_t j = 0;
		for (int ci = 0; ci < 8; ci++) {
			auto child = node->children[ci];
			if (!child) continue;
			auto numRejected = numRejectedPerChild[ci];
			auto rej = make_shared<vector<uint8_t>>();
			for (int i = 0; i < child->numPoints; i++) {
				uint8_t* p = child->points->data() + (int64_t)i * bpp;
				Point& pt = points[mainToSort[j]];
				uint16_t rgb[3] = {(uint16_t)(pt.r / pt.w), (uint16_t)(pt.g / pt.w), (uint16_t)(pt.b / pt.w)};
				memcpy(p + offsetRGB, rgb, 6);
				if (flags[ci][i]) acc->insert(acc->end(), p, p + bpp);
				rej->insert(rej->end(), p, p + bpp);
				j++;
			}
			if (numRejected == 0) node->children[ci] = nullptr;
			if (numRejected > 0) { child->points = rej; onNodeCompleted(child.get()); }
		}
		node->points = acc;
		node->numPoints = numAccepted;
	});
}

static void sampleRandom(Node* root, Attributes& attributes, uint32_t seed, const Callback& onNodeCompleted) {
	// sampler_random.h:14-232
	int64_t bpp = attributes.bytes;
	Vec3 scale = attributes.posScale, offset = attributes.posOffset;
	const int64_t G = 128;
	static thread_local vector<int64_t> grid(G * G * G, -1);
	static thread_local int64_t iteration = 0;
	traversePost(root, [&](Node* node) {
		node->sampled = true;
		iteration++;
		Vec3 min = node->min, max = node->max, size = max - min;
		if (node->isLeaf()) {
			vector<int> indices(node->numPoints);
			for (int i = 0; i < node->numPoints; i++) indices[i] = i;
			std::shuffle(indices.begin(), indices.end(), std::default_random_engine(seed));
			auto buf = make_shared<vector<uint8_t>>(node->points->size());
			for (int i = 0; i < node->numPoints; i++) memcpy(buf->data() + (int64_t)indices[i] * bpp, node->points->data() + (int64_t)i * bpp, bpp);
			node->points = buf;
			return;
		}
		vector<vector<int8_t>> flags(8);
		vector<int64_t> numRejectedPerChild(8, 0);
		int64_t numAccepted = 0;
		static const double all = sqrt(3.0);
		for (int ci = 0; ci < 8; ci++) {
			auto child = node->children[ci];
			if (!child) continue;
			flags[ci].assign(child->numPoints, 0);
			int64_t numRejected = 0;
			for (int i = 0; i < child->numPoints; i++) {
				const uint8_t* p = child->points->data() + (int64_t)i * bpp;
				double x = (rd<int32_t>(p) * scale.x) + offset.x;
				double y = (rd<int32_t>(p + 4) * scale.y) + offset.y;
				double z = (rd<int32_t>(p + 8) * scale.z) + offset.z;
				double nx = (x - min.x) / size.x, ny = (y - min.y) / size.y, nz = (z - min.z) / size.z;
				double lx = 2.0 * fmod(double(G) * nx, 1.0) - 1.0;
				double ly = 2.0 * fmod(double(G) * ny, 1.0) - 1.0;
				double lz = 2.0 * fmod(double(G) * nz, 1.0) - 1.0;
				double distance = sqrt(lx * lx + ly * ly + lz * lz);
				int64_t cx = double(G) * nx, cy = double(G) * ny, cz = double(G) * nz;
				cx = std::max(int64_t(0), std::min(cx, G - 1));
				cy = std::max(int64_t(0), std::min(cy, G - 1));
				cz = std::max(int64_t(0), std::min(cz, G - 1));
				auto& gv = grid[cx + cy * G + cz * G * G];
				bool ok;
				if (child->numPoints < 100) ok = true;
				else if (distance < 0.7 * all && gv < iteration) ok = true;
				else ok = false;
				if (ok) { gv = iteration; numAccepted++; } else numRejected++;
				flags[ci][i] = ok ? 1 : 0;
			}
			numRejectedPerChild[ci] = numRejected;
		}
		auto acc = make_shared<vector<uint8_t>>();
		for (int ci = 0; ci < 8; ci++) {
			auto child = node->children[ci];
			if (!child) continue;
			auto numRejected = numRejectedPerChild[ci];
			auto rej = make_shared<vector<uint8_t>>();
			for (int i = 0; i < child->numPoints; i++) {
				const uint8_t* p = child->points->data() + (int64_t)i * bpp;
				if (flags[ci][i]) acc->insert(acc->end(), p, p + bpp); else rej->insert(rej->end(), p, p + bpp);
			}
			if (numRejected == 0 && child->isLeaf()) node->children[ci] = nullptr;
			if (numRejected > 0) { child->points = rej; child->numPoints = numRejected; onNodeCompleted(child.get()); }
			else if (numRejected == 0) { child->points = nullptr; child->numPoints = 0; onNodeCompleted(child.get()); }
		}
		node->points = acc;
		node->numPoints = numAccepted;
	});
}

// ------------------------------------------------------------- hierarchy
// HierarchyFlusher (indexer.h:120-244) + HierarchyBuilder (HierarchyBuilder.h)
struct HNode { string name; int numPoints = 0; uint8_t childMask = 0; uint64_t byteOffset = 0, byteSize = 0; int type = 1; uint64_t proxyByteOffset = 0, proxyByteSize = 0; };
struct HChunk { string name; vector<shared_ptr<HNode>> nodes; int64_t byteOffset = 0; };
struct HBatch {
	string name; int numNodes = 0; int64_t byteSize = 0;
	vector<shared_ptr<HNode>> nodes; vector<shared_ptr<HChunk>> chunks;
	std::unordered_map<string, shared_ptr<HNode>> nodeMap; std::unordered_map<string, shared_ptr<HChunk>> chunkMap;
};
enum { NORMAL = 0, LEAF = 1, PROXY = 2 };
static const int stepSize = 4;

static shared_ptr<HBatch> loadBatch(const string& batchName, const vector<Indexer::HRec>& recs) {
	auto batch = make_shared<HBatch>();
	batch->name = batchName;
	batch->numNodes = (int)recs.size();
	for (auto& r : recs) {
		auto node = make_shared<HNode>();
		node->name = r.name;
		node->numPoints = (int)(uint32_t)r.numPoints;
		node->byteOffset = (uint64_t)(int64_t)r.byteOffset;
		node->byteSize = (uint64_t)(int64_t)(int32_t)(uint32_t)r.byteSize;
		int chunkLevel = (int)((node->name.size() - 2) / 4);
		string key = node->name.substr(0, stepSize * chunkLevel + 1);
		if (node->name == batch->name) key = node->name;
		if (!batch->chunkMap.count(key)) {
			auto c = make_shared<HChunk>(); c->name = key;
			batch->chunkMap[key] = c; batch->chunks.push_back(c);
		}
		batch->chunkMap[key]->nodes.push_back(node);
		batch->nodes.push_back(node);
		batch->nodeMap[node->name] = batch->nodes.back();
		bool isChunkKey = ((node->name.size() - 1) % stepSize) == 0;
		bool isBatchSubChunk = node->name.size() > stepSize + 1;
		if (isChunkKey && isBatchSubChunk) {
			if (!batch->chunkMap.count(node->name)) {
				auto c = make_shared<HChunk>(); c->name = node->name;
				batch->chunkMap[node->name] = c; batch->chunks.push_back(c);
			}
			batch->chunkMap[node->name]->nodes.push_back(node);
		}
	}
	auto bfs = [](const string& a, const string& b) { return a.size() != b.size() ? a.size() < b.size() : a < b; };
	std::sort(batch->chunks.begin(), batch->chunks.end(), [&](const shared_ptr<HChunk>& a, const shared_ptr<HChunk>& b) { return bfs(a->name, b->name); });
	for (auto& node : batch->nodes) {
		node->type = LEAF;
		string parentName = node->name.substr(0, node->name.size() - 1);
		auto it = batch->nodeMap.find(parentName);
		if (it != batch->nodeMap.end()) {
			int childIndex = node->name.back() - '0';
			it->second->type = NORMAL;
			it->second->childMask = it->second->childMask | (1 << childIndex);
		}
	}
	for (auto& chunk : batch->chunks) {
		auto it = batch->nodeMap.find(chunk->name);
		if (it != batch->nodeMap.end()) it->second->type = PROXY;
	}
	for (auto& chunk : batch->chunks)
		std::sort(chunk->nodes.begin(), chunk->nodes.end(), [&](const shared_ptr<HNode>& a, const shared_ptr<HNode>& b) { return bfs(a->name, b->name); });
	return batch;
}

static bool processBatch(HBatch& batch) {
	int64_t off = 0;
	for (auto& chunk : batch.chunks) {
		chunk->byteOffset = off;
		if (chunk->name != batch.name) {
			string parentName = chunk->name.substr(0, chunk->name.size() - stepSize);
			if (!batch.chunkMap.count(parentName)) return false;
			auto proxy = batch.nodeMap[chunk->name];
			if (!proxy) return false;
			proxy->type = PROXY;
			proxy->proxyByteOffset = chunk->byteOffset;
			proxy->proxyByteSize = 22 * chunk->nodes.size();
		}
		off += 22 * chunk->nodes.size();
	}
	batch.byteSize = off;
	return true;
}

static vector<uint8_t> serializeBatch(HBatch& batch, int64_t bytesWritten) {
	size_t numRecords = 0;
	for (auto& c : batch.chunks) numRecords += c->nodes.size();
	vector<uint8_t> buf(22 * numRecords);
	size_t k = 0;
	for (auto& chunk : batch.chunks) {
		for (auto& node : chunk->nodes) {
			bool isProxyNode = node->type == PROXY && node->name != chunk->name;
			uint8_t type = (uint8_t)node->type;
			if (node->type == PROXY && !isProxyNode) type = NORMAL;
			uint64_t bs = isProxyNode ? node->proxyByteSize : node->byteSize;
			uint64_t bo = isProxyNode ? bytesWritten + node->proxyByteOffset : node->byteOffset;
			uint32_t np = (uint32_t)node->numPoints;
			buf[22 * k + 0] = type;
			buf[22 * k + 1] = node->childMask;
			memcpy(&buf[22 * k + 2], &np, 4);
			memcpy(&buf[22 * k + 6], &bo, 8);
			memcpy(&buf[22 * k + 14], &bs, 8);
			k++;
		}
	}
	batch.byteSize = (int64_t)buf.size();
	return buf;
}

static bool buildHierarchyFile(const vector<Indexer::HRec>& flushed, vector<uint8_t>& out, int64_t& firstChunkSize) {
	// grouping, indexer.h:171-193 (appends keep completion order per file)
	std::map<string, vector<Indexer::HRec>> groups;  // file name order == key order
	for (auto& n : flushed) {
		string key = n.name.substr(0, stepSize + 1);
		if (n.name.size() <= (size_t)stepSize + 1) key = "r";
		groups[key].push_back(n);
		if (n.name.size() == (size_t)stepSize + 1) groups[n.name].push_back(n);
	}
	if (!groups.count("r")) return false;
	auto root = loadBatch("r", groups["r"]);
	out.assign(22 * root->nodes.size(), 0);
	int64_t bytesWritten = (int64_t)out.size();
	for (auto& [key, recs] : groups) {  // HierarchyBuilder.h:302-331 in file-name order
		if (key == "r") continue;
		auto batch = loadBatch(key, recs);
		if (!processBatch(*batch)) return false;
		auto buf = serializeBatch(*batch, bytesWritten);
		if (batch->nodes.size() > 1) {
			auto proxy = root->nodeMap[batch->name];
			proxy->type = PROXY;
			proxy->proxyByteOffset = bytesWritten;
			proxy->proxyByteSize = 22 * batch->chunkMap[batch->name]->nodes.size();
		} else {
			root->nodeMap[batch->name]->type = LEAF;
		}
		out.insert(out.end(), buf.begin(), buf.end());
		bytesWritten += (int64_t)buf.size();
	}
	auto rootBuf = serializeBatch(*root, 0);
	memcpy(out.data(), rootBuf.data(), rootBuf.size());
	firstChunkSize = root->byteSize;
	return true;
}

// ------------------------------------------------------------- metadata
static string createMetadata(const string& name, int64_t pointsTotal, int64_t firstChunkSize, int64_t depth, const Attributes& attributes, double spacing, Vec3 min, Vec3 max) {
	// indexer.cpp:354-524
	auto d = [](double v) { stringstream ss; ss << std::setprecision(std::numeric_limits<double>::max_digits10); ss << v; return ss.str(); };
	auto s = [](const string& str) { return "\"" + str + "\""; };
	auto t = [](int n) { return string(n, '\t'); };
	auto toJson = [&](Vec3 v) { return "[" + d(v.x) + ", " + d(v.y) + ", " + d(v.z) + "]"; };
	auto vecToJson = [&](vector<double> v) {
		stringstream ss; ss << "[";
		for (size_t i = 0; i < v.size(); i++) { ss << d(v[i]); if (i < v.size() - 1) ss << ", "; }
		ss << "]"; return ss.str();
	};
	auto vecI64 = [](const vector<int64_t>& v) {
		stringstream ss; ss << "[";
		for (size_t i = 0; i < v.size(); i++) { ss << v[i]; if (i < v.size() - 1) ss << ", "; }
		ss << "]"; return ss.str();
	};
	stringstream h;
	h << "{" << std::endl;
	h << t(2) << s("firstChunkSize") << ": " << firstChunkSize << ", " << std::endl;
	h << t(2) << s("stepSize") << ": " << stepSize << ", " << std::endl;
	h << t(2) << s("depth") << ": " << depth << std::endl;
	h << t(1) << "}";
	stringstream bb;
	bb << "{" << std::endl;
	bb << t(2) << s("min") << ": " << toJson(min) << ", " << std::endl;
	bb << t(2) << s("max") << ": " << toJson(max) << std::endl;
	bb << t(1) << "}";
	stringstream at;
	at << "[" << std::endl;
	for (size_t i = 0; i < attributes.list.size(); i++) {
		auto& a = attributes.list[i];
		if (i == 0) at << t(2) << "{" << std::endl;
		at << t(3) << s("name") << ": " << s(a.name) << "," << std::endl;
		at << t(3) << s("description") << ": " << s(a.description) << "," << std::endl;
		at << t(3) << s("size") << ": " << a.size << "," << std::endl;
		at << t(3) << s("numElements") << ": " << a.numElements << "," << std::endl;
		at << t(3) << s("elementSize") << ": " << a.elementSize << "," << std::endl;
		at << t(3) << s("type") << ": " << s(typeName(a.type)) << "," << std::endl;
		bool empty = true;
		for (auto v : a.histogram) if (v != 0) empty = false;
		if (a.size == 1 && !empty) at << t(3) << s("histogram") << ": " << vecI64(a.histogram) << ", " << std::endl;
		if (a.numElements == 1) {
			at << t(3) << s("min") << ": " << vecToJson({a.min.x}) << "," << std::endl;
			at << t(3) << s("max") << ": " << vecToJson({a.max.x}) << "," << std::endl;
			at << t(3) << s("scale") << ": " << vecToJson({a.scale.x}) << "," << std::endl;
			at << t(3) << s("offset") << ": " << vecToJson({a.offset.x}) << std::endl;
		} else if (a.numElements == 2) {
			at << t(3) << s("min") << ": " << vecToJson({a.min.x, a.min.y}) << "," << std::endl;
			at << t(3) << s("max") << ": " << vecToJson({a.max.x, a.max.y}) << "," << std::endl;
			at << t(3) << s("scale") << ": " << vecToJson({a.scale.x, a.scale.y}) << "," << std::endl;
			at << t(3) << s("offset") << ": " << vecToJson({a.offset.x, a.offset.y}) << std::endl;
		} else if (a.numElements == 3) {
			at << t(3) << s("min") << ": " << vecToJson({a.min.x, a.min.y, a.min.z}) << "," << std::endl;
			at << t(3) << s("max") << ": " << vecToJson({a.max.x, a.max.y, a.max.z}) << "," << std::endl;
			at << t(3) << s("scale") << ": " << vecToJson({a.scale.x, a.scale.y, a.scale.z}) << "," << std::endl;
			at << t(3) << s("offset") << ": " << vecToJson({a.offset.x, a.offset.y, a.offset.z}) << std::endl;
		}
		if (i < attributes.list.size() - 1) at << t(2) << "},{" << std::endl; else at << t(2) << "}" << std::endl;
	}
	at << t(1) << "]";
	stringstream ss;
	ss << t(0) << "{" << std::endl;
	ss << t(1) << s("version") << ": " << s("2.0") << "," << std::endl;
	ss << t(1) << s("name") << ": " << s(name) << "," << std::endl;
	ss << t(1) << s("description") << ": " << s("") << "," << std::endl;
	ss << t(1) << s("points") << ": " << pointsTotal << "," << std::endl;
	ss << t(1) << s("projection") << ": " << s("") << "," << std::endl;
	ss << t(1) << s("hierarchy") << ": " << h.str() << "," << std::endl;
	ss << t(1) << s("offset") << ": " << toJson(attributes.posOffset) << "," << std::endl;
	ss << t(1) << s("scale") << ": " << toJson(attributes.posScale) << "," << std::endl;
	ss << t(1) << s("spacing") << ": " << d(spacing) << "," << std::endl;
	ss << t(1) << s("boundingBox") << ": " << bb.str() << "," << std::endl;
	ss << t(1) << s("encoding") << ": " << s("DEFAULT") << "," << std::endl;
	ss << t(1) << s("attributes") << ": " << at.str() << std::endl;
	ss << t(0) << "}" << std::endl;
	return ss.str();
}

// ------------------------------------------------------------ doIndexing
struct CRNode {  // indexer.h:258-301
	string name; Node* node = nullptr; vector<shared_ptr<CRNode>> children; vector<Node*> fcrs; int numPoints = 0;
	CRNode() { children.resize(8, nullptr); }
	bool isLeaf() const { for (auto& c : children) if (c) return false; return true; }
};

static void traverseNode(Node* n, const function<void(Node*)>& cb) { cb(n); for (auto& c : n->children) if (c) traverseNode(c.get(), cb); }
static void traverseCR(CRNode* n, const function<void(CRNode*)>& cb) { cb(n); for (auto& c : n->children) if (c) traverseCR(c.get(), cb); }
static void traverseCRPost(CRNode* n, const function<void(CRNode*)>& cb) { for (auto& c : n->children) if (c) traverseCRPost(c.get(), cb); cb(n); }

static void addDescendant(Node* root, shared_ptr<Node> desc) {  // structures.h:61-88
	int dl = (int)desc->name.size() - 1;
	Node* cur = root;
	for (int level = 1; level < dl; level++) {
		int index = desc->name[level] - '0';
		if (cur->children[index]) cur = cur->children[index].get();
		else {
			Vec3 mn, mx; childBox(cur->min, cur->max, index, mn, mx);
			auto ch = make_shared<Node>(cur->name + std::to_string(index), mn, mx);
			cur->children[index] = ch;
			cur = ch.get();
		}
	}
	cur->children[desc->name[dl] - '0'] = desc;
}

static bool runIndexing(Job& job, vector<Chunk>& chunks, Attributes& attrs, Vec3 min, Vec3 max, Result& res) {
	Indexer ix;
	ix.attributes = attrs;
	ix.root = make_shared<Node>("r", min, max);
	ix.spacing = (max - min).x / 128.0;  // indexer.cpp:1603
	ix.seed = job.seed;
	Callback done = [&ix](Node* n) { ix.onNodeCompleted(n); };
	auto sample = [&](Node* n) {
		if (job.method == "poisson") samplePoisson(n, ix.attributes, ix.spacing, done);
		else if (job.method == "poisson_average") samplePoissonAverage(n, ix.attributes, ix.spacing, done);
		else sampleRandom(n, ix.attributes, ix.seed, done);
	};
	int64_t bpp = attrs.bytes;
	vector<shared_ptr<Node>> chunkRoots;
	for (auto& c : chunks) {  // indexer.cpp:1639-1702, one chunk at a time
		auto cr = make_shared<Node>(c.id, c.min, c.max);
		auto buf = make_shared<vector<uint8_t>>(std::move(c.data));
		int64_t n = (int64_t)buf->size() / bpp;
		buildHierarchy(&ix, cr.get(), buf, n);
		sample(cr.get());
		cr->children.clear();
		cr->children.resize(0);
		if (cr->name.size() > 1) addDescendant(ix.root.get(), cr);
		chunkRoots.push_back(cr);
	}
	{  // processChunkRoots, indexer.cpp:202-281
		std::unordered_map<string, shared_ptr<CRNode>> map;
		vector<shared_ptr<CRNode>> list;
		traverseNode(ix.root.get(), [&](Node* n) {
			auto c = make_shared<CRNode>(); c->name = n->name; c->node = n; c->children.resize(n->children.size());
			list.push_back(c); map[c->name] = c;
		});
		for (auto& c : list) {
			string pn = c->name.substr(0, c->name.size() - 1);
			if (pn != "") map[pn]->children[c->name.back() - '0'] = c;
		}
		for (auto& cr : chunkRoots) {  // flushed in completion (== chunk) order
			auto c = map[cr->name];
			if (!c) continue;
			c->fcrs.push_back(cr.get());
			c->numPoints += (int)cr->numPoints;
		}
		traverseCRPost(map["r"].get(), [](CRNode* n) {
			if (n->isLeaf()) return;
			int np = 0;
			for (auto& c : n->children) if (c) np += c->numPoints;
			n->numPoints = np;
			if (n->numPoints < 5'000'000) {
				for (auto& c : n->children) if (c) n->fcrs.insert(n->fcrs.end(), c->fcrs.begin(), c->fcrs.end());
				n->children.clear();
			}
		});
		vector<Node*> tasks;
		traverseCR(map["r"].get(), [&](CRNode* n) { if (!n->fcrs.empty()) tasks.push_back(n->node); });
		for (Node* t : tasks) { sample(t); t->children.clear(); t->children.resize(0); }
	}
	if (chunks.size() == 1) ix.root = chunkRoots[0];
	else if (!ix.root->sampled) sample(ix.root.get());
	ix.onNodeCompleted(ix.root.get());

	int64_t firstChunkSize = 0;
	if (!buildHierarchyFile(ix.flushed, res.hierarchy, firstChunkSize)) { job.err = "hierarchy build failed"; return false; }
	res.octree = std::move(ix.octree);
	string md = createMetadata(job.name, job.totalPoints, firstChunkSize, ix.octreeDepth, ix.attributes, ix.spacing, ix.root->min, ix.root->max);
	res.metadata.assign(md.begin(), md.end());
	for (auto& r : ix.flushed) res.nodes.push_back({r.name, r.byteOffset, r.byteSize, r.numPoints});
	return true;
}

bool convert(const vector<SourceImage>& sources, const vector<string>& attributes, const string& method, const string& name, uint32_t seed,
             Result& res, string& err) {
	Job job;
	job.method = method; job.name = name; job.seed = seed; job.requested = attributes;
	if (method != "poisson" && method != "poisson_average" && method != "random") { err = "unknown method"; return false; }
	if (sources.empty()) { err = "no input"; return false; }
	for (auto& si : sources) {
		Source src;
		src.las = si.las;
		if (!parseHeader(si.las, si.size, src.header, job.err)) { err = job.err; return false; }
		job.sources.push_back(std::move(src));
	}
	if (!setup(job)) { err = job.err; return false; }
	if (method == "poisson_average" && job.attributes.getOffset("rgb") < 0) { err = "poisson_average needs rgb (undefined in the reference)"; return false; }
	vector<Chunk> chunks; Attributes attrs; Vec3 min, max;
	if (!doChunking(job, chunks, attrs, min, max)) { err = job.err; return false; }
	res.chunkIds.clear(); res.chunkCounts.clear();
	for (auto& c : chunks) { res.chunkIds.push_back(c.id); res.chunkCounts.push_back((int64_t)c.data.size() / attrs.bytes); }
	if (!runIndexing(job, chunks, attrs, min, max, res)) { err = job.err; return false; }
	return true;
}

bool convert(const uint8_t* las, size_t size, const string& method, const string& name, uint32_t seed, Result& res, string& err) {
	return convert(vector<SourceImage>{{las, size}}, {}, method, name, seed, res, err);
}

// The counting pass alone for one LAS image (countPointsInCells,
// chunker_countsort_laszip.cpp:131-361): every point's quantized X, Y, Z and
// count-grid cell, and the grid of counts. X/Y/Z/cell hold the point count,
// grid gridSize^3 entries.
bool decodeCount(const uint8_t* las, size_t size, int32_t* X, int32_t* Y, int32_t* Z, uint32_t* cell, vector<int64_t>& grid,
                 int64_t& gridSize, string& err) {
	Job job;
	Source src;
	src.las = las;
	if (!parseHeader(las, size, src.header, job.err)) { err = job.err; return false; }
	job.sources.push_back(std::move(src));
	if (!setup(job)) { err = job.err; return false; }
	const int64_t total = job.totalPoints;
	gridSize = total < 100'000'000 ? 128 : (total < 500'000'000 ? 256 : 512);  // :1214-1220
	grid.assign(gridSize * gridSize * gridSize, 0);
	const Attributes& out = job.attributes;
	const Vec3 posScale = out.posScale, posOffset = out.posOffset, min = job.min, max = job.max;
	const double cubeSize = (max - min).max();
	const Vec3 csize(cubeSize, cubeSize, cubeSize);
	const double dG = double(gridSize);
	int64_t k = 0;
	for (auto& s : job.sources) for (int64_t i = 0; i < s.header.numPoints; i++, k++) {
		PointCoord c = lasCoordinates(s, i);
		X[k] = int32_t((c.x - posOffset.x) / posScale.x);
		Y[k] = int32_t((c.y - posOffset.y) / posScale.y);
		Z[k] = int32_t((c.z - posOffset.z) / posScale.z);
		double ux = (double(X[k]) * posScale.x + posOffset.x - min.x) / csize.x;
		double uy = (double(Y[k]) * posScale.y + posOffset.y - min.y) / csize.y;
		double uz = (double(Z[k]) * posScale.z + posOffset.z - min.z) / csize.z;
		if (!(ux >= 0.0 && uy >= 0.0 && uz >= 0.0 && ux <= 1.0 && uy <= 1.0 && uz <= 1.0)) { err = "point outside bounding box"; return false; }
		int64_t ix = int64_t(std::min(dG * ux, dG - 1.0));
		int64_t iy = int64_t(std::min(dG * uy, dG - 1.0));
		int64_t iz = int64_t(std::min(dG * uz, dG - 1.0));
		const int64_t index = ix + iy * gridSize + iz * gridSize * gridSize;
		cell[k] = (uint32_t)index;
		grid[index]++;
	}
	return true;
}

}  // namespace pcref

// ----------------------------------------------------------------- C API
extern "C" {

struct pcref_output {
	uint8_t* octree; uint64_t octree_size;
	uint8_t* hierarchy; uint64_t hierarchy_size;
	char* metadata; uint64_t metadata_size;
	int32_t num_chunks;
	char* chunk_ids;         // num_chunks NUL-terminated ids, concatenated
	int64_t* chunk_counts;   // points per chunk, chunk (file-name) order
	char error[256];
	int64_t num_nodes;       // completed nodes, completion order
	char* node_names;        // NUL-terminated names, concatenated
	int64_t* node_info;      // per node: byte offset, byte size, point count
};

// Several sources (the reference's input list, in order) and an optional
// --attributes list (attrs may be NULL when nattrs is 0).
int pcref_convert_sources(const void* const* las, const uint64_t* sizes, int32_t nsources, const char* const* attrs, int32_t nattrs,
                          const char* method, const char* name, uint32_t seed, pcref_output* out) {
	memset(out, 0, sizeof(*out));
	std::vector<pcref::SourceImage> srcs;
	for (int32_t i = 0; i < nsources; i++) srcs.push_back({(const uint8_t*)las[i], (size_t)sizes[i]});
	std::vector<std::string> names;
	for (int32_t i = 0; i < nattrs; i++) names.push_back(attrs[i]);
	pcref::Result res;
	std::string err;
	if (!pcref::convert(srcs, names, method, name, seed, res, err)) {
		snprintf(out->error, sizeof(out->error), "%s", err.c_str());
		return 1;
	}
	out->octree_size = res.octree.size();
	out->octree = (uint8_t*)malloc(res.octree.size() + 1);
	memcpy(out->octree, res.octree.data(), res.octree.size());
	out->hierarchy_size = res.hierarchy.size();
	out->hierarchy = (uint8_t*)malloc(res.hierarchy.size() + 1);
	memcpy(out->hierarchy, res.hierarchy.data(), res.hierarchy.size());
	out->metadata_size = res.metadata.size();
	out->metadata = (char*)malloc(res.metadata.size() + 1);
	memcpy(out->metadata, res.metadata.data(), res.metadata.size());
	out->metadata[res.metadata.size()] = 0;
	out->num_chunks = (int32_t)res.chunkIds.size();
	size_t idBytes = 0;
	for (auto& s : res.chunkIds) idBytes += s.size() + 1;
	out->chunk_ids = (char*)malloc(idBytes + 1);
	size_t p = 0;
	for (auto& s : res.chunkIds) { memcpy(out->chunk_ids + p, s.c_str(), s.size() + 1); p += s.size() + 1; }
	out->chunk_counts = (int64_t*)malloc(sizeof(int64_t) * (res.chunkCounts.size() + 1));
	for (size_t i = 0; i < res.chunkCounts.size(); i++) out->chunk_counts[i] = res.chunkCounts[i];
	out->num_nodes = (int64_t)res.nodes.size();
	size_t nameBytes = 0;
	for (auto& n : res.nodes) nameBytes += n.name.size() + 1;
	out->node_names = (char*)malloc(nameBytes + 1);
	out->node_info = (int64_t*)malloc(sizeof(int64_t) * 3 * (res.nodes.size() + 1));
	p = 0;
	for (size_t i = 0; i < res.nodes.size(); i++) {
		memcpy(out->node_names + p, res.nodes[i].name.c_str(), res.nodes[i].name.size() + 1);
		p += res.nodes[i].name.size() + 1;
		out->node_info[3 * i] = res.nodes[i].byteOffset;
		out->node_info[3 * i + 1] = res.nodes[i].byteSize;
		out->node_info[3 * i + 2] = res.nodes[i].numPoints;
	}
	return 0;
}

// decodeCount: X/Y/Z/cell hold the point count, grid 512^3 at most (the
// grid size used is returned); returns 0 or 1 with the message in err.
int pcref_decode_count(const void* las, uint64_t size, int32_t* X, int32_t* Y, int32_t* Z, uint32_t* cell, int64_t* grid,
                       int64_t grid_capacity, int64_t* grid_size, char* err) {
	std::vector<int64_t> g;
	std::string e;
	int64_t gs = 0;
	if (!pcref::decodeCount((const uint8_t*)las, size, X, Y, Z, cell, g, gs, e)) { snprintf(err, 256, "%s", e.c_str()); return 1; }
	if ((int64_t)g.size() > grid_capacity) { snprintf(err, 256, "grid capacity too small"); return 1; }
	memcpy(grid, g.data(), g.size() * sizeof(int64_t));
	*grid_size = gs;
	return 0;
}

int pcref_convert(const void* las, uint64_t size, const char* method, const char* name, uint32_t seed, pcref_output* out) {
	return pcref_convert_sources(&las, &size, 1, nullptr, 0, method, name, seed, out);
}

void pcref_free(pcref_output* out) {
	free(out->octree); free(out->hierarchy); free(out->metadata); free(out->chunk_ids); free(out->chunk_counts); free(out->node_names); free(out->node_info);
	memset(out, 0, sizeof(*out));
}

}  // extern "C"

// Test hooks: the library behaviour the samplers rely on, straight from
// libstdc++ (the same standard library the reference links).
extern "C" void pcref_std_sort_perm(const double* keys, int64_t n, int32_t* perm) {
	struct E { double k; int32_t i; };
	std::vector<E> v(n);
	for (int64_t i = 0; i < n; i++) v[i] = {keys[i], (int32_t)i};
	std::sort(v.begin(), v.end(), [](const E& a, const E& b) { return a.k < b.k; });
	for (int64_t i = 0; i < n; i++) perm[i] = v[i].i;
}

extern "C" void pcref_std_shuffle(int64_t n, uint32_t seed, int32_t* perm) {
	std::vector<int> v(n);
	for (int64_t i = 0; i < n; i++) v[i] = (int)i;
	std::shuffle(v.begin(), v.end(), std::default_random_engine(seed));
	for (int64_t i = 0; i < n; i++) perm[i] = v[i];
}

// ------------------------------------------------------------ stage hooks
// One stage of the pipeline at a time, for the parity tests of the library's
// stage entry points (include/pcgpu.h pcg_kernel_lut, _scatter, _octree,
// _accept). Each runs the restatement's own function of that stage.

// createLUT (chunker_countsort_laszip.cpp:1074-1204) of a count grid:
// chunks in file-name order (ids 16 bytes each, info: level, x, y, z,
// count), the LUT remapped to that order. Returns 1 when the chunk list
// exceeds capacity (*num_chunks = chunks found).
extern "C" int pcref_lut(const int64_t* grid, int64_t grid_size, int64_t max_points_per_chunk, int32_t* lut_out, char* ids_out,
                         int64_t* info_out, int64_t capacity, int64_t* num_chunks) {
	using namespace pcref;
	vector<int64_t> g(grid, grid + grid_size * grid_size * grid_size);
	vector<ChunkNode> nodes;
	vector<int32_t> lut;
	createLUT(g, grid_size, max_points_per_chunk, nodes, lut);
	*num_chunks = (int64_t)nodes.size();
	if ((int64_t)nodes.size() > capacity) return 1;
	vector<size_t> order(nodes.size());
	for (size_t i = 0; i < order.size(); i++) order[i] = i;
	std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return nodes[a].id + ".bin" < nodes[b].id + ".bin"; });
	vector<int32_t> rank(nodes.size());
	for (size_t r = 0; r < order.size(); r++) {
		const ChunkNode& n = nodes[order[r]];
		rank[order[r]] = (int32_t)r;
		memset(ids_out + 16 * r, 0, 16);
		memcpy(ids_out + 16 * r, n.id.c_str(), std::min<size_t>(n.id.size(), 15));
		int64_t level = (int64_t)n.id.size() - 1;
		info_out[5 * r] = level;
		info_out[5 * r + 1] = n.x;
		info_out[5 * r + 2] = n.y;
		info_out[5 * r + 3] = n.z;
		info_out[5 * r + 4] = n.numPoints;
	}
	for (size_t i = 0; i < lut.size(); i++) lut_out[i] = lut[i] < 0 ? -1 : rank[lut[i]];
	return 0;
}

// distributePoints' bucket fill (chunker_countsort_laszip.cpp:837-904, one
// chunker thread): point indices appended to their chunk in input order.
extern "C" int pcref_scatter(const uint32_t* cell, int64_t n, const int32_t* lut, int32_t num_chunks, uint32_t* ids_out,
                             int64_t* chunk_start) {
	std::vector<std::vector<uint32_t>> buckets(num_chunks);
	for (int64_t i = 0; i < n; i++) {
		int32_t k = lut[cell[i]];
		if (k < 0 || k >= num_chunks) return 1;
		buckets[k].push_back((uint32_t)i);
	}
	int64_t off = 0;
	for (int32_t k = 0; k < num_chunks; k++) {
		chunk_start[k] = off;
		memcpy(ids_out + off, buckets[k].data(), buckets[k].size() * sizeof(uint32_t));
		off += (int64_t)buckets[k].size();
	}
	chunk_start[num_chunks] = off;
	return 0;
}

namespace {

// Attributes of the stage hooks' records: position, then the point's input
// index (and rgb for the averaging sampler), so the points can be followed
// through the restatement's record shuffling.
pcref::Attributes hookAttributes(const double* scale, const double* offset, bool rgb) {
	using namespace pcref;
	vector<Attribute> list = {Attribute("position", 12, 3, 4, AType::INT32), Attribute("index", 4, 1, 4, AType::UINT32)};
	if (rgb) list.push_back(Attribute("rgb", 6, 3, 2, AType::UINT16));
	Attributes a(list);
	a.posScale = {scale[0], scale[1], scale[2]};
	a.posOffset = {offset[0], offset[1], offset[2]};
	return a;
}

void packRecord(uint8_t* p, int32_t X, int32_t Y, int32_t Z, uint32_t index) {
	memcpy(p, &X, 4); memcpy(p + 4, &Y, 4); memcpy(p + 8, &Z, 4); memcpy(p + 12, &index, 4);
}

}  // namespace

// buildHierarchy (indexer.cpp:823-1109) of one chunk: its subtree's nodes
// sorted by name (names 32 bytes each; info: start, count, is_leaf), point
// indices in the order the restatement leaves them.
extern "C" int pcref_octree(const int32_t* X, const int32_t* Y, const int32_t* Z, int64_t n, const double* scale, const double* offset,
                            const double* box_min, const double* box_max, const char* root_name, uint32_t* order_out, char* names_out,
                            int64_t* info_out, int64_t capacity, int64_t* num_nodes, int64_t* octree_depth) {
	using namespace pcref;
	Indexer indexer;
	indexer.attributes = hookAttributes(scale, offset, false);
	const int64_t bpp = indexer.attributes.bytes;
	auto points = std::make_shared<vector<uint8_t>>(n * bpp);
	for (int64_t i = 0; i < n; i++) packRecord(points->data() + i * bpp, X[i], Y[i], Z[i], (uint32_t)i);
	auto root = std::make_shared<Node>(root_name, Vec3{box_min[0], box_min[1], box_min[2]}, Vec3{box_max[0], box_max[1], box_max[2]});
	buildHierarchy(&indexer, root.get(), points, n);
	vector<Node*> all;
	traverseNode(root.get(), [&](Node* nd) { all.push_back(nd); });
	std::sort(all.begin(), all.end(), [](Node* a, Node* b) { return a->name < b->name; });
	*num_nodes = (int64_t)all.size();
	*octree_depth = indexer.octreeDepth;
	if ((int64_t)all.size() > capacity) return 1;
	int64_t off = 0;
	for (size_t k = 0; k < all.size(); k++) {
		Node* nd = all[k];
		memset(names_out + 32 * k, 0, 32);
		memcpy(names_out + 32 * k, nd->name.c_str(), std::min<size_t>(nd->name.size(), 31));
		const bool leaf = nd->isLeaf();
		int64_t cnt = (leaf && nd->points) ? nd->numPoints : 0;
		info_out[3 * k] = off;
		info_out[3 * k + 1] = cnt;
		info_out[3 * k + 2] = leaf ? 1 : 0;
		for (int64_t i = 0; i < cnt; i++) order_out[off + i] = rd<uint32_t>(nd->points->data() + i * bpp + 12);
		off += cnt;
	}
	for (int64_t i = off; i < n; i++) order_out[i] = 0xffffffffu;  // dropped by the duplicate rule
	return 0;
}

// One inner node sampled by the restatement's sampler (method 0 poisson, 1
// poisson_average, 2 random): the candidates are the children's points,
// child[] non-decreasing; the children count as already sampled (no leaf
// shuffle); the node is named "r" so its spacing is baseSpacing.
extern "C" int pcref_accept(int32_t method, const int32_t* X, const int32_t* Y, const int32_t* Z, const uint8_t* child, const uint16_t* rgb,
                            int64_t n, const double* scale, const double* offset, const double* box_min, const double* box_max,
                            double spacing, uint8_t* accepted_out, uint16_t* rgb_out) {
	using namespace pcref;
	Attributes attrs = hookAttributes(scale, offset, method == 1);
	const int64_t bpp = attrs.bytes;
	auto node = std::make_shared<Node>("r", Vec3{box_min[0], box_min[1], box_min[2]}, Vec3{box_max[0], box_max[1], box_max[2]});
	shared_ptr<Node> kids[8];
	for (int64_t i = 0; i < n; i++) {
		int c = child[i];
		if (c > 7 || (i > 0 && child[i - 1] > c)) return 1;
		if (!kids[c]) {
			kids[c] = std::make_shared<Node>();
			childBox(node->min, node->max, c, kids[c]->min, kids[c]->max);
			kids[c]->name = "r" + std::to_string(c);
			kids[c]->children.resize(8);
			kids[c]->points = std::make_shared<vector<uint8_t>>();
			kids[c]->sampled = true;
			node->children[c] = kids[c];
		}
		auto& buf = *kids[c]->points;
		size_t at = buf.size();
		buf.resize(at + bpp);
		packRecord(buf.data() + at, X[i], Y[i], Z[i], (uint32_t)i);
		if (method == 1) memcpy(buf.data() + at + 16, rgb + 3 * i, 6);
		kids[c]->numPoints++;
	}
	auto noop = [](Node*) {};
	memset(accepted_out, 0, n);
	if (method == 0) samplePoisson(node.get(), attrs, spacing, noop);
	else if (method == 1) samplePoissonAverage(node.get(), attrs, spacing, noop);
	else {
		// the random sampler's visit counter: this node is the thread's first
		sampleRandom(node.get(), attrs, 0, noop);
	}
	for (int64_t i = 0; i < node->numPoints; i++) accepted_out[rd<uint32_t>(node->points->data() + i * bpp + 12)] = 1;
	if (method == 1 && rgb_out) {
		// every candidate's record carries the averaged colour (:440-445);
		// the children were given their rejected and kept points
		for (int c = 0; c < 8; c++) {
			if (!kids[c] || !kids[c]->points) continue;
			const auto& buf = *kids[c]->points;
			for (size_t k = 0; k + bpp <= buf.size(); k += bpp) memcpy(rgb_out + 3 * rd<uint32_t>(buf.data() + k + 12), buf.data() + k + 16, 6);
		}
	}
	return 0;
}
