// Internal declarations shared by the host orchestration (C++) and the CUDA
// kernels of libpcgpu. Nothing here is part of the C ABI.
#pragma once

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "laz.cuh"

namespace pcg {

// ---------------------------------------------------------------- geometry
// FP64 3-vector whose operators evaluate exactly like the reference's
// Vector3 (Vector3.h:65-87): component-wise, no fused multiply-add.
struct Vec3d {
	double x = 0.0, y = 0.0, z = 0.0;
	Vec3d() {}
	Vec3d(double x_, double y_, double z_) : x(x_), y(y_), z(z_) {}
	double maxc() const { return x > y ? (x > z ? x : z) : (y > z ? y : z); }
	Vec3d operator-(const Vec3d& r) const { return {x - r.x, y - r.y, z - r.z}; }
	Vec3d operator+(const Vec3d& r) const { return {x + r.x, y + r.y, z + r.z}; }
	Vec3d operator+(double s) const { return {x + s, y + s, z + s}; }
	Vec3d operator*(double s) const { return {x * s, y * s, z * s}; }
};

// std::max(std::max(x, y), z) as Vector3::max() (Vector3.h:60-63)
inline double vmax3(const Vec3d& v) {
	double a = (v.x < v.y) ? v.y : v.x;
	return (a < v.z) ? v.z : a;
}

// Octant box of a node, childBoundingBoxOf (converter_utils.h:106-136).
inline void child_box(const Vec3d& mn, const Vec3d& mx, int index, Vec3d& omin, Vec3d& omax) {
	Vec3d size = mx - mn;
	Vec3d center = mn + (size * 0.5);
	if ((index & 4) == 0) { omin.x = mn.x; omax.x = center.x; } else { omin.x = center.x; omax.x = mx.x; }
	if ((index & 2) == 0) { omin.y = mn.y; omax.y = center.y; } else { omin.y = center.y; omax.y = mx.y; }
	if ((index & 1) == 0) { omin.z = mn.z; omax.z = center.z; } else { omin.z = center.z; omax.z = mx.z; }
}

// ------------------------------------------------------------- attributes
enum class AttrType : int { INT8 = 0, INT16 = 1, INT32 = 2, INT64 = 3, UINT8 = 10, UINT16 = 11, UINT32 = 12, UINT64 = 13, FLOAT = 20, DOUBLE = 21, UNDEFINED = 123456 };

const char* attr_type_name(AttrType t);
int attr_type_size(AttrType t);

// Which decode rule fills an output attribute (chunker_countsort_laszip.cpp:391-545).
enum AttrKind : int {
	AK_POSITION = 0, AK_INTENSITY, AK_RETURN_NUMBER, AK_NUMBER_OF_RETURNS, AK_CLASSIFICATION,
	AK_SCAN_ANGLE_RANK, AK_USER_DATA, AK_POINT_SOURCE_ID, AK_GPS_TIME, AK_RGB, AK_EXTRA
};

struct AttrDesc {
	std::string name, description;
	int size = 0, numElements = 0, elementSize = 0;
	AttrType type = AttrType::UNDEFINED;
	Vec3d scale = {1, 1, 1}, offset = {0, 0, 0};
	int kind = AK_EXTRA;
	int out_offset = 0;   // byte offset in the output record
	int src_offset = 0;   // byte offset in the LAS record (extra bytes)
};

struct LasInfo {
	int version_minor = 0;
	int pdrf = -1;
	int record_length = 0;
	uint64_t offset_to_points = 0;
	int64_t num_points = 0;
	Vec3d scale, offset, min, max;
	struct Vlr { uint16_t record_id; std::vector<uint8_t> data; };
	std::vector<Vlr> vlrs;
	// LAZ (point format with a compression bit): record layout and chunks
	bool compressed = false;
	laz::Layout laz_layout{};
	std::vector<laz::Chunk> laz_chunks;
};

// One input file as the chunker's attribute handlers see it
// (createAttributeHandlers, chunker_countsort_laszip.cpp:380-658, built per
// source from its own attribute list, :952-983).
struct SourceSetup {
	LasInfo las;
	std::vector<AttrDesc> attrs;    // the source's own attribute list (PotreeConverter.h:136-193)
	int std_record_length = 0;      // LAS record bytes before extra bytes
	// extra-bytes handlers (:579-653): `size` bytes from LAS record offset
	// src_off to output offset dst_off; statistics go to output attribute
	// out_index, read with that attribute's type and element layout
	struct Extra { int src_off, dst_off, size, out_index; };
	std::vector<Extra> extras;
	bool zero_fill = false;         // some output bytes stay zero (memset, :729-732)
};

// All FP64 set-up the reference performs on the host before chunking, for
// the sources in the order given: output attribute schema (union by name,
// then the --attributes filter, PotreeConverter.h:195-276), scale/offset
// (PotreeConverter.h:29-76), cubic box (main.cpp:215-284), chunk grid size
// and chunk capacity (chunker_countsort_laszip.cpp:1210-1220).
struct Setup {
	std::vector<SourceSetup> sources;
	std::vector<AttrDesc> attrs;    // output attributes
	int bpp = 0;
	Vec3d pos_scale, pos_offset;
	Vec3d cube_min, cube_max;       // max = min + cubeSize (main.cpp:237-239)
	double chunk_cube_size = 0;     // (max - min).max(), recomputed (chunker :205-207)
	Vec3d root_max;                 // chunk metadata max (chunker :1252-1254)
	int64_t total_points = 0;
	int grid_size = 128;
	int max_points_per_chunk = 0;   // min(total/20, 10M) as int
};

// points_elsewhere: the point records are not part of this buffer (they are
// already in device memory), so only the header and VLRs must be present.
bool parse_las(const uint8_t* las, uint64_t size, LasInfo& info, std::string& err, bool points_elsewhere = false);
// requested: the --attributes names (empty: every attribute). Jobs whose
// result the reference leaves undefined are refused with a message.
bool make_setup(const std::vector<LasInfo>& sources, const std::vector<std::string>& requested, Setup& s, std::string& err);
inline bool make_setup(const LasInfo& info, Setup& s, std::string& err) { return make_setup(std::vector<LasInfo>{info}, {}, s, err); }

// ---------------------------------------------------------- device params
struct ExtraDesc {
	int src_off, dst_off, size, type, num_elements, element_size, stat_index, pad;
};

constexpr int MAX_EXTRA = 16;
constexpr int MAX_ATTRS = 32;

// One input file on the device: where its records are, how its coordinates
// decode, and which bytes its handlers move.
struct SourceDesc {
	double in_scale[3], in_offset[3];
	const uint8_t* recs;  // device pointer to its first point record
	int64_t first;        // job index of its first point
	int64_t count;        // its points
	int rec_len;
	int src_gps, src_rgb; // record offsets of GPS time / RGB, -1 when absent
	int zero_fill;        // output bytes not written by its handlers stay zero
	int n_extra, pad;
	ExtraDesc extra[MAX_EXTRA];
};

struct DecodeParams {
	double pos_scale[3], pos_offset[3];
	double cmin[3];
	double csize;         // chunk_cube_size
	int64_t n;            // points over all sources
	int bpp, grid;
	// output offsets of the standard attributes, -1 when not in the output
	int off_intensity, off_retnum, off_nret, off_class, off_sar, off_user, off_psid, off_gps, off_rgb;
	int stat_intensity, stat_retnum, stat_nret, stat_class, stat_sar, stat_user, stat_psid, stat_gps, stat_rgb, stat_pos;
	int nsrc;             // sources; kernels for one source read src0
	int max_rec_len;
	const SourceDesc* srcs;     // device table of the nsrc sources
	const int64_t* src_first;   // device: first job index of every source
	SourceDesc src0;
};

// Attribute statistics as order-preserving uint64 encodings of doubles.
struct AttrStatsDev {
	unsigned long long mn[3];
	unsigned long long mx[3];
};

}  // namespace pcg
