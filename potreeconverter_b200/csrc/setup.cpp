// Host-side FP64 set-up: LAS header, attribute schema, scale/offset, cubic
// bounding box and chunk-grid parameters, evaluated with the same
// expressions (and therefore the same rounding) as the reference.

#include <algorithm>
#include <cmath>
#include <cstring>

#include "pcg_internal.h"

namespace pcg {

const char* attr_type_name(AttrType t) {  // Attributes.h:51-78
	switch (t) {
	case AttrType::INT8: return "int8";
	case AttrType::INT16: return "int16";
	case AttrType::INT32: return "int32";
	case AttrType::INT64: return "int64";
	case AttrType::UINT8: return "uint8";
	case AttrType::UINT16: return "uint16";
	case AttrType::UINT32: return "uint32";
	case AttrType::UINT64: return "uint64";
	case AttrType::FLOAT: return "float";
	case AttrType::DOUBLE: return "double";
	case AttrType::UNDEFINED: return "undefined";
	}
	return "error";
}

int attr_type_size(AttrType t) {  // Attributes.h:33-49
	switch (t) {
	case AttrType::UINT8: case AttrType::INT8: return 1;
	case AttrType::UINT16: case AttrType::INT16: return 2;
	case AttrType::UINT32: case AttrType::INT32: case AttrType::FLOAT: return 4;
	case AttrType::UINT64: case AttrType::INT64: case AttrType::DOUBLE: return 8;
	default: return 0;
	}
}

template <class T> static T get(const uint8_t* p) { T v; std::memcpy(&v, p, sizeof(T)); return v; }

// Header fields as LASzip reports them (LasLoader.cpp:72-128); for a LAZ
// file (point format with a compression bit) also the laszip record and
// the chunk table.
bool parse_las(const uint8_t* las, uint64_t size, LasInfo& info, std::string& err, bool points_elsewhere) {
	if (size < 227 || std::memcmp(las, "LASF", 4) != 0) { err = "input is not a LAS file"; return false; }
	info.version_minor = las[25];
	uint16_t header_size = get<uint16_t>(las + 94);
	info.offset_to_points = get<uint32_t>(las + 96);
	uint32_t num_vlrs = get<uint32_t>(las + 100);
	uint8_t fmt = las[104];
	info.compressed = (fmt & 0xC0) != 0;  // LASzip marks compressed formats with bit 7 (6 in old files)
	info.pdrf = fmt & 0x3f;
	info.record_length = get<uint16_t>(las + 105);
	uint64_t legacy = get<uint32_t>(las + 107);
	info.scale = {get<double>(las + 131), get<double>(las + 139), get<double>(las + 147)};
	info.offset = {get<double>(las + 155), get<double>(las + 163), get<double>(las + 171)};
	info.max.x = get<double>(las + 179); info.min.x = get<double>(las + 187);
	info.max.y = get<double>(las + 195); info.min.y = get<double>(las + 203);
	info.max.z = get<double>(las + 211); info.min.z = get<double>(las + 219);
	uint64_t ext = 0;
	if (info.version_minor >= 4 && header_size >= 375 && size >= 255) ext = get<uint64_t>(las + 247);
	const uint64_t count = ext > legacy ? ext : legacy;  // LasLoader.cpp:103
	if (count > (uint64_t(1) << 40)) { err = "implausible point count in the LAS header"; return false; }
	info.num_points = (int64_t)count;
	uint64_t pos = header_size;
	const uint8_t* laszip_vlr = nullptr;
	uint32_t laszip_len = 0;
	for (uint32_t i = 0; i < num_vlrs; i++) {
		if (pos + 54 > size) { err = "truncated variable length record"; return false; }
		LasInfo::Vlr v;
		v.record_id = get<uint16_t>(las + pos + 18);
		uint16_t len = get<uint16_t>(las + pos + 20);
		if (pos + 54 + len > size) { err = "truncated variable length record"; return false; }
		v.data.assign(las + pos + 54, las + pos + 54 + len);
		if (v.record_id == 22204 && std::memcmp(las + pos + 2, "laszip encoded", 14) == 0) {
			laszip_vlr = las + pos + 54;
			laszip_len = len;
		}
		info.vlrs.push_back(std::move(v));
		pos += 54 + len;
	}
	if (info.compressed) {
		// the chunk table is read unless the records are already decoded
		if (points_elsewhere) return true;
		return laz::parse_table(las, size, info.offset_to_points, info.num_points, info.pdrf, info.record_length, laszip_vlr, laszip_len,
		                        info.laz_layout, info.laz_chunks, err);
	}
	// offset + count x record length <= size, without overflow
	if (!points_elsewhere && info.num_points > 0 &&
	    (info.offset_to_points > size || info.record_length == 0 ||
	     (uint64_t)info.num_points > (size - info.offset_to_points) / (uint64_t)info.record_length)) {
		err = "truncated point data";
		return false;
	}
	return true;
}

static void las_type_info(int type_id, AttrType& type, int& num_elements) {  // LasLoader.cpp:7-69
	static const AttrType base[] = {AttrType::UNDEFINED, AttrType::UINT8, AttrType::INT8, AttrType::UINT16, AttrType::INT16,
	                                AttrType::UINT32, AttrType::INT32, AttrType::UINT64, AttrType::INT64, AttrType::FLOAT, AttrType::DOUBLE};
	if (type_id == 0) { type = AttrType::UNDEFINED; num_elements = 1; return; }
	type = base[(type_id - 1) % 10 + 1];
	num_elements = type_id <= 10 ? 1 : (type_id <= 20 ? 2 : 3);
}

// The source's own attribute list (PotreeConverter.h:136-193): the
// standard attributes of its point format, then its extra bytes
// (PotreeConverter.h:80-133) with their record offsets.
static bool source_attributes(const LasInfo& info, SourceSetup& src, std::string& err) {
	auto mk = [](const char* name, int size, int ne, int es, AttrType t, int kind) {
		AttrDesc a; a.name = name; a.size = size; a.numElements = ne; a.elementSize = es; a.type = t; a.kind = kind; return a;
	};
	AttrDesc xyz = mk("position", 12, 3, 4, AttrType::INT32, AK_POSITION);
	AttrDesc intensity = mk("intensity", 2, 1, 2, AttrType::UINT16, AK_INTENSITY);
	AttrDesc retnum = mk("return number", 1, 1, 1, AttrType::UINT8, AK_RETURN_NUMBER);
	AttrDesc nret = mk("number of returns", 1, 1, 1, AttrType::UINT8, AK_NUMBER_OF_RETURNS);
	AttrDesc cls = mk("classification", 1, 1, 1, AttrType::UINT8, AK_CLASSIFICATION);
	AttrDesc sar = mk("scan angle rank", 1, 1, 1, AttrType::UINT8, AK_SCAN_ANGLE_RANK);
	AttrDesc user = mk("user data", 1, 1, 1, AttrType::UINT8, AK_USER_DATA);
	AttrDesc psid = mk("point source id", 2, 1, 2, AttrType::UINT16, AK_POINT_SOURCE_ID);
	AttrDesc gps = mk("gps-time", 8, 1, 8, AttrType::DOUBLE, AK_GPS_TIME);
	AttrDesc rgb = mk("rgb", 6, 3, 2, AttrType::UINT16, AK_RGB);
	src.las = info;
	switch (info.pdrf) {
	case 0: src.attrs = {xyz, intensity, retnum, nret, cls, sar, user, psid}; src.std_record_length = 20; break;
	case 1: src.attrs = {xyz, intensity, retnum, nret, cls, sar, user, psid, gps}; src.std_record_length = 28; break;
	case 2: src.attrs = {xyz, intensity, retnum, nret, cls, sar, user, psid, rgb}; src.std_record_length = 26; break;
	case 3: src.attrs = {xyz, intensity, retnum, nret, cls, sar, user, psid, gps, rgb}; src.std_record_length = 34; break;
	default: err = "unsupported LAS point data format " + std::to_string(info.pdrf) + " (0-3 are supported)"; return false;
	}
	if (info.record_length < src.std_record_length) { err = "point record length shorter than its format"; return false; }
	const size_t n_standard = src.attrs.size();
	int off = src.std_record_length;
	for (auto& vlr : info.vlrs) {
		if (vlr.record_id != 4) continue;
		int num = (int)vlr.data.size() / 192;
		for (int i = 0; i < num; i++) {
			const uint8_t* r = vlr.data.data() + i * 192;
			char name[33] = {0}, desc[33] = {0};
			std::memcpy(name, r + 4, 32);
			std::memcpy(desc, r + 160, 32);
			AttrType t; int ne;
			las_type_info(r[2], t, ne);
			int es = attr_type_size(t);
			AttrDesc a = mk(name, ne * es, ne, es, t, AK_EXTRA);
			a.description = desc;
			if (r[3] & 0b01000) std::memcpy(&a.scale, r + 112, 24);
			if (r[3] & 0b10000) std::memcpy(&a.offset, r + 136, 24);
			a.src_offset = off;
			off += a.size;
			// an extra named like a standard attribute would also receive
			// that attribute's handler (:531-545); not supported
			for (size_t k = 0; k < n_standard; k++)
				if (src.attrs[k].name == a.name) { err = "extra-bytes attribute named like a standard attribute: " + a.name; return false; }
			src.attrs.push_back(a);
		}
	}
	if (off > info.record_length) { err = "extra bytes exceed the point record length"; return false; }
	return true;
}

bool make_setup(const std::vector<LasInfo>& infos, const std::vector<std::string>& requested, Setup& s, std::string& err) {
	if (infos.empty()) { err = "no input"; return false; }
	// computeOutputAttributes(sources, requestedAttributes), PotreeConverter.h:195-276
	const double inf = INFINITY;
	Vec3d scale_min = {inf, inf, inf}, mn = {inf, inf, inf}, mx = {-inf, -inf, -inf};
	std::vector<AttrDesc> full;
	s.sources.assign(infos.size(), SourceSetup{});
	s.total_points = 0;
	for (size_t k = 0; k < infos.size(); k++) {
		const LasInfo& info = infos[k];
		SourceSetup& src = s.sources[k];
		if (!source_attributes(info, src, err)) {
			if (infos.size() > 1) err = "source " + std::to_string(k) + ": " + err;
			return false;
		}
		for (auto& a : src.attrs) {  // union by name, first seen first
			bool added = false;
			for (auto& f : full) added = added || f.name == a.name;
			if (!added) full.push_back(a);
		}
		scale_min.x = std::min(scale_min.x, info.scale.x); scale_min.y = std::min(scale_min.y, info.scale.y); scale_min.z = std::min(scale_min.z, info.scale.z);
		mn.x = std::min(mn.x, info.min.x); mn.y = std::min(mn.y, info.min.y); mn.z = std::min(mn.z, info.min.z);
		mx.x = std::max(mx.x, info.max.x); mx.y = std::max(mx.y, info.max.y); mx.z = std::max(mx.z, info.max.z);
		s.total_points += info.num_points;
	}
	// the filter (:252-275): "position" first, then every requested name
	// found in the full list, in request order
	if (requested.empty()) {
		s.attrs = full;
	} else {
		std::vector<std::string> should = requested;
		should.insert(should.begin(), "position");
		for (size_t i = 0; i < should.size(); i++)
			for (size_t j = 0; j < i; j++)
				if (should[i] == should[j]) { err = "attribute listed twice: " + should[i]; return false; }
		s.attrs.clear();
		for (auto& name : should)
			for (auto& f : full)
				if (f.name == name) { s.attrs.push_back(f); break; }
	}
	int out_off = 0;
	for (auto& a : s.attrs) { a.out_offset = out_off; out_off += a.size; }
	s.bpp = out_off;
	auto out_index = [&](const std::string& name) {
		for (size_t i = 0; i < s.attrs.size(); i++) if (s.attrs[i].name == name) return (int)i;
		return -1;
	};

	// each source's handlers (:380-658): standard attributes go to their
	// output offsets; extra bytes kept in the output go to the source's
	// standard size plus the sizes of the kept extras before them (:565-653)
	for (auto& src : s.sources) {
		std::vector<bool> written(s.bpp, false);
		for (int b = 0; b < 12; b++) written[b] = true;
		int attribute_offset = 0;
		size_t first_extra = 0;
		for (auto& a : src.attrs) {
			if (a.kind == AK_EXTRA) break;
			attribute_offset += a.size;
			first_extra++;
		}
		for (size_t k = 1; k < first_extra; k++) {
			int oi = out_index(src.attrs[k].name);
			if (oi < 0) continue;
			for (int b = 0; b < s.attrs[oi].size; b++) written[s.attrs[oi].out_offset + b] = true;
		}
		for (size_t k = first_extra; k < src.attrs.size(); k++) {
			const AttrDesc& ia = src.attrs[k];
			int oi = out_index(ia.name);
			if (oi < 0) continue;
			const AttrDesc& oa = s.attrs[oi];
			if (attribute_offset + ia.size > s.bpp) {
				err = "attribute " + ia.name + " would be written past the point record (the reference's result is undefined)";
				return false;
			}
			if (ia.src_offset + oa.numElements * oa.elementSize > src.las.record_length) {
				err = "attribute " + ia.name + " would be read past the LAS record (the reference's result is undefined)";
				return false;
			}
			src.extras.push_back({ia.src_offset, attribute_offset, ia.size, oi});
			for (int b = 0; b < ia.size; b++) written[attribute_offset + b] = true;
			attribute_offset += oa.size;
		}
		src.zero_fill = false;
		for (bool w : written) src.zero_fill = src.zero_fill || !w;
	}
	// computeScaleOffset(min, max, scaleMin), PotreeConverter.h:29-76
	Vec3d size = mx - mn;
	double msx = size.x / std::pow(2.0, 30.0), msy = size.y / std::pow(2.0, 30.0), msz = size.z / std::pow(2.0, 30.0);
	s.pos_scale = {scale_min.x < msx ? msx : scale_min.x, scale_min.y < msy ? msy : scale_min.y, scale_min.z < msz ? msz : scale_min.z};
	s.pos_offset = mn;
	// computeStats, main.cpp:215-284, over the same header boxes
	double cube = vmax3(mx - mn);
	if (cube == 0.0) { err = "invalid bounding box: at least one axis has a size of zero"; return false; }
	s.cube_min = mn;
	s.cube_max = mn + cube;
	if ((s.cube_max - mn).x == 0.0) { err = "invalid bounding box"; return false; }
	// main.cpp:273-281 rejects a box with any zero-size cubic axis
	s.chunk_cube_size = vmax3(s.cube_max - s.cube_min);  // chunker_countsort_laszip.cpp:205-207
	s.root_max = s.cube_min + vmax3(s.cube_max - s.cube_min);  // :1252-1254
	int64_t t20 = s.total_points / 20;
	s.max_points_per_chunk = (int)(t20 < 10'000'000 ? t20 : 10'000'000);
	s.grid_size = s.total_points < 100'000'000 ? 128 : (s.total_points < 500'000'000 ? 256 : 512);
	return true;
}

}  // namespace pcg
