// Host build of the library's set-up (potreeconverter_b200/csrc/setup.cpp)
// for the CPU tests: parses the given LAS/LAZ files as one job, applies an
// --attributes list, and prints the resulting schema as JSON (or the error).
//   setup_check <file> [<file> ...] [--attributes <name> ...]
#include <cstdio>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "pcg_internal.h"

static std::string esc(const std::string& s) {
	std::string o;
	for (char c : s) {
		if (c == '"' || c == '\\') o += '\\';
		o += c;
	}
	return o;
}

int main(int argc, char** argv) {
	std::vector<std::string> files, attrs;
	bool in_attrs = false;
	for (int i = 1; i < argc; i++) {
		std::string a = argv[i];
		if (a == "--attributes") in_attrs = true;
		else if (in_attrs) attrs.push_back(a);
		else files.push_back(a);
	}
	std::vector<pcg::LasInfo> infos;
	std::string err;
	for (auto& f : files) {
		std::ifstream in(f, std::ios::binary);
		std::vector<uint8_t> b((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
		pcg::LasInfo info;
		if (!pcg::parse_las(b.data(), b.size(), info, err)) {
			printf("{\"error\": \"%s\"}\n", esc(err).c_str());
			return 0;
		}
		infos.push_back(info);
	}
	pcg::Setup s;
	if (!pcg::make_setup(infos, attrs, s, err)) {
		printf("{\"error\": \"%s\"}\n", esc(err).c_str());
		return 0;
	}
	printf("{\"bpp\": %d, \"points\": %lld, \"scale\": [%.17g, %.17g, %.17g], \"offset\": [%.17g, %.17g, %.17g],\n", s.bpp,
	       (long long)s.total_points, s.pos_scale.x, s.pos_scale.y, s.pos_scale.z, s.pos_offset.x, s.pos_offset.y, s.pos_offset.z);
	printf(" \"min\": [%.17g, %.17g, %.17g], \"max\": [%.17g, %.17g, %.17g], \"grid\": %d, \"chunk_capacity\": %d,\n", s.cube_min.x,
	       s.cube_min.y, s.cube_min.z, s.root_max.x, s.root_max.y, s.root_max.z, s.grid_size, s.max_points_per_chunk);
	printf(" \"attributes\": [");
	for (size_t i = 0; i < s.attrs.size(); i++)
		printf("%s{\"name\": \"%s\", \"size\": %d, \"offset\": %d, \"type\": \"%s\"}", i ? ", " : "", esc(s.attrs[i].name).c_str(),
		       s.attrs[i].size, s.attrs[i].out_offset, pcg::attr_type_name(s.attrs[i].type));
	printf("],\n \"sources\": [");
	for (size_t k = 0; k < s.sources.size(); k++) {
		const auto& src = s.sources[k];
		printf("%s{\"points\": %lld, \"compressed\": %s, \"laz_chunks\": %zu, \"zero_fill\": %s, \"extras\": [", k ? ", " : "",
		       (long long)src.las.num_points, src.las.compressed ? "true" : "false", src.las.laz_chunks.size(),
		       src.zero_fill ? "true" : "false");
		for (size_t e = 0; e < src.extras.size(); e++)
			printf("%s[%d, %d, %d, %d]", e ? ", " : "", src.extras[e].src_off, src.extras[e].dst_off, src.extras[e].size,
			       src.extras[e].out_index);
		printf("]}");
	}
	printf("]}\n");
	return 0;
}
