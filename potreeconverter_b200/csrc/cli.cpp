// PotreeConverter-compatible command line (flags of main.cpp:21-145):
//
//   PotreeConverter <source> [<source> ...] -o <outdir>
//                   [-m poisson|poisson_average|random]
//                   [--attributes <name> ...] [--projection <string>]
//                   [--encoding DEFAULT] [--plain] [--device N] [--seed N]
//
// Sources are LAS files or directories of them, taken like the reference's
// curateSources (main.cpp:146-200; directory entries in name order); all
// are converted as one point cloud named after the first source's stem.
// --attributes keeps "position" and the named attributes, in that order
// (PotreeConverter.h:252-275). Writes octree.bin, hierarchy.bin and
// metadata.json through libpcgpu. --plain selects the one-launch-per-node
// form; --seed sets the random sampler's leaf-shuffle seed (the pinned
// reference uses 1592614637). Flags of the reference that this build does
// not implement (BROTLI encoding, page generation) are rejected.

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "pcgpu.h"

namespace fs = std::filesystem;

static int usage() {
	fprintf(stderr, "PotreeConverter <source> [<source> ...] -o <outdir> [-m poisson|poisson_average|random] [--attributes a ...] [--projection P] [--plain]\n");
	return 1;
}

static bool ends_with_ci(const std::string& s, const char* suffix) {  // iEndsWith (unsuck.hpp)
	const size_t n = std::strlen(suffix);
	if (s.size() < n) return false;
	for (size_t i = 0; i < n; i++)
		if (std::tolower((unsigned char)s[s.size() - n + i]) != std::tolower((unsigned char)suffix[i])) return false;
	return true;
}

int main(int argc, char** argv) {
	std::vector<std::string> source, attributes;
	std::string outdir, method = "poisson", encoding = "DEFAULT", projection;
	pcg_opts opts{0, 1592614637u, PCG_FORM_BATCHED, PCG_RECORDS_AUTO, nullptr, 0};
	bool in_attributes = false;
	for (int i = 1; i < argc; i++) {
		std::string a = argv[i];
		auto val = [&]() -> std::string {
			if (i + 1 >= argc) { fprintf(stderr, "missing value for %s\n", a.c_str()); exit(1); }
			return argv[++i];
		};
		if (!a.empty() && a[0] == '-') in_attributes = false;
		if (a == "-h" || a == "--help") return usage() ? 0 : 0;
		else if (a == "-i" || a == "--source") source.push_back(val());
		else if (a == "-o" || a == "--outdir") outdir = val();
		else if (a == "-m" || a == "--method") method = val();
		else if (a == "--encoding") encoding = val();
		else if (a == "--projection") projection = val();
		else if (a == "--attributes") in_attributes = true;
		else if (a == "--plain") opts.form = PCG_FORM_PLAIN;
		else if (a == "--device") opts.device = atoi(val().c_str());
		else if (a == "--seed") opts.random_seed = (uint32_t)strtoul(val().c_str(), nullptr, 10);
		else if (a == "--chunkMethod") { if (val() != "LASZIP") { fprintf(stderr, "only --chunkMethod LASZIP is supported\n"); return 1; } }
		else if (a == "-p" || a == "--generate-page" || a == "--title") { fprintf(stderr, "%s is not supported by this build\n", a.c_str()); return 1; }
		else if (a == "--keep-chunks" || a == "--no-chunking" || a == "--no-indexing") { fprintf(stderr, "%s is not supported (no chunk files are written)\n", a.c_str()); return 1; }
		else if (!a.empty() && a[0] == '-') { fprintf(stderr, "unknown flag %s\n", a.c_str()); return 1; }
		else if (in_attributes) attributes.push_back(a);
		else source.push_back(a);
	}
	if (source.empty()) return usage();
	if (encoding != "DEFAULT" && encoding != "UNCOMPRESSED") { fprintf(stderr, "encoding %s is not supported\n", encoding.c_str()); return 1; }
	int m = method == "poisson" ? PCG_POISSON : method == "poisson_average" ? PCG_POISSON_AVERAGE : method == "random" ? PCG_RANDOM : -1;
	if (m < 0) { fprintf(stderr, "unknown method %s\n", method.c_str()); return 1; }
	if (!fs::exists(source[0])) { fprintf(stderr, "file does not exist: %s\n", source[0].c_str()); return 123; }
	if (outdir.empty()) outdir = source[0] + "/../" + fs::path(source[0]).filename().string() + "_converted";  // main.cpp:64-101
	// curateSources, main.cpp:146-200
	std::string name;
	std::vector<std::string> paths;
	for (auto& path : source) {
		if (fs::is_directory(path)) {
			std::vector<std::string> entries;
			for (auto& e : fs::directory_iterator(path)) {
				std::string str = e.path().string();
				if (ends_with_ci(str, "las") || ends_with_ci(str, "laz")) entries.push_back(str);
			}
			std::sort(entries.begin(), entries.end());
			paths.insert(paths.end(), entries.begin(), entries.end());
		} else if (fs::is_regular_file(path)) {
			if (ends_with_ci(path, "las") || ends_with_ci(path, "laz")) paths.push_back(path);
		}
		if (name.empty()) name = fs::path(path).stem().string();
	}
	if (paths.empty()) { fprintf(stderr, "no LAS input among the sources\n"); return 1; }
	std::vector<std::vector<uint8_t>> images;
	for (auto& path : paths) {
		std::ifstream f(path, std::ios::binary);
		images.emplace_back((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
	}
	std::vector<pcg_source> srcs;
	for (auto& img : images) srcs.push_back({img.data(), img.size(), nullptr});
	std::vector<const char*> attr_names;
	for (auto& a : attributes) attr_names.push_back(a.c_str());

	pcg_ctx* ctx = nullptr;
	pcg_status st = pcg_create(&ctx, &opts);
	if (st != PCG_OK) { fprintf(stderr, "pcg_create failed: %s\n", pcg_status_string(st)); return 1; }
	pcg_job job{};
	job.method = m;
	job.name = name.c_str();
	job.projection = projection.c_str();
	job.num_sources = (int32_t)srcs.size();
	job.sources = srcs.data();
	job.num_attributes = (int32_t)attr_names.size();
	job.attributes = attr_names.empty() ? nullptr : attr_names.data();
	pcg_result res{};
	st = pcg_convert(ctx, &job, &res);
	if (st != PCG_OK) {
		fprintf(stderr, "conversion failed (%s): %s\n", pcg_status_string(st), pcg_last_error(ctx));
		pcg_destroy(ctx);
		return st == PCG_OUT_OF_BOX ? 123 : 1;
	}
	fs::create_directories(outdir);
	st = pcg_write_files(&res, outdir.c_str());
	const pcg_stats& s = res.stats;
	printf("#points: %lld, #chunks: %lld, #nodes: %lld, depth: %lld\n", (long long)s.num_points, (long long)s.num_chunks,
	       (long long)s.num_nodes, (long long)s.octree_depth);
	printf("duration: %.3f ms (h2d %.2f, chunking %.2f, octree %.2f, sampling %.2f, output %.2f, d2h %.2f, writers %.2f)\n", s.ms_total,
	       s.ms_h2d, s.ms_chunking, s.ms_octree, s.ms_sampling, s.ms_output, s.ms_d2h, s.ms_host_writers);
	printf("throughput: %.1f Mpts/s, kernel launches: %lld, escalated FP64 pairs: %lld\n", s.num_points / (s.ms_total * 1e3),
	       (long long)s.gpu_launches, (long long)s.escalated_pairs);
	pcg_result_free(&res);
	pcg_destroy(ctx);
	return st == PCG_OK ? 0 : 1;
}
