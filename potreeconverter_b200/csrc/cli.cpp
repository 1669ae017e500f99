// PotreeConverter-compatible command line (flags of main.cpp:21-145):
//
//   PotreeConverter <input.las> -o <outdir> [-m poisson|poisson_average|random]
//                   [--projection <string>] [--encoding DEFAULT]
//                   [--plain] [--device N] [--seed N]
//
// Writes octree.bin, hierarchy.bin and metadata.json through libpcgpu.
// --plain selects the one-launch-per-node form; --seed sets the random
// sampler's leaf-shuffle seed (the pinned reference uses 1592614637).
// Flags of the reference that this build does not implement (BROTLI
// encoding, --attributes filtering, page generation) are rejected.

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
	fprintf(stderr, "PotreeConverter <source> -o <outdir> [-m poisson|poisson_average|random] [--projection P] [--plain]\n");
	return 1;
}

int main(int argc, char** argv) {
	std::string source, outdir, method = "poisson", encoding = "DEFAULT", projection;
	pcg_opts opts{0, 1592614637u, PCG_FORM_BATCHED, 0};
	for (int i = 1; i < argc; i++) {
		std::string a = argv[i];
		auto val = [&]() -> std::string {
			if (i + 1 >= argc) { fprintf(stderr, "missing value for %s\n", a.c_str()); exit(1); }
			return argv[++i];
		};
		if (a == "-h" || a == "--help") return usage() ? 0 : 0;
		else if (a == "-i" || a == "--source") source = val();
		else if (a == "-o" || a == "--outdir") outdir = val();
		else if (a == "-m" || a == "--method") method = val();
		else if (a == "--encoding") encoding = val();
		else if (a == "--projection") projection = val();
		else if (a == "--plain") opts.form = PCG_FORM_PLAIN;
		else if (a == "--device") opts.device = atoi(val().c_str());
		else if (a == "--seed") opts.random_seed = (uint32_t)strtoul(val().c_str(), nullptr, 10);
		else if (a == "--chunkMethod") { if (val() != "LASZIP") { fprintf(stderr, "only --chunkMethod LASZIP is supported\n"); return 1; } }
		else if (a == "--attributes" || a == "-p" || a == "--generate-page" || a == "--title") { fprintf(stderr, "%s is not supported by this build\n", a.c_str()); return 1; }
		else if (a == "--keep-chunks" || a == "--no-chunking" || a == "--no-indexing") { fprintf(stderr, "%s is not supported (no chunk files are written)\n", a.c_str()); return 1; }
		else if (!a.empty() && a[0] == '-') { fprintf(stderr, "unknown flag %s\n", a.c_str()); return 1; }
		else source = a;
	}
	if (source.empty()) return usage();
	if (encoding != "DEFAULT" && encoding != "UNCOMPRESSED") { fprintf(stderr, "encoding %s is not supported\n", encoding.c_str()); return 1; }
	int m = method == "poisson" ? PCG_POISSON : method == "poisson_average" ? PCG_POISSON_AVERAGE : method == "random" ? PCG_RANDOM : -1;
	if (m < 0) { fprintf(stderr, "unknown method %s\n", method.c_str()); return 1; }
	if (!fs::exists(source)) { fprintf(stderr, "file does not exist: %s\n", source.c_str()); return 123; }
	if (outdir.empty()) outdir = source + "/../" + fs::path(source).filename().string() + "_converted";  // main.cpp:64-101
	std::ifstream f(source, std::ios::binary);
	std::vector<uint8_t> las((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
	std::string name = fs::path(source).stem().string();  // main.cpp:171-173

	pcg_ctx* ctx = nullptr;
	pcg_status st = pcg_create(&ctx, &opts);
	if (st != PCG_OK) { fprintf(stderr, "pcg_create failed: %s\n", pcg_status_string(st)); return 1; }
	pcg_job job{las.data(), las.size(), m, 0, name.c_str(), projection.c_str()};
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
