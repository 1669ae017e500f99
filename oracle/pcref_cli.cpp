// ORACLE -- test infrastructure only. Command line front end of the CPU
// restatement: pcref_cli <in.las> -o <outdir> [-m method] [--seed N]
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "pcref.h"

int main(int argc, char** argv) {
	std::string in, out, method = "poisson";
	uint32_t seed = 1592614637u;
	for (int i = 1; i < argc; i++) {
		std::string a = argv[i];
		if ((a == "-o" || a == "--outdir") && i + 1 < argc) out = argv[++i];
		else if ((a == "-m" || a == "--method") && i + 1 < argc) method = argv[++i];
		else if (a == "--seed" && i + 1 < argc) seed = (uint32_t)strtoul(argv[++i], nullptr, 10);
		else in = a;
	}
	if (in.empty() || out.empty()) { fprintf(stderr, "usage: pcref_cli <in.las> -o <outdir> [-m method]\n"); return 2; }
	std::ifstream f(in, std::ios::binary);
	std::vector<uint8_t> las((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
	pcref::Result res;
	std::string err;
	std::string name = std::filesystem::path(in).stem().string();
	if (!pcref::convert(las.data(), las.size(), method, name, seed, res, err)) { fprintf(stderr, "error: %s\n", err.c_str()); return 1; }
	std::filesystem::create_directories(out);
	auto wr = [&](const std::string& p, const std::vector<uint8_t>& d) { std::ofstream o(out + "/" + p, std::ios::binary); o.write((const char*)d.data(), d.size()); };
	wr("octree.bin", res.octree);
	wr("hierarchy.bin", res.hierarchy);
	wr("metadata.json", res.metadata);
	return 0;
}
