// ORACLE -- test infrastructure only. Command line front end of the CPU
// restatement:
//   pcref_cli <in.las> [<in.las> ...] -o <outdir> [-m method] [--seed N]
//             [--attributes name ...]
// Sources are taken in the order given; the name is the first source's stem
// (main.cpp:146-200).
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "pcref.h"

int main(int argc, char** argv) {
	std::vector<std::string> in, attributes;
	std::string out, method = "poisson";
	uint32_t seed = 1592614637u;
	bool inAttributes = false;
	for (int i = 1; i < argc; i++) {
		std::string a = argv[i];
		if ((a == "-o" || a == "--outdir") && i + 1 < argc) { out = argv[++i]; inAttributes = false; }
		else if ((a == "-m" || a == "--method") && i + 1 < argc) { method = argv[++i]; inAttributes = false; }
		else if (a == "--seed" && i + 1 < argc) { seed = (uint32_t)strtoul(argv[++i], nullptr, 10); inAttributes = false; }
		else if (a == "--attributes") inAttributes = true;
		else if (inAttributes) attributes.push_back(a);
		else in.push_back(a);
	}
	if (in.empty() || out.empty()) { fprintf(stderr, "usage: pcref_cli <in.las> ... -o <outdir> [-m method] [--attributes a ...]\n"); return 2; }
	std::vector<std::vector<uint8_t>> files;
	std::vector<pcref::SourceImage> sources;
	for (auto& path : in) {
		std::ifstream f(path, std::ios::binary);
		files.emplace_back((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
	}
	for (auto& f : files) sources.push_back({f.data(), f.size()});
	pcref::Result res;
	std::string err;
	std::string name = std::filesystem::path(in[0]).stem().string();
	if (!pcref::convert(sources, attributes, method, name, seed, res, err)) { fprintf(stderr, "error: %s\n", err.c_str()); return 1; }
	std::filesystem::create_directories(out);
	auto wr = [&](const std::string& p, const std::vector<uint8_t>& d) { std::ofstream o(out + "/" + p, std::ios::binary); o.write((const char*)d.data(), d.size()); };
	wr("octree.bin", res.octree);
	wr("hierarchy.bin", res.hierarchy);
	wr("metadata.json", res.metadata);
	return 0;
}
