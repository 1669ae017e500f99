// Host build of the library's header parsing and job set-up
// (potreeconverter_b200/csrc/setup.cpp) under AddressSanitizer and UBSan:
// LAS and LAZ images with mutated headers, VLRs, counts and chunk tables,
// alone and beside an intact source. Parsing may succeed or refuse; it must
// stay inside the image and never yield a negative point count.
//   parse_fuzz <seed> <trials> <file> [<file> ...]
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <random>
#include <vector>
#include "pcg_internal.h"
int main(int argc, char** argv) {
	std::mt19937 rng(atoi(argv[1]));
	int trials = atoi(argv[2]);
	std::vector<std::vector<uint8_t>> seeds;
	for (int i = 3; i < argc; i++) {
		std::ifstream f(argv[i], std::ios::binary);
		seeds.emplace_back((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
	}
	int ok = 0, err = 0;
	for (int t = 0; t < trials; t++) {
		std::vector<uint8_t> img = seeds[rng() % seeds.size()];
		const size_t hdr = std::min<size_t>(img.size(), 2048);
		int mode = t % 6;
		if (mode == 5 && img.size() > 260) { uint64_t v = ((uint64_t)rng() << 32) | rng(); if (rng() % 2) v |= 1ull << 63; std::memcpy(&img[247], &v, 8); img[25] = 4; }
		if (mode == 0) for (int k = 0; k < 1 + (int)(rng() % 6); k++) img[rng() % hdr] = (uint8_t)rng();          // header / VLR bytes
		if (mode == 1) img.resize(rng() % std::min<size_t>(img.size(), 4096));                                      // truncated
		if (mode == 2) { size_t o = 94 + 2 * (rng() % 20); if (o + 4 <= img.size()) { uint32_t v = rng(); std::memcpy(&img[o], &v, 4); } }  // counts / offsets
		if (mode == 3) for (int k = 0; k < 8; k++) img[img.size() - 1 - rng() % std::min<size_t>(img.size(), 4096)] ^= (uint8_t)(1 + rng() % 255);  // chunk table area
		if (mode == 4) { img.resize(img.size() / 2); }
		std::vector<uint8_t> exact(img);  // exact-size buffer
		pcg::LasInfo info;
		std::string e;
		bool elsewhere = (t % 7) == 0;
		if (!pcg::parse_las(exact.data(), exact.size(), info, e, elsewhere)) { err++; continue; }
		pcg::Setup s;
		std::vector<std::string> attrs;
		if (t % 3 == 0) attrs = {"rgb", "intensity", "amplitude"};
		// alone, and beside an intact source
		pcg::LasInfo good;
		std::string e2;
		pcg::parse_las(seeds[0].data(), seeds[0].size(), good, e2);
		if (pcg::make_setup(std::vector<pcg::LasInfo>{info}, attrs, s, e)) ok++; else err++;
		pcg::Setup s2;
		if (pcg::make_setup(std::vector<pcg::LasInfo>{good, info}, attrs, s2, e) && s2.total_points < 0) { printf("negative total\n"); return 1; }
		for (auto& src : s2.sources) if (src.las.num_points < 0) { printf("negative source count\n"); return 1; }
	}
	printf("accepted %d rejected %d\n", ok, err);
}
