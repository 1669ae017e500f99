// Host build of the library's LAZ decoder (potreeconverter_b200/csrc/laz.cuh)
// for the CPU tests: decodes every chunk of a LAZ file and writes the point
// records, which the test compares with the records of the LAS file the LAZ
// was made from.
//   laz_check <in.laz> <out.bin>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "laz.cuh"

int main(int argc, char** argv) {
	if (argc < 3) return 2;
	std::ifstream f(argv[1], std::ios::binary);
	std::vector<uint8_t> las((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
	auto u16 = [&](size_t o) { uint16_t v; std::memcpy(&v, &las[o], 2); return (uint32_t)v; };
	auto u32 = [&](size_t o) { uint32_t v; std::memcpy(&v, &las[o], 4); return v; };
	const uint32_t header_size = u16(94), offset = u32(96), nvlr = u32(100);
	const int pdrf = las[104] & 0x3f, rec_len = (int)u16(105);
	uint64_t n = u32(107);
	if (las[25] >= 4 && header_size >= 375) { uint64_t e; std::memcpy(&e, &las[247], 8); if (e > n) n = e; }
	const uint8_t* vlr = nullptr;
	uint32_t vlr_len = 0;
	size_t pos = header_size;
	for (uint32_t i = 0; i < nvlr; i++) {
		const uint32_t rid = u16(pos + 18), len = u16(pos + 20);
		if (rid == 22204 && std::memcmp(&las[pos + 2], "laszip encoded", 14) == 0) { vlr = &las[pos + 54]; vlr_len = len; }
		pos += 54 + len;
	}
	pcg::laz::Layout L;
	std::vector<pcg::laz::Chunk> chunks;
	std::string err;
	if (!pcg::laz::parse_table(las.data(), las.size(), offset, (int64_t)n, pdrf, rec_len, vlr, vlr_len, L, chunks, err)) {
		fprintf(stderr, "table: %s\n", err.c_str());
		return 1;
	}
	const uint32_t words = pcg::laz::arena_words(L);
	std::vector<uint32_t> arena(words);
	std::vector<uint8_t> out(n * (uint64_t)rec_len);
	for (size_t c = 0; c < chunks.size(); c++) {
		const auto& ch = chunks[c];
		pcg::laz::ChunkState state;
		if (!pcg::laz::decode_chunk(las.data() + ch.start, las.data() + ch.end, ch.count, L, state, nullptr, 0, arena.data(), words,
		                            out.data() + ch.first * rec_len)) {
			fprintf(stderr, "chunk %zu malformed\n", c);
			return 1;
		}
	}
	std::ofstream o(argv[2], std::ios::binary);
	o.write((const char*)out.data(), out.size());
	printf("chunks %zu points %llu arena_words %u\n", chunks.size(), (unsigned long long)n, words);
	return 0;
}
