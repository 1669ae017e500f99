// Host build of the library's LAZ decoder (potreeconverter_b200/csrc/laz.cuh)
// under AddressSanitizer and UBSan: decodes chunks of a LAZ file corrupted at
// random (bytes flipped, cut short, replaced, overwritten), untouched chunks
// with shared-memory stand-ins of random size, and corrupted chunk tables.
// Decoding may succeed or refuse; it must never touch memory outside its
// inputs, arenas and records.
//   laz_fuzz <in.laz> <seed> <trials>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <random>
#include <vector>
#include "laz.cuh"
int main(int argc, char** argv) {
	std::ifstream f(argv[1], std::ios::binary);
	std::vector<uint8_t> las((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
	auto u16 = [&](size_t o) { uint16_t v; std::memcpy(&v, &las[o], 2); return (uint32_t)v; };
	auto u32 = [&](size_t o) { uint32_t v; std::memcpy(&v, &las[o], 4); return v; };
	const uint32_t header_size = u16(94), offset = u32(96), nvlr = u32(100);
	const int pdrf = las[104] & 0x3f, rec_len = (int)u16(105);
	uint64_t n = u32(107);
	if (las[25] >= 4 && header_size >= 375) { uint64_t e; std::memcpy(&e, &las[247], 8); if (e > n) n = e; }
	const uint8_t* vlr = nullptr; uint32_t vlr_len = 0; size_t pos = header_size;
	for (uint32_t i = 0; i < nvlr; i++) { const uint32_t rid = u16(pos + 18), len = u16(pos + 20); if (rid == 22204) { vlr = &las[pos + 54]; vlr_len = len; } pos += 54 + len; }
	pcg::laz::Layout L; std::vector<pcg::laz::Chunk> chunks; std::string err;
	if (!pcg::laz::parse_table(las.data(), las.size(), offset, (int64_t)n, pdrf, rec_len, vlr, vlr_len, L, chunks, err)) { printf("table %s\n", err.c_str()); return 1; }
	const uint32_t words = pcg::laz::arena_words(L);
	std::mt19937 rng(atoi(argv[2]));
	int bad = 0, good = 0, valid_ok = 0;
	static pcg::laz::ChunkState S;
	for (int trial = 0; trial < atoi(argv[3]); trial++) {
		const auto& ch = chunks[rng() % chunks.size()];
		std::vector<uint8_t> bytes(las.begin() + ch.start, las.begin() + ch.end);
		std::vector<uint32_t> arena(words), fastbuf(1000 + rng() % 60000);
		std::vector<uint8_t> out((size_t)ch.count * rec_len);
		if (trial % 5 == 4) {  // untouched chunk with a random fast region: must decode
			valid_ok += pcg::laz::decode_chunk(bytes.data(), bytes.data() + bytes.size(), ch.count, L, S, fastbuf.data(), (uint32_t)fastbuf.size(), arena.data(), words, out.data());
			continue;
		}
		int mode = trial % 4;
		if (mode == 0) for (int k = 0; k < 1 + (int)(rng() % 8); k++) bytes[rng() % bytes.size()] ^= (uint8_t)(1 + rng() % 255);
		if (mode == 1) bytes.resize(rng() % bytes.size() + 1);
		if (mode == 2) for (auto& b : bytes) b = (uint8_t)rng();
		if (mode == 3 && bytes.size() > 64) std::memset(bytes.data() + rec_len + rng() % (bytes.size() - rec_len - 8), 0xFF, 8);
		std::vector<uint8_t> in(bytes);
		bool ok = pcg::laz::decode_chunk(in.data(), in.data() + in.size(), ch.count, L, S, fastbuf.data(), (uint32_t)fastbuf.size(), arena.data(), words, out.data());
		ok ? good++ : bad++;
	}
	printf("valid decoded %d, corrupted ok %d rejected %d\n", valid_ok, good, bad);
	for (int trial = 0; trial < 2000; trial++) {
		std::vector<uint8_t> c(las);
		uint64_t tpos; std::memcpy(&tpos, &c[offset], 8);
		for (int k = 0; k < 4; k++) c[tpos + 8 + rng() % (c.size() - tpos - 8)] ^= (uint8_t)(1 + rng() % 255);
		std::vector<pcg::laz::Chunk> ch2; pcg::laz::Layout L2;
		pcg::laz::parse_table(c.data(), c.size(), offset, (int64_t)n, pdrf, rec_len, vlr, vlr_len, L2, ch2, err);
	}
	printf("table fuzz done\n");
	return 0;
}
