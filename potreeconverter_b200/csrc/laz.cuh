// LAZ point decoding for point formats 0-3 (LASzip "pointwise chunked"
// compressor, items POINT10 v2, GPSTIME11 v2, RGB12 v2 and BYTE v2), written
// for both the host (the chunk table) and the device (the point records).
//
// The method is LASzip's (M. Isenburg, "LASzip: lossless compression of LiDAR
// data", PE&RS 79(2), 2013): an adaptive binary arithmetic coder with 32-bit
// range, periodic model updates and table-assisted symbol search (A. Said,
// "Introduction to arithmetic coding - theory and practice", HP Labs
// HPL-2004-76; Lossless Compression Handbook ch. 5), integer residuals coded
// as a bit-length class plus the bits within the class, and per-field
// predictors. The behaviour specification is the LASzip 3.4r3 the reference
// links (Converter/libs/laszip/src): arithmeticdecoder.cpp,
// arithmeticmodel.cpp, integercompressor.cpp, lasreaditemcompressed_v2.cpp,
// laszip_common_v2.hpp, lasreadpoint.cpp. The reference reads .laz inputs
// through it (chunker_countsort_laszip.cpp:194-203, 750-772).
//
// All model state of one LASzip chunk lives in a flat uint32 arena, so one
// chunk is decoded by one thread with nothing but a pointer to its slice.
// Every index is bounded by construction and every loop by a constant or by
// the chunk's point count; malformed input sets `bad` instead of reading or
// writing outside the chunk, its arena or its records.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#ifdef __CUDACC__
#define LAZ_HD __host__ __device__ __forceinline__
// rarely taken routines stay out of line: one decoder chain per chunk is
// bound by its own issue latency, and inlining them at every call site
// multiplies the code the instruction cache has to hold
#define LAZ_RARE inline __host__ __device__ __noinline__
#else
#define LAZ_HD inline
#define LAZ_RARE inline
#endif

namespace pcg {
namespace laz {

constexpr uint32_t kMinLength = 1u << 24;  // renormalise below this range
constexpr uint32_t kBitShift = 13;         // bit model: probability bits
constexpr uint32_t kBitMaxCount = 1u << 13;
constexpr uint32_t kSymShift = 15;         // symbol model: probability bits
constexpr uint32_t kSymMaxCount = 1u << 15;

// ------------------------------------------------------------------ arena
// Model storage of one chunk decoder: words are taken from a fast region
// first (the block's shared memory on the device; none on the host), then
// from a global region. A null global region only measures.
struct Arena {
	uint32_t* fast;
	uint32_t f_top, f_cap;
	uint32_t* glob;
	uint32_t g_top, g_cap;
	bool overflow;
	LAZ_HD bool measuring() const { return glob == nullptr; }
	LAZ_HD uint32_t* take(uint32_t words) {
		if (fast && f_top + words <= f_cap) {
			uint32_t* p = fast + f_top;
			f_top += words;
			return p;
		}
		return take_global(words);
	}
	LAZ_HD uint32_t* take_global(uint32_t words) {
		uint32_t* p = glob ? glob + g_top : nullptr;
		g_top += words;
		if (g_top > g_cap) {
			overflow = true;
			return nullptr;
		}
		return p;
	}
};

// A symbol model is a pointer h to: a header of M_HDR words, then 16-bit
// arrays: cumulative distribution[n], counts[n] and, for n > 16, a decoder
// table of table_size + 2 entries. Every value fits 16 bits: distribution
// values are below 2^15, counts below 2^15 + 8 (n + 6) (they are halved
// when their total passes 2^15 at an update, at most 8 (n + 6) symbols
// apart), table entries below n <= 516.
enum { M_N = 0, M_SHIFT, M_TSIZE, M_TOTAL, M_CYCLE, M_UNTIL, M_HDR };

LAZ_HD uint32_t table_bits_for(uint32_t n) {
	uint32_t tb = 3;
	while (n > (1u << (tb + 2))) ++tb;
	return tb;
}

LAZ_HD uint32_t model_words(uint32_t n) {
	const uint32_t halves = 2 * n + (n > 16 ? (1u << table_bits_for(n)) + 2 : 0);
	return M_HDR + (halves + 1) / 2;
}

LAZ_HD uint16_t* model_dist(uint32_t* h) { return reinterpret_cast<uint16_t*>(h + M_HDR); }

// counts halved at the limit, cumulative distribution, decoder table, next
// update interval (5/4 of the last, at most 8 (n + 6))
LAZ_RARE void model_update(uint32_t* h) {
	const uint32_t n = h[M_N];
	uint16_t* dist = model_dist(h);
	uint16_t* cnt = dist + n;
	if ((h[M_TOTAL] += h[M_CYCLE]) > kSymMaxCount) {
		uint32_t t = 0;
		for (uint32_t k = 0; k < n; k++) {
			const uint32_t c = ((uint32_t)cnt[k] + 1) >> 1;
			cnt[k] = (uint16_t)c;
			t += c;
		}
		h[M_TOTAL] = t;
	}
	const uint32_t scale = 0x80000000u / h[M_TOTAL];
	uint32_t sum = 0;
	if (h[M_TSIZE] == 0) {
		for (uint32_t k = 0; k < n; k++) {
			dist[k] = (uint16_t)((scale * sum) >> (31 - kSymShift));
			sum += cnt[k];
		}
	} else {
		uint16_t* tab = cnt + n;
		const uint32_t shift = h[M_SHIFT], tsize = h[M_TSIZE];
		uint32_t s = 0;
		for (uint32_t k = 0; k < n; k++) {
			const uint32_t dk = (scale * sum) >> (31 - kSymShift);
			dist[k] = (uint16_t)dk;
			sum += cnt[k];
			const uint32_t w = dk >> shift;
			while (s < w && s < tsize) tab[++s] = (uint16_t)(k - 1);
		}
		tab[0] = 0;
		while (s <= tsize) tab[++s] = (uint16_t)(n - 1);
	}
	uint32_t cycle = (5 * h[M_CYCLE]) >> 2;
	const uint32_t max_cycle = (n + 6) << 3;
	if (cycle > max_cycle) cycle = max_cycle;
	h[M_CYCLE] = h[M_UNTIL] = cycle;
}

// uniform counts, then the first update after (n + 6) / 2 symbols
LAZ_RARE void model_init(uint32_t* h) {
	const uint32_t n = h[M_N];
	uint16_t* cnt = model_dist(h) + n;
	h[M_TOTAL] = 0;
	h[M_CYCLE] = n;
	for (uint32_t k = 0; k < n; k++) cnt[k] = 1;
	model_update(h);
	h[M_CYCLE] = h[M_UNTIL] = (n + 6) >> 1;
}

LAZ_HD void model_header(uint32_t* h, uint32_t n) {
	h[M_N] = n;
	if (n > 16) {
		const uint32_t tb = table_bits_for(n);
		h[M_TSIZE] = 1u << tb;
		h[M_SHIFT] = kSymShift - tb;
	} else {
		h[M_TSIZE] = h[M_SHIFT] = 0;
	}
}

LAZ_RARE uint32_t* model_new(Arena& ar, uint32_t n) {
	uint32_t* h = ar.take(model_words(n));
	if (h) model_header(h, n);
	return h;
}

// bit model: count of zeros, count, probability of zero, interval
enum { B_ZERO = 0, B_COUNT, B_PROB, B_CYCLE, B_UNTIL, B_WORDS };

LAZ_HD void bit_init(uint32_t* h) {
	h[B_ZERO] = 1;
	h[B_COUNT] = 2;
	h[B_PROB] = 1u << (kBitShift - 1);
	h[B_CYCLE] = h[B_UNTIL] = 4;
}

LAZ_RARE void bit_update(uint32_t* h) {
	if ((h[B_COUNT] += h[B_CYCLE]) > kBitMaxCount) {
		h[B_COUNT] = (h[B_COUNT] + 1) >> 1;
		h[B_ZERO] = (h[B_ZERO] + 1) >> 1;
		if (h[B_ZERO] == h[B_COUNT]) ++h[B_COUNT];
	}
	const uint32_t scale = 0x80000000u / h[B_COUNT];
	h[B_PROB] = (h[B_ZERO] * scale) >> (31 - kBitShift);
	uint32_t cycle = (5 * h[B_CYCLE]) >> 2;
	if (cycle > 64) cycle = 64;
	h[B_CYCLE] = h[B_UNTIL] = cycle;
}

// ---------------------------------------------------------------- decoder
struct Decoder {
	const uint8_t* p;
	const uint8_t* end;
	uint32_t value, length;
	bool bad;

	LAZ_HD uint32_t next_byte() {
		if (p < end) return *p++;
		bad = true;  // the reference stops with an end-of-chunk error
		return 0;
	}
	LAZ_HD void start(const uint8_t* from, const uint8_t* to) {
		p = from;
		end = to;
		bad = false;
		length = 0xFFFFFFFFu;
		value = next_byte() << 24;
		value |= next_byte() << 16;
		value |= next_byte() << 8;
		value |= next_byte();
	}
	// a valid stream needs at most three bytes; a zero range is malformed
	LAZ_HD void renorm() {
		int guard = 0;
		do {
			value = (value << 8) | next_byte();
			length <<= 8;
		} while (length < kMinLength && ++guard < 4);
		if (length < kMinLength) {
			bad = true;
			length = kMinLength;
		}
	}
	LAZ_HD uint32_t bit(uint32_t* h) {
		const uint32_t x = h[B_PROB] * (length >> kBitShift);
		const uint32_t sym = value >= x;
		if (sym == 0) {
			length = x;
			++h[B_ZERO];
		} else {
			value -= x;
			length -= x;
		}
		if (length < kMinLength) renorm();
		if (--h[B_UNTIL] == 0) bit_update(h);
		return sym;
	}
	LAZ_HD uint32_t symbol(uint32_t* h) {
		const uint32_t nsym = h[M_N];
		const uint16_t* dist = model_dist(h);
		uint32_t n, sym, x, y = length;
		if (h[M_TSIZE]) {
			const uint16_t* tab = dist + 2 * nsym;
			const uint32_t dv = value / (length >>= kSymShift);
			uint32_t t = dv >> h[M_SHIFT];
			if (t > h[M_TSIZE]) t = h[M_TSIZE];
			sym = tab[t];
			n = (uint32_t)tab[t + 1] + 1;
			if (n > nsym) n = nsym;
			if (sym >= nsym) sym = nsym - 1;
			while (n > sym + 1) {
				const uint32_t k = (sym + n) >> 1;
				if (dist[k] > dv) n = k;
				else sym = k;
			}
			x = dist[sym] * length;
			if (sym != nsym - 1) y = dist[sym + 1] * length;
		} else {
			x = sym = 0;
			length >>= kSymShift;
			n = nsym;
			uint32_t k = n >> 1;
			do {
				const uint32_t z = length * dist[k];
				if (z > value) {
					n = k;
					y = z;
				} else {
					sym = k;
					x = z;
				}
			} while ((k = (sym + n) >> 1) != sym);
		}
		value -= x;
		length = y - x;
		if (length < kMinLength) renorm();
		uint16_t* cnt = model_dist(h) + nsym;
		++cnt[sym];
		if (--h[M_UNTIL] == 0) model_update(h);
		return sym;
	}
	// raw bits (readBits, readShort, readInt)
	LAZ_HD uint32_t raw(uint32_t bits) {
		const uint32_t sym = value / (length >>= bits);
		value -= length * sym;
		if (length < kMinLength) renorm();
		if (sym >> bits) bad = true;
		return sym;
	}
	LAZ_HD uint32_t raw_bits(uint32_t bits) {
		if (bits > 19) {
			const uint32_t lo = raw(16);
			return (raw(bits - 16) << 16) | lo;
		}
		return raw(bits);
	}
	LAZ_HD uint32_t raw_int() {
		const uint32_t lo = raw(16);
		const uint32_t hi = raw(16);
		return (hi << 16) | lo;
	}
};

// ----------------------------------------------------- integer residuals
// A value is coded as pred + c: first the class k (the bit length of c,
// symbol model per context), then, for k <= bits_high, c within the class
// with one symbol model per k, else its top bits with that model and the
// rest raw. corr_bits / corr_range / corr_min follow from `bits`.
struct IntCoder {
	uint32_t bits_high, corr_bits, corr_range;
	int32_t corr_min;
	uint32_t contexts, mbits_words;
	uint32_t* mbits;    // `contexts` class models, back to back
	uint32_t* corr0;    // bit model for k = 0
	uint32_t* corr[33]; // symbol model per k = 1..corr_bits; for k > bits_high
	                    // created when the class first occurs
	Arena* arena;       // where those come from
	uint32_t k;         // class of the last value

	LAZ_HD void setup(uint32_t bits, uint32_t nctx, uint32_t high = 8) {
		bits_high = high;
		contexts = nctx;
		if (bits && bits < 32) {
			corr_bits = bits;
			corr_range = 1u << bits;
			corr_min = -(int32_t)(corr_range / 2);
		} else {
			corr_bits = 32;
			corr_range = 0;
			corr_min = (int32_t)0x80000000u;
		}
		mbits_words = model_words(corr_bits + 1);
		mbits = corr0 = nullptr;
		for (int i = 0; i < 33; i++) corr[i] = nullptr;
		arena = nullptr;
		k = 0;
	}
	LAZ_RARE void alloc_classes(Arena& ar) {
		arena = &ar;
		mbits = ar.take(contexts * mbits_words);
		if (mbits)
			for (uint32_t i = 0; i < contexts; i++) model_header(mbits + i * mbits_words, corr_bits + 1);
		corr0 = ar.take(B_WORDS);
	}
	LAZ_RARE void alloc_correctors(Arena& ar, uint32_t lo, uint32_t hi) {
		for (uint32_t i = lo; i <= hi && i <= corr_bits; i++) corr[i] = model_new(ar, i <= bits_high ? (1u << i) : (1u << bits_high));
	}
	LAZ_HD void init() {
		for (uint32_t i = 0; i < contexts; i++) model_init(mbits + i * mbits_words);
		bit_init(corr0);
		for (uint32_t i = 1; i <= corr_bits; i++)
			if (corr[i]) model_init(corr[i]);
		k = 0;
	}
	// the corrector model of class kk, created (fresh, as the reference's
	// model initialised at the chunk start) when kk first occurs
	LAZ_HD uint32_t* corr_model(Decoder& d, uint32_t kk) {
		uint32_t* m = corr[kk];
		if (!m) {
			m = model_new(*arena, 1u << bits_high);
			if (!m) {
				d.bad = true;
				return mbits;
			}
			model_init(m);
			corr[kk] = m;
		}
		return m;
	}
	LAZ_HD int32_t corrector(Decoder& d, uint32_t ctx) {
		if (ctx >= contexts) {
			d.bad = true;
			ctx = 0;
		}
		k = d.symbol(mbits + ctx * mbits_words);
		uint32_t c;
		if (k) {
			if (k < 32) {
				if (k <= bits_high) {
					c = d.symbol(corr[k]);
				} else {
					const uint32_t k1 = k - bits_high;
					c = d.symbol(corr_model(d, k));
					const uint32_t c1 = d.raw_bits(k1);
					c = (c << k1) | c1;
				}
				// [0, 2^(k-1)) -> [-(2^k - 1), -2^(k-1)]; [2^(k-1), 2^k) -> [2^(k-1) + 1, 2^k]
				if (c >= (1u << (k - 1))) c += 1;
				else c -= ((1u << k) - 1);
			} else {
				c = (uint32_t)corr_min;
			}
		} else {
			c = d.bit(corr0);
		}
		return (int32_t)c;
	}
	LAZ_HD int32_t decode(Decoder& d, int32_t pred, uint32_t ctx = 0) {
		int32_t real = (int32_t)((uint32_t)pred + (uint32_t)corrector(d, ctx));
		if (real < 0) real = (int32_t)((uint32_t)real + corr_range);
		else if ((uint32_t)real >= corr_range) real = (int32_t)((uint32_t)real - corr_range);
		return real;
	}
};

// ------------------------------------------------------------ item state
// running median of the last five values (laszip_common_v2.hpp)
struct Median5 {
	int32_t v[5];
	bool high;
	LAZ_HD void init() {
		v[0] = v[1] = v[2] = v[3] = v[4] = 0;
		high = true;
	}
	LAZ_HD int32_t get() const { return v[2]; }
	LAZ_HD void add(int32_t x) {
		if (high) {
			if (x < v[2]) {
				v[4] = v[3];
				v[3] = v[2];
				if (x < v[0]) { v[2] = v[1]; v[1] = v[0]; v[0] = x; }
				else if (x < v[1]) { v[2] = v[1]; v[1] = x; }
				else v[2] = x;
			} else {
				if (x < v[3]) { v[4] = v[3]; v[3] = x; }
				else v[4] = x;
				high = false;
			}
		} else {
			if (v[2] < x) {
				v[0] = v[1];
				v[1] = v[2];
				if (v[4] < x) { v[2] = v[3]; v[3] = v[4]; v[4] = x; }
				else if (v[3] < x) { v[2] = v[3]; v[3] = x; }
				else v[2] = x;
			} else {
				if (v[1] < x) { v[0] = v[1]; v[1] = x; }
				else v[0] = x;
				high = true;
			}
		}
	}
};

// context of (number of returns n, return number r) for intensity, x and y
// (laszip_common_v2.hpp number_return_map) and for z (number_return_level)
LAZ_HD uint32_t return_map(uint32_t n, uint32_t r) {
	constexpr uint8_t t[8][8] = {{15, 14, 13, 12, 11, 10, 9, 8}, {14, 0, 1, 3, 6, 10, 10, 9}, {13, 1, 2, 4, 7, 11, 11, 10},
	                             {12, 3, 4, 5, 8, 12, 12, 11},   {11, 6, 7, 8, 9, 13, 13, 12}, {10, 10, 11, 12, 13, 14, 14, 13},
	                             {9, 10, 11, 12, 13, 14, 15, 14}, {8, 9, 10, 11, 12, 13, 14, 15}};
	return t[n & 7][r & 7];
}
LAZ_HD uint32_t return_level(uint32_t n, uint32_t r) {
	const int d = (int)(n & 7) - (int)(r & 7);
	return (uint32_t)(d < 0 ? -d : d);
}

// int64 + int32 modulo 2^64 (a malformed time stream may overflow)
LAZ_HD int64_t add_wrap(int64_t a, int32_t b) { return (int64_t)((uint64_t)a + (uint64_t)(int64_t)b); }

LAZ_HD int32_t fold8(int32_t v) { return v < 0 ? v + 256 : (v > 255 ? v - 256 : v); }
LAZ_HD int32_t clamp8(int32_t v) { return v <= 0 ? 0 : (v >= 255 ? 255 : v); }

template <class T> LAZ_HD T rd(const uint8_t* p) {
	T v;
	uint8_t* q = reinterpret_cast<uint8_t*>(&v);
	for (unsigned i = 0; i < sizeof(T); i++) q[i] = p[i];
	return v;
}
template <class T> LAZ_HD void wr(uint8_t* p, T v) {
	const uint8_t* q = reinterpret_cast<const uint8_t*>(&v);
	for (unsigned i = 0; i < sizeof(T); i++) p[i] = q[i];
}

constexpr int kMaxExtraBytes = 64;  // BYTE item size this decoder accepts

// The record layout of a LAZ source: items in record order.
struct Layout {
	int has_gps, has_rgb, n_extra, rec_len;
};

// The models of one chunk decoder, placed so that the fast region holds
// what the data uses: first the models every point needs (the classes of
// every integer coder, the per-point symbol models, correctors of classes
// up to 8), then, in order of first use, the 256-symbol correctors of larger
// classes and the models of the three 256-context tables of POINT10 (bit
// byte, classification, user data). A model created at first use starts as
// the reference's model initialised at the chunk start.
struct Models {
	uint32_t* changed;
	uint32_t* scan_angle[2];
	IntCoder ic_intensity, ic_psid, ic_dx, ic_dy, ic_z, ic_gps;
	uint32_t* lazy;  // 3 x 256 handles: 0 none yet, else 1 + word offset | 2^31 when in the fast region
	uint32_t* gps_multi;
	uint32_t* gps_0diff;
	uint32_t* rgb_used;
	uint32_t* rgb_diff[6];
	uint32_t* byte_model[kMaxExtraBytes];

	LAZ_RARE void create(Arena& ar, const Layout& L) {
		ic_intensity.setup(16, 4);
		ic_psid.setup(16, 1);
		ic_dx.setup(32, 2);
		ic_dy.setup(32, 22);
		ic_z.setup(32, 20);
		ic_gps.setup(32, 9);
		changed = model_new(ar, 64);
		ic_dx.alloc_classes(ar);
		ic_dy.alloc_classes(ar);
		ic_z.alloc_classes(ar);
		ic_intensity.alloc_classes(ar);
		ic_psid.alloc_classes(ar);
		if (L.has_gps) {
			gps_0diff = model_new(ar, 6);
			gps_multi = model_new(ar, 516);  // 500 multipliers, -10 .. -1, unchanged, full, 4 sequence switches
			ic_gps.alloc_classes(ar);
		}
		scan_angle[0] = model_new(ar, 256);
		scan_angle[1] = model_new(ar, 256);
		if (L.has_rgb) {
			rgb_used = model_new(ar, 128);
			for (int i = 0; i < 6; i++) rgb_diff[i] = model_new(ar, 256);
		}
		for (int i = 0; i < L.n_extra && i < kMaxExtraBytes; i++) byte_model[i] = model_new(ar, 256);
		// correctors of classes up to 8 now; the larger ones (256 symbols
		// each) when their class first occurs, so the fast region holds what
		// the data uses (a measuring arena counts them all)
		const uint32_t upto = ar.measuring() ? 32 : 8;
		ic_dx.alloc_correctors(ar, 1, upto);
		ic_dy.alloc_correctors(ar, 1, upto);
		ic_z.alloc_correctors(ar, 1, upto);
		ic_intensity.alloc_correctors(ar, 1, upto);
		ic_psid.alloc_correctors(ar, 1, upto);
		if (L.has_gps) ic_gps.alloc_correctors(ar, 1, upto);
		lazy = ar.take_global(3 * 256);
	}
};

// Everything a chunk decoder indexes at run time besides the models: the
// arena, the model handles and the predictor state. The device keeps it in
// the block's shared memory, the host on its stack.
struct ChunkState {
	Arena ar;
	Models M;
	Median5 mx[16], my[16];
	uint16_t last_intensity[16];
	int32_t last_height[8];
	int64_t gps[4];
	int32_t gps_diff[4], gps_extreme[4];
	uint8_t last_extra[kMaxExtraBytes];
};

// Global words one chunk decoder may need with no fast region: the models
// plus one 256-symbol model for each of the 3 x 256 lazily created contexts.
inline uint32_t arena_words(const Layout& L) {
	Arena ar{nullptr, 0, 0, nullptr, 0, 0xFFFFFFFFu, false};
	Models M;
	M.create(ar, L);
	return ar.g_top + 3 * 256 * model_words(256);
}

// Decodes one LASzip chunk of `count` points from bytes [p, end) into
// `count` consecutive records of L.rec_len bytes at out. Models go to the
// fast region (fast, f_words; may be null) first, then to the global
// region (glob, g_words >= arena_words(L)). Returns false on malformed
// input. Follows LASreadPoint::read (lasreadpoint.cpp:405-497): the first
// point is stored raw, the arithmetic decoder starts after it.
LAZ_HD bool decode_chunk(const uint8_t* p, const uint8_t* end, int64_t count, const Layout& L, ChunkState& S, uint32_t* fast,
                         uint32_t f_words, uint32_t* glob, uint32_t g_words, uint8_t* out) {
	if (count <= 0) return true;
	const int rl = L.rec_len;
	const int std_len = 20 + (L.has_gps ? 8 : 0) + (L.has_rgb ? 6 : 0);
	if (L.n_extra < 0 || L.n_extra > kMaxExtraBytes || std_len + L.n_extra != rl) return false;
	if (end - p < rl) return false;
	S.ar = Arena{fast, 0, fast ? f_words : 0u, glob, 0, g_words, false};
	Arena& ar = S.ar;
	Models& M = S.M;
	M.create(ar, L);
	if (ar.overflow) return false;
	// first point: raw item bytes, which initialise the item predictors
	for (int b = 0; b < rl; b++) out[b] = p[b];
	p += rl;
	// POINT10 state (LASreadItemCompressed_POINT10_v2::init)
	uint8_t last[20];
	for (int b = 0; b < 20; b++) last[b] = out[b];
	last[12] = last[13] = 0;
	Median5* mx = S.mx;
	Median5* my = S.my;
	uint16_t* last_intensity = S.last_intensity;
	int32_t* last_height = S.last_height;
	for (int i = 0; i < 16; i++) {
		mx[i].init();
		my[i].init();
		last_intensity[i] = 0;
	}
	for (int i = 0; i < 8; i++) last_height[i] = 0;
	model_init(M.changed);
	M.ic_intensity.init();
	model_init(M.scan_angle[0]);
	model_init(M.scan_angle[1]);
	M.ic_psid.init();
	M.ic_dx.init();
	M.ic_dy.init();
	M.ic_z.init();
	uint32_t* lazy = M.lazy;
	for (int i = 0; i < 3 * 256; i++) lazy[i] = 0;
	// GPSTIME11 state
	int64_t* gps = S.gps;
	int32_t* gps_diff = S.gps_diff;
	int32_t* gps_extreme = S.gps_extreme;
	for (int i = 0; i < 4; i++) gps[i] = gps_diff[i] = gps_extreme[i] = 0;
	uint32_t gps_last = 0, gps_next = 0;
	if (L.has_gps) {
		model_init(M.gps_multi);
		model_init(M.gps_0diff);
		M.ic_gps.init();
		gps[0] = rd<int64_t>(out + 20);
	}
	// RGB12 state
	uint16_t last_rgb[3] = {0, 0, 0};
	const int rgb_off = 20 + (L.has_gps ? 8 : 0);
	if (L.has_rgb) {
		model_init(M.rgb_used);
		for (int i = 0; i < 6; i++) model_init(M.rgb_diff[i]);
		for (int i = 0; i < 3; i++) last_rgb[i] = rd<uint16_t>(out + rgb_off + 2 * i);
	}
	// BYTE state
	uint8_t* last_extra = S.last_extra;
	for (int i = 0; i < L.n_extra; i++) {
		model_init(M.byte_model[i]);
		last_extra[i] = out[std_len + i];
	}
	Decoder d;
	d.start(p, end);
	// lazily created 256-symbol model of table t (0 bit byte, 1 class, 2 user data) for context c
	auto lazy_model = [&](int t, uint32_t c) -> uint32_t* {
		uint32_t& slot = lazy[t * 256 + (c & 255)];
		if (slot == 0) {
			uint32_t* m = model_new(ar, 256);
			if (!m) {
				d.bad = true;
				return M.scan_angle[0];
			}
			model_init(m);
			slot = (fast && m >= fast && m < fast + f_words) ? (0x80000000u | (uint32_t)(m - fast)) : (uint32_t)(m - glob) + 1;
			return m;
		}
		return (slot & 0x80000000u) ? fast + (slot & 0x7FFFFFFFu) : glob + (slot - 1);
	};

	for (int64_t i = 1; i < count && !d.bad; i++) {
		uint8_t* rec = out + i * rl;
		// ---- POINT10 v2 (lasreaditemcompressed_v2.cpp, POINT10 read)
		const uint32_t changed = d.symbol(M.changed);
		uint32_t r, n;
		if (changed) {
			if (changed & 32) last[14] = (uint8_t)d.symbol(lazy_model(0, last[14]));
			r = last[14] & 7;
			n = (last[14] >> 3) & 7;
			const uint32_t m = return_map(n, r);
			if (changed & 16) {
				const uint16_t v = (uint16_t)M.ic_intensity.decode(d, last_intensity[m], m < 3 ? m : 3);
				wr<uint16_t>(last + 12, v);
				last_intensity[m] = v;
			} else {
				wr<uint16_t>(last + 12, last_intensity[m]);
			}
			if (changed & 8) last[15] = (uint8_t)d.symbol(lazy_model(1, last[15]));
			if (changed & 4) {
				const int32_t v = (int32_t)d.symbol(M.scan_angle[(last[14] >> 6) & 1]);
				last[16] = (uint8_t)fold8(v + last[16]);
			}
			if (changed & 2) last[17] = (uint8_t)d.symbol(lazy_model(2, last[17]));
			if (changed & 1) wr<uint16_t>(last + 18, (uint16_t)M.ic_psid.decode(d, rd<uint16_t>(last + 18)));
		} else {
			r = last[14] & 7;
			n = (last[14] >> 3) & 7;
		}
		const uint32_t m = return_map(n, r), l = return_level(n, r);
		{
			const int32_t diff = M.ic_dx.decode(d, mx[m].get(), n == 1);
			wr<int32_t>(last + 0, (int32_t)((uint32_t)rd<int32_t>(last + 0) + (uint32_t)diff));
			mx[m].add(diff);
		}
		{
			const uint32_t kb = M.ic_dx.k;
			const int32_t diff = M.ic_dy.decode(d, my[m].get(), (n == 1) + (kb < 20 ? (kb & ~1u) : 20));
			wr<int32_t>(last + 4, (int32_t)((uint32_t)rd<int32_t>(last + 4) + (uint32_t)diff));
			my[m].add(diff);
		}
		{
			const uint32_t kb = (M.ic_dx.k + M.ic_dy.k) / 2;
			const int32_t z = M.ic_z.decode(d, last_height[l], (n == 1) + (kb < 18 ? (kb & ~1u) : 18));
			wr<int32_t>(last + 8, z);
			last_height[l] = z;
		}
		for (int b = 0; b < 20; b++) rec[b] = last[b];
		// ---- GPSTIME11 v2
		if (L.has_gps) {
			for (int guard = 0;; guard++) {
				if (guard >= 4) {
					d.bad = true;
					break;
				}
				bool again = false;
				if (gps_diff[gps_last] == 0) {
					const uint32_t multi = d.symbol(M.gps_0diff);
					if (multi == 1) {
						gps_diff[gps_last] = M.ic_gps.decode(d, 0, 0);
						gps[gps_last] = add_wrap(gps[gps_last], gps_diff[gps_last]);
						gps_extreme[gps_last] = 0;
					} else if (multi == 2) {
						gps_next = (gps_next + 1) & 3;
						const uint32_t hi = (uint32_t)M.ic_gps.decode(d, (int32_t)(uint32_t)((uint64_t)gps[gps_last] >> 32), 8);
						const uint32_t lo = d.raw_int();
						gps[gps_next] = (int64_t)(((uint64_t)hi << 32) | lo);
						gps_last = gps_next;
						gps_diff[gps_last] = 0;
						gps_extreme[gps_last] = 0;
					} else if (multi > 2) {
						gps_last = (gps_last + multi - 2) & 3;
						again = true;
					}
				} else {
					const int32_t multi = (int32_t)d.symbol(M.gps_multi);
					const int32_t ld = gps_diff[gps_last];
					auto times = [](int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); };
					if (multi == 1) {
						gps[gps_last] = add_wrap(gps[gps_last], M.ic_gps.decode(d, ld, 1));
						gps_extreme[gps_last] = 0;
					} else if (multi < 511) {
						int32_t gd;
						if (multi == 0) {
							gd = M.ic_gps.decode(d, 0, 7);
							if (++gps_extreme[gps_last] > 3) {
								gps_diff[gps_last] = gd;
								gps_extreme[gps_last] = 0;
							}
						} else if (multi < 500) {
							gd = M.ic_gps.decode(d, times(multi, ld), multi < 10 ? 2 : 3);
						} else if (multi == 500) {
							gd = M.ic_gps.decode(d, times(500, ld), 4);
							if (++gps_extreme[gps_last] > 3) {
								gps_diff[gps_last] = gd;
								gps_extreme[gps_last] = 0;
							}
						} else {
							const int32_t mm = 500 - multi;  // -1 .. -10
							if (mm > -10) {
								gd = M.ic_gps.decode(d, times(mm, ld), 5);
							} else {
								gd = M.ic_gps.decode(d, times(-10, ld), 6);
								if (++gps_extreme[gps_last] > 3) {
									gps_diff[gps_last] = gd;
									gps_extreme[gps_last] = 0;
								}
							}
						}
						gps[gps_last] = add_wrap(gps[gps_last], gd);
					} else if (multi == 512) {
						gps_next = (gps_next + 1) & 3;
						const uint32_t hi = (uint32_t)M.ic_gps.decode(d, (int32_t)(uint32_t)((uint64_t)gps[gps_last] >> 32), 8);
						const uint32_t lo = d.raw_int();
						gps[gps_next] = (int64_t)(((uint64_t)hi << 32) | lo);
						gps_last = gps_next;
						gps_diff[gps_last] = 0;
						gps_extreme[gps_last] = 0;
					} else if (multi > 512) {
						gps_last = (gps_last + (uint32_t)multi - 512) & 3;
						again = true;
					}
				}
				if (!again) break;
			}
			wr<int64_t>(rec + 20, gps[gps_last]);
		}
		// ---- RGB12 v2
		if (L.has_rgb) {
			uint16_t c[3];
			const uint32_t sym = d.symbol(M.rgb_used);
			if (sym & 1) c[0] = (uint16_t)fold8((int32_t)(uint8_t)d.symbol(M.rgb_diff[0]) + (last_rgb[0] & 255));
			else c[0] = last_rgb[0] & 0xFF;
			if (sym & 2) c[0] |= (uint16_t)(fold8((int32_t)(uint8_t)d.symbol(M.rgb_diff[1]) + (last_rgb[0] >> 8)) << 8);
			else c[0] |= last_rgb[0] & 0xFF00;
			if (sym & 64) {
				int32_t diff = (int32_t)(c[0] & 0xFF) - (int32_t)(last_rgb[0] & 0xFF);
				if (sym & 4) c[1] = (uint16_t)fold8((int32_t)(uint8_t)d.symbol(M.rgb_diff[2]) + clamp8(diff + (last_rgb[1] & 255)));
				else c[1] = last_rgb[1] & 0xFF;
				if (sym & 16) {
					const int32_t corr = (int32_t)(uint8_t)d.symbol(M.rgb_diff[4]);
					diff = (diff + ((int32_t)(c[1] & 0xFF) - (int32_t)(last_rgb[1] & 0xFF))) / 2;
					c[2] = (uint16_t)fold8(corr + clamp8(diff + (last_rgb[2] & 255)));
				} else {
					c[2] = last_rgb[2] & 0xFF;
				}
				diff = (int32_t)(c[0] >> 8) - (int32_t)(last_rgb[0] >> 8);
				if (sym & 8)
					c[1] |= (uint16_t)(fold8((int32_t)(uint8_t)d.symbol(M.rgb_diff[3]) + clamp8(diff + (last_rgb[1] >> 8))) << 8);
				else
					c[1] |= last_rgb[1] & 0xFF00;
				if (sym & 32) {
					const int32_t corr = (int32_t)(uint8_t)d.symbol(M.rgb_diff[5]);
					diff = (diff + ((int32_t)(c[1] >> 8) - (int32_t)(last_rgb[1] >> 8))) / 2;
					c[2] |= (uint16_t)(fold8(corr + clamp8(diff + (last_rgb[2] >> 8))) << 8);
				} else {
					c[2] |= last_rgb[2] & 0xFF00;
				}
			} else {
				c[1] = c[0];
				c[2] = c[0];
			}
			for (int k = 0; k < 3; k++) {
				last_rgb[k] = c[k];
				wr<uint16_t>(rec + rgb_off + 2 * k, c[k]);
			}
		}
		// ---- BYTE v2
		for (int e = 0; e < L.n_extra; e++) {
			last_extra[e] = (uint8_t)fold8((int32_t)last_extra[e] + (int32_t)d.symbol(M.byte_model[e]));
			rec[std_len + e] = last_extra[e];
		}
	}
	return !d.bad;
}

}  // namespace laz
}  // namespace pcg

// ------------------------------------------------------------- host side
namespace pcg {
namespace laz {

// One LASzip chunk: its bytes [start, end) in the file and its points.
struct Chunk {
	uint64_t start, end;
	int64_t first, count;
};

// The laszip VLR (record 22204, user "laszip encoded"; LASzip::unpack,
// laszip.cpp:82-135) and the chunk table (LASreadPoint::read_chunk_table,
// lasreadpoint.cpp:588-720) of a LAZ file whose header gives
// offset_to_points, num_points, point format pdrf and record length.
// Accepts what LASzip writes for point formats 0-3: compressor 2 (pointwise
// chunked), coder 0, items POINT10, [GPSTIME11], [RGB12], [BYTE] at version
// 2, fixed or variable chunk sizes.
inline bool parse_table(const uint8_t* file, uint64_t size, uint64_t offset_to_points, int64_t num_points, int pdrf, int rec_len,
                        const uint8_t* vlr, uint32_t vlr_len, Layout& L, std::vector<Chunk>& chunks, std::string& err) {
	auto u16 = [](const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8); };
	auto u32 = [](const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24); };
	auto i64 = [&](const uint8_t* p) { return (int64_t)((uint64_t)u32(p) | ((uint64_t)u32(p + 4) << 32)); };
	if (!vlr || vlr_len < 34 || (vlr_len - 34) % 6 != 0) { err = "LAZ file without a valid laszip record"; return false; }
	const uint32_t compressor = u16(vlr), coder = u16(vlr + 2);
	const uint32_t chunk_size = u32(vlr + 12);
	const uint32_t num_items = u16(vlr + 32);
	if (34 + 6 * num_items != vlr_len) { err = "malformed laszip record"; return false; }
	if (compressor != 2 || coder != 0) { err = "unsupported LAZ compressor (only LASzip's chunked point-wise coding of formats 0-3)"; return false; }
	if (pdrf < 0 || pdrf > 3) { err = "unsupported LAZ point format"; return false; }
	L.has_gps = (pdrf == 1 || pdrf == 3);
	L.has_rgb = (pdrf == 2 || pdrf == 3);
	L.rec_len = rec_len;
	L.n_extra = 0;
	// expected items: POINT10 (6) 20 B, GPSTIME11 (7) 8 B, RGB12 (8) 6 B, BYTE (0) n B, all version 2
	std::vector<uint32_t> want_type = {6}, want_size = {20};
	if (L.has_gps) { want_type.push_back(7); want_size.push_back(8); }
	if (L.has_rgb) { want_type.push_back(8); want_size.push_back(6); }
	const int std_len = 20 + (L.has_gps ? 8 : 0) + (L.has_rgb ? 6 : 0);
	if (rec_len > std_len) { want_type.push_back(0); want_size.push_back((uint32_t)(rec_len - std_len)); }
	if (num_items != want_type.size()) { err = "LAZ items do not match the point format"; return false; }
	for (uint32_t i = 0; i < num_items; i++) {
		const uint8_t* it = vlr + 34 + 6 * i;
		if (u16(it) != want_type[i] || u16(it + 2) != want_size[i] || u16(it + 4) != 2) {
			err = "unsupported LAZ item (type " + std::to_string(u16(it)) + " version " + std::to_string(u16(it + 4)) + ")";
			return false;
		}
	}
	L.n_extra = rec_len - std_len;
	if (L.n_extra > kMaxExtraBytes) { err = "too many extra bytes for the LAZ decoder"; return false; }
	chunks.clear();
	if (num_points == 0) return true;
	if (offset_to_points + 8 > size) { err = "truncated LAZ file"; return false; }
	int64_t table = i64(file + offset_to_points);
	const uint64_t chunks_start = offset_to_points + 8;
	if (table == -1) {  // written to a stream: the position is in the last 8 bytes
		if (size < 8) { err = "truncated LAZ file"; return false; }
		table = i64(file + size - 8);
	}
	if (table < (int64_t)chunks_start || (uint64_t)table + 8 > size) { err = "LAZ file without a chunk table"; return false; }
	if (u32(file + table) != 0) { err = "unsupported LAZ chunk table version"; return false; }
	const uint32_t n = u32(file + table + 4);
	// every chunk holds at least one point
	if (n == 0 || (int64_t)n > num_points) { err = "malformed LAZ chunk table"; return false; }
	// entries: IntCoder(32 bits, 2 contexts) over the previous entry
	const bool variable = chunk_size == 0xFFFFFFFFu;
	IntCoder ic;
	ic.setup(32, 2);
	Arena measure{nullptr, 0, 0, nullptr, 0, 0xFFFFFFFFu, false};
	ic.alloc_classes(measure);
	ic.alloc_correctors(measure, 1, 32);
	std::vector<uint32_t> A(measure.g_top);
	Arena ar{nullptr, 0, 0, A.data(), 0, (uint32_t)A.size(), false};
	ic.setup(32, 2);
	ic.alloc_classes(ar);
	ic.alloc_correctors(ar, 1, 32);
	ic.init();
	Decoder d;
	d.start(file + table + 8, file + size);
	std::vector<uint32_t> totals(n + 1, 0), sizes(n + 1, 0);
	for (uint32_t i = 1; i <= n; i++) {
		if (variable) totals[i] = (uint32_t)ic.decode(d, (int32_t)(i > 1 ? totals[i - 1] : 0), 0);
		sizes[i] = (uint32_t)ic.decode(d, (int32_t)(i > 1 ? sizes[i - 1] : 0), 1);
	}
	if (d.bad) { err = "malformed LAZ chunk table"; return false; }
	uint64_t start = chunks_start;
	int64_t first = 0;
	for (uint32_t i = 1; i <= n && first < num_points; i++) {
		Chunk c;
		c.start = start;
		c.end = start + sizes[i];
		c.first = first;
		int64_t cnt = variable ? (int64_t)totals[i] : (int64_t)chunk_size;
		if (cnt > num_points - first) cnt = num_points - first;
		c.count = cnt;
		if (sizes[i] == 0 || c.end > (uint64_t)table || cnt <= 0) { err = "malformed LAZ chunk table"; return false; }
		chunks.push_back(c);
		start = c.end;
		first += cnt;
	}
	if (first != num_points) { err = "LAZ chunk table does not cover every point"; return false; }
	return true;
}

}  // namespace laz
}  // namespace pcg
