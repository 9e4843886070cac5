// fls_host.cpp -- host (CPU) encoders of the FastLanes column format.
//
// These produce the device-resident format that the CUDA kernels decode:
//   * FastLanes 32-bit bit-packing of one 1024-value vector
//     (fastlanes/src/pack.cpp:1954-1990 for the lane/word order);
//   * the transposed order of transpose_i (fastlanes/src/transpose.cpp:4110)
//     and unrsum (fastlanes/src/unrsum.cpp:120) for delta;
//   * rle.hpp's run index (fastlanes/src/include/fls_gen/rle/rle.hpp:8-44);
//   * per-vector {bw, base, offset} metadata as in compress_ssb.cu:404-454.
// All entry points are exported through the C ABI in include/fls_gpu.h.
#include "fls_internal.h"

#include <algorithm>
#include <cstring>
#include <vector>

namespace fls {

// ------------------------------------------------------------------ layout

// Original index j -> position in the transposed order.  Chunk c = j/32 goes to
// lane (c>>1)|((c&1)<<4); element s = j%32 of the chunk sits at row
// 4*(s&7) + {0,2,1,3}[s>>3], the row visited at step s of rsum.cuh's running sum.
uint32_t transposed_pos(uint32_t j) {
	static const uint32_t quad[4] = {0, 2, 1, 3};
	const uint32_t        c = j >> 5, s = j & 31u;
	const uint32_t        lane = (c >> 1) | ((c & 1u) << 4);
	return 32u * (4u * (s & 7u) + quad[s >> 3]) + lane;
}

namespace {
struct TransposeTable {
	uint16_t pos[1024];
	TransposeTable() {
		for (uint32_t j = 0; j < 1024; ++j) { pos[j] = static_cast<uint16_t>(transposed_pos(j)); }
	}
};
const TransposeTable& ttable() {
	static const TransposeTable t;
	return t;
}

inline uint32_t lane_mask(unsigned bw) { return bw >= 32 ? 0xffffffffu : ((1u << bw) - 1u); }
inline uint32_t round_words4(uint32_t w) { return (w + 3u) & ~3u; }
inline unsigned bits_of(uint32_t v) { return v ? 32u - static_cast<unsigned>(__builtin_clz(v)) : 0u; }
} // namespace

unsigned bit_width(uint32_t v) { return bits_of(v); }

void transpose_i(const uint32_t* in, uint32_t* out) {
	const auto& t = ttable();
	for (uint32_t j = 0; j < 1024; ++j) { out[t.pos[j]] = in[j]; }
}

void untranspose(const uint32_t* in, uint32_t* out) {
	const auto& t = ttable();
	for (uint32_t j = 0; j < 1024; ++j) { out[j] = in[t.pos[j]]; }
}

// Row visited at step s of a lane's running sum (rsum.cuh order).
static inline uint32_t rsum_row(uint32_t s) {
	static const uint32_t quad[4] = {0, 2, 1, 3};
	return 4u * (s & 7u) + quad[s >> 3];
}

void unrsum(const uint32_t* in, uint32_t* out) {
	for (uint32_t lane = 0; lane < 32; ++lane) {
		uint32_t prev = in[lane];
		out[lane]     = 0;
		for (uint32_t s = 1; s < 32; ++s) {
			const uint32_t p = 32u * rsum_row(s) + lane;
			out[p]           = in[p] - prev;
			prev             = in[p];
		}
	}
}

// ------------------------------------------------------------- bit-packing

// Lane l of the vector owns rows r = 0..31 (value in[32r+l]); their bw-bit
// fields are laid LSB-first into the lane's private word stream, whose word k
// is out[32k+l].
void pack(const uint32_t* in, uint32_t* out, unsigned bw) {
	if (bw == 0) { return; }
	const uint32_t m = lane_mask(bw);
	for (uint32_t lane = 0; lane < 32; ++lane) {
		uint64_t acc  = 0;
		unsigned fill = 0;
		uint32_t k    = 0;
		for (uint32_t r = 0; r < 32; ++r) {
			acc |= static_cast<uint64_t>(in[32u * r + lane] & m) << fill;
			fill += bw;
			if (fill >= 32) {
				out[32u * k++ + lane] = static_cast<uint32_t>(acc);
				acc >>= 32;
				fill -= 32;
			}
		}
	}
}

// Sequential LSB-first packing of n dictionary values; returns words written
// (padded to a multiple of 4).
static uint32_t pack_sequential(const uint32_t* v, uint32_t n, unsigned bw, uint32_t* out) {
	const uint32_t words = round_words4((n * bw + 31u) / 32u);
	std::memset(out, 0, sizeof(uint32_t) * words);
	if (bw == 0) { return words; }
	uint64_t acc  = 0;
	unsigned fill = 0;
	uint32_t k    = 0;
	for (uint32_t i = 0; i < n; ++i) {
		acc |= static_cast<uint64_t>(v[i] & lane_mask(bw)) << fill;
		fill += bw;
		if (fill >= 32) {
			out[k++] = static_cast<uint32_t>(acc);
			acc >>= 32;
			fill -= 32;
		}
	}
	if (fill) { out[k] = static_cast<uint32_t>(acc); }
	return words;
}

// --------------------------------------------------------- vector schemes

namespace {
struct MinMax {
	int32_t mn, mx;
};
MinMax min_max(const int32_t* v) {
	int32_t mn = v[0], mx = v[0];
	for (uint32_t j = 1; j < 1024; ++j) {
		mn = std::min(mn, v[j]);
		mx = std::max(mx, v[j]);
	}
	return {mn, mx};
}

// rle.hpp: one dictionary entry per run, restarting at every 256-value
// mini-vector; the run index of value j is the global dictionary position.
uint32_t run_index(const int32_t* v, uint32_t* gidx, int32_t* dict) {
	uint32_t n = 0;
	for (uint32_t j = 0; j < 1024; ++j) {
		if ((j & 255u) == 0 || v[j] != v[j - 1]) { dict[n++] = v[j]; }
		gidx[j] = n - 1;
	}
	return n;
}
} // namespace

uint32_t vec_payload_words(uint32_t scheme, uint32_t bw, uint32_t aux) {
	switch (scheme) {
	case FLS_SCHEME_FOR: return 32u * bw;
	case FLS_SCHEME_DELTA: return 32u + 32u * bw;
	case FLS_SCHEME_RLE: return 48u + round_words4((aux * bw + 31u) / 32u);
	case FLS_SCHEME_CONST: return 0;
	case FLS_SCHEME_DICT: return 32u * bits_of(aux - 1u) + round_words4((aux * bw + 31u) / 32u);
	default: return 0;
	}
}

// Encodes one full vector; returns false if `scheme` cannot represent it.
bool encode_vector(const int32_t* in, uint32_t scheme, uint32_t layout, bool round4, uint32_t* out,
                   fls_vec_meta* m) {
	uint32_t     tmp[1024], tr[1024];
	const MinMax mm = min_max(in);
	*m              = fls_vec_meta {0, 0, static_cast<uint8_t>(scheme), 0, 0};
	switch (scheme) {
	case FLS_SCHEME_CONST:
		if (mm.mn != mm.mx) { return false; }
		m->base = mm.mn;
		return true;
	case FLS_SCHEME_FOR: {
		unsigned bw = bits_of(static_cast<uint32_t>(mm.mx) - static_cast<uint32_t>(mm.mn));
		if (round4 && bw) { bw = (bw + 3u) & ~3u; }
		for (uint32_t j = 0; j < 1024; ++j) { tmp[j] = static_cast<uint32_t>(in[j]) - static_cast<uint32_t>(mm.mn); }
		if (layout == FLS_LAYOUT_TRANSPOSED) {
			transpose_i(tmp, tr);
			pack(tr, out, bw);
		} else {
			pack(tmp, out, bw);
		}
		m->base = mm.mn;
		m->bw   = static_cast<uint8_t>(bw);
		return true;
	}
	case FLS_SCHEME_DELTA: {
		uint32_t d[1024];
		transpose_i(reinterpret_cast<const uint32_t*>(in), tr);
		unrsum(tr, d);
		uint32_t mx = 0;
		for (uint32_t j = 0; j < 1024; ++j) { mx = std::max(mx, d[j]); }
		const unsigned bw = bits_of(mx);
		std::memcpy(out, tr, sizeof(uint32_t) * 32);
		pack(d, out + 32, bw);
		m->bw = static_cast<uint8_t>(bw);
		return true;
	}
	case FLS_SCHEME_RLE: {
		uint32_t gidx[1024], d[1024];
		int32_t  dict[1024];
		const uint32_t n = run_index(in, gidx, dict);
		transpose_i(gidx, tr);
		unrsum(tr, d);
		auto* b16 = reinterpret_cast<uint16_t*>(out);
		for (uint32_t l = 0; l < 32; ++l) { b16[l] = static_cast<uint16_t>(tr[l]); }
		pack(d, out + 16, 1);
		int32_t dmn = dict[0], dmx = dict[0];
		for (uint32_t k = 1; k < n; ++k) {
			dmn = std::min(dmn, dict[k]);
			dmx = std::max(dmx, dict[k]);
		}
		const unsigned bw = bits_of(static_cast<uint32_t>(dmx) - static_cast<uint32_t>(dmn));
		for (uint32_t k = 0; k < n; ++k) { tmp[k] = static_cast<uint32_t>(dict[k]) - static_cast<uint32_t>(dmn); }
		pack_sequential(tmp, n, bw, out + 48);
		m->base = dmn;
		m->bw   = static_cast<uint8_t>(bw);
		m->aux  = static_cast<uint16_t>(n);
		return true;
	}
	case FLS_SCHEME_DICT: {
		int32_t sorted[1024];
		std::memcpy(sorted, in, sizeof(sorted));
		std::sort(sorted, sorted + 1024);
		const uint32_t n   = static_cast<uint32_t>(std::unique(sorted, sorted + 1024) - sorted);
		const unsigned cbw = bits_of(n - 1u);
		for (uint32_t j = 0; j < 1024; ++j) {
			tmp[j] = static_cast<uint32_t>(std::lower_bound(sorted, sorted + n, in[j]) - sorted);
		}
		if (layout == FLS_LAYOUT_TRANSPOSED) {
			transpose_i(tmp, tr);
			pack(tr, out, cbw);
		} else {
			pack(tmp, out, cbw);
		}
		const unsigned bw = bits_of(static_cast<uint32_t>(sorted[n - 1]) - static_cast<uint32_t>(sorted[0]));
		for (uint32_t k = 0; k < n; ++k) {
			tmp[k] = static_cast<uint32_t>(sorted[k]) - static_cast<uint32_t>(sorted[0]);
		}
		pack_sequential(tmp, n, bw, out + 32u * cbw);
		m->base = sorted[0];
		m->bw   = static_cast<uint8_t>(bw);
		m->aux  = static_cast<uint16_t>(n);
		return true;
	}
	default: return false;
	}
}

// Exact encoded size (payload + 16 B metadata) of every scheme for one vector,
// computed without packing.
void scheme_sizes(const int32_t* v, uint32_t* size5) {
	const MinMax   mm       = min_max(v);
	const unsigned rbw      = bits_of(static_cast<uint32_t>(mm.mx) - static_cast<uint32_t>(mm.mn));
	uint32_t       max_d    = 0;
	uint32_t       n_runs   = 0;
	for (uint32_t j = 0; j < 1024; ++j) {
		if ((j & 31u) != 0) { max_d = std::max(max_d, static_cast<uint32_t>(v[j]) - static_cast<uint32_t>(v[j - 1])); }
		if ((j & 255u) == 0 || v[j] != v[j - 1]) { ++n_runs; }
	}
	int32_t sorted[1024];
	std::memcpy(sorted, v, sizeof(sorted));
	std::sort(sorted, sorted + 1024);
	const uint32_t n_dist = static_cast<uint32_t>(std::unique(sorted, sorted + 1024) - sorted);
	size5[FLS_SCHEME_FOR]   = 16u + 4u * vec_payload_words(FLS_SCHEME_FOR, rbw, 0);
	size5[FLS_SCHEME_DELTA] = 16u + 4u * vec_payload_words(FLS_SCHEME_DELTA, bits_of(max_d), 0);
	// The run values span the vector's range, so their bit width is rbw.
	size5[FLS_SCHEME_RLE]   = 16u + 4u * vec_payload_words(FLS_SCHEME_RLE, rbw, n_runs);
	size5[FLS_SCHEME_CONST] = (mm.mn == mm.mx) ? 16u : 0xffffffffu;
	size5[FLS_SCHEME_DICT]  = 16u + 4u * vec_payload_words(FLS_SCHEME_DICT, rbw, n_dist);
}

// Decode-cost order used to break size ties (cheapest first), as measured for
// decode fused with a sum on B200: FOR 1x, DELTA 1.5x, RLE 2x, DICT 4.5x
// (CONST has no payload).
static const uint8_t k_cost_order[FLS_N_SCHEMES] = {FLS_SCHEME_CONST, FLS_SCHEME_FOR, FLS_SCHEME_DELTA,
                                                    FLS_SCHEME_RLE, FLS_SCHEME_DICT};

uint8_t best_scheme(const uint32_t* size5) {
	uint8_t best = k_cost_order[0];
	for (uint32_t i = 1; i < FLS_N_SCHEMES; ++i) {
		const uint8_t s = k_cost_order[i];
		if (size5[s] < size5[best]) { best = s; }
	}
	return best;
}

// 16 per-vector statistics for the learned selector, all in [0, 1].  Every
// feature is an integer count or bit width divided by a power of two, so the
// CPU and GPU (fls_mlp.cu) computations agree bit for bit.
//   0 bit width of max-min              8 bit width of mean |delta| (sum >> 10)
//   1 bit width of the largest transposed delta (DELTA payload width)
//   2 runs (rle.hpp, restarts every 256)  9 values < 2^(rbw/2) above min
//   3 rising neighbours                10 values < 2^(rbw-4) above min
//   4 falling neighbours               11 bit width of |min|
//   5 equal neighbours                 12 constant vector
//   6 occupied slots of a 1024-bit hash bitmap (distinct-value proxy)
//   7 bit width of that occupancy      13 bit width of the run count
//   14 constant 32-value chunks        15 bias (1)
void vector_stats(const int32_t* v, float* f) {
	const MinMax   mm  = min_max(v);
	const uint32_t rng = static_cast<uint32_t>(mm.mx) - static_cast<uint32_t>(mm.mn);
	const unsigned rbw = bits_of(rng);
	uint32_t       max_d = 0, n_runs = 0, n_up = 0, n_down = 0, n_eq = 0, low_half = 0, low_quarter = 0;
	uint64_t       sum_abs_d = 0;
	uint32_t       bitmap[32] = {0};
	uint32_t       const_chunks = 0;
	for (uint32_t c = 0; c < 32; ++c) {
		bool same = true;
		for (uint32_t s2 = 1; s2 < 32; ++s2) { same = same && v[32 * c + s2] == v[32 * c]; }
		const_chunks += same ? 1u : 0u;
	}
	for (uint32_t j = 0; j < 1024; ++j) {
		const uint32_t x = static_cast<uint32_t>(v[j]) - static_cast<uint32_t>(mm.mn);
		if (rbw == 0 || x < (1u << (rbw / 2))) { ++low_half; }
		if (rbw <= 4 || x < (1u << (rbw - 4))) { ++low_quarter; }
		const uint32_t h = (static_cast<uint32_t>(v[j]) * 0x9e3779b1u) >> 22; // 10-bit hash
		bitmap[h >> 5] |= 1u << (h & 31u);
		if (j == 0) {
			++n_runs;
			continue;
		}
		const int64_t dd = static_cast<int64_t>(v[j]) - static_cast<int64_t>(v[j - 1]);
		sum_abs_d += static_cast<uint64_t>(dd < 0 ? -dd : dd);
		n_up += dd > 0;
		n_down += dd < 0;
		n_eq += dd == 0;
		if ((j & 31u) != 0) { max_d = std::max(max_d, static_cast<uint32_t>(v[j]) - static_cast<uint32_t>(v[j - 1])); }
		if ((j & 255u) == 0 || dd != 0) { ++n_runs; }
	}
	uint32_t set = 0;
	for (uint32_t w = 0; w < 32; ++w) { set += static_cast<uint32_t>(__builtin_popcount(bitmap[w])); }
	const uint64_t mean_d = sum_abs_d >> 10;
	const uint32_t amin   = mm.mn < 0 ? static_cast<uint32_t>(-static_cast<int64_t>(mm.mn)) : static_cast<uint32_t>(mm.mn);
	f[0]  = static_cast<float>(rbw) / 32.0f;
	f[1]  = static_cast<float>(bits_of(max_d)) / 32.0f;
	f[2]  = static_cast<float>(n_runs) / 1024.0f;
	f[3]  = static_cast<float>(n_up) / 1024.0f;
	f[4]  = static_cast<float>(n_down) / 1024.0f;
	f[5]  = static_cast<float>(n_eq) / 1024.0f;
	f[6]  = static_cast<float>(set) / 1024.0f;
	f[7]  = static_cast<float>(bits_of(set)) / 16.0f;
	f[8]  = static_cast<float>(bits_of(static_cast<uint32_t>(std::min<uint64_t>(mean_d, 0xffffffffu)))) / 32.0f;
	f[9]  = static_cast<float>(low_half) / 1024.0f;
	f[10] = static_cast<float>(low_quarter) / 1024.0f;
	f[11] = static_cast<float>(bits_of(amin)) / 32.0f;
	f[12] = (mm.mn == mm.mx) ? 1.0f : 0.0f;
	f[13] = static_cast<float>(bits_of(n_runs)) / 16.0f;
	f[14] = static_cast<float>(const_chunks) / 32.0f;
	f[15] = 1.0f;
}

} // namespace fls
