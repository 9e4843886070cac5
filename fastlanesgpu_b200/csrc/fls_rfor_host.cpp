// fls_rfor_host.cpp -- host encoder of the tile-based run-length format
// (RFOR) of the reference's tile_based codecs (tile_based/src/rlebinpack.cpp:
// 9-146): tiles of 512 values, each described by its runs' values and lengths
// in two FOR bit-packed streams.  The layout is the reference's so that its
// decoder and this library's read the same bytes; the code is this project's:
// two passes over the tiles (sizes, then a prefix sum of block offsets and
// the packing), both parallel over tiles.
#include <algorithm>
#include <cstring>
#include <vector>

#include "fls_internal.h"

namespace fls {
namespace {

constexpr uint32_t kTile = FLS_RFOR_TILE;

uint32_t packed_words(uint32_t count, uint32_t bw) {
	const uint64_t bits = static_cast<uint64_t>(count) * bw;
	return bits == 0 ? 1u : static_cast<uint32_t>((bits + 31u) / 32u);
}

// Runs of one tile (the input padded with its last value past n).
struct TileRuns {
	uint32_t count = 0, min_val = 0, min_rl = 0, val_bw = 0, rl_bw = 0;
};

uint32_t at(const uint32_t* in, uint64_t n, uint64_t i) { return i < n ? in[i] : in[n - 1]; }

TileRuns scan_tile(const uint32_t* in, uint64_t n, uint64_t t, uint32_t* vals, uint32_t* lens) {
	TileRuns       r;
	const uint64_t s = t * kTile;
	uint32_t       cur = at(in, n, s), run = 1;
	for (uint32_t i = 1; i < kTile; ++i) {
		const uint32_t x = at(in, n, s + i);
		if (x != cur) {
			vals[r.count] = cur;
			lens[r.count] = run;
			++r.count;
			cur = x;
			run = 1;
		} else {
			++run;
		}
	}
	vals[r.count] = cur;
	lens[r.count] = run;
	++r.count;
	r.min_val = *std::min_element(vals, vals + r.count);
	r.min_rl  = *std::min_element(lens, lens + r.count);
	uint32_t vmax = 0, lmax = 0;
	for (uint32_t k = 0; k < r.count; ++k) {
		vmax = std::max(vmax, vals[k] - r.min_val);
		lmax = std::max(lmax, lens[k] - r.min_rl);
	}
	r.val_bw = bit_width(vmax);
	r.rl_bw  = bit_width(lmax);
	return r;
}

// Block of one stream: {minimum, bw in each byte, count, packed fields}.
void write_block(uint32_t* dst, const uint32_t* x, uint32_t count, uint32_t min, uint32_t bw) {
	dst[0]          = min;
	dst[1]          = bw * 0x01010101u;
	dst[2]          = count;
	const uint32_t w = packed_words(count, bw);
	std::memset(dst + 3, 0, 4u * w);
	if (bw == 0) { return; }
	for (uint32_t k = 0; k < count; ++k) {
		const uint64_t bit = static_cast<uint64_t>(k) * bw;
		const uint32_t v   = x[k] - min;
		const uint32_t wi = static_cast<uint32_t>(bit >> 5), sh = static_cast<uint32_t>(bit & 31u);
		dst[3 + wi] |= v << sh;
		if (sh + bw > 32u) { dst[3 + wi + 1] |= v >> (32u - sh); }
	}
}

} // namespace
} // namespace fls

using namespace fls;

extern "C" {

uint64_t fls_rfor_bound_words(uint64_t n) {
	const uint64_t tiles = (n + kTile - 1) / kTile;
	return 4u + tiles * (3u + kTile);
}

fls_status fls_rfor_encode(const uint32_t* values, uint64_t n, uint32_t* val_stream, uint32_t* rl_stream,
                           uint32_t* val_offsets, uint32_t* rl_offsets, uint64_t* n_val_words, uint64_t* n_rl_words) {
	if (!values || !val_stream || !rl_stream || !val_offsets || !rl_offsets || !n_val_words || !n_rl_words) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_rfor_encode: null pointer");
	}
	if (n == 0 || n > 0xffffffffull) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_rfor_encode: 1..2^32-1 values (the format counts rows in 32 bits)");
	}
	const uint64_t tiles = (n + kTile - 1) / kTile;
	if (fls_rfor_bound_words(n) > 0xffffffffull) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_rfor_encode: streams would pass 32-bit word offsets");
	}
	std::vector<TileRuns> runs(tiles);
#pragma omp parallel
	{
		std::vector<uint32_t> v(kTile), l(kTile);
#pragma omp for schedule(static)
		for (int64_t t = 0; t < static_cast<int64_t>(tiles); ++t) { runs[t] = scan_tile(values, n, t, v.data(), l.data()); }
	}
	// block offsets: header of 4 words, then the tiles' blocks in order
	uint64_t vo = 4, ro = 4;
	for (uint64_t t = 0; t < tiles; ++t) {
		val_offsets[t] = static_cast<uint32_t>(vo);
		rl_offsets[t]  = static_cast<uint32_t>(ro);
		vo += 3u + packed_words(runs[t].count, runs[t].val_bw);
		ro += 3u + packed_words(runs[t].count, runs[t].rl_bw);
	}
	val_offsets[tiles] = static_cast<uint32_t>(vo);
	rl_offsets[tiles]  = static_cast<uint32_t>(ro);
	const uint32_t head[4] = {kTile, 4u, static_cast<uint32_t>(tiles * kTile), values[0]};
	std::memcpy(val_stream, head, sizeof(head));
	std::memcpy(rl_stream, head, sizeof(head));
#pragma omp parallel
	{
		std::vector<uint32_t> v(kTile), l(kTile);
#pragma omp for schedule(static)
		for (int64_t t = 0; t < static_cast<int64_t>(tiles); ++t) {
			const TileRuns r = scan_tile(values, n, t, v.data(), l.data());
			write_block(val_stream + val_offsets[t], v.data(), r.count, r.min_val, r.val_bw);
			write_block(rl_stream + rl_offsets[t], l.data(), r.count, r.min_rl, r.rl_bw);
		}
	}
	*n_val_words = vo;
	*n_rl_words  = ro;
	return FLS_OK;
}

} // extern "C"
