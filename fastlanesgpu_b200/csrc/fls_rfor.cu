// fls_rfor.cu -- GPU decoder of the tile-based run-length format (RFOR) of
// the reference's tile_based codecs: decode to HBM and decode fused with a
// uint64 sum.
//
// The reference decodes a 512-value tile with a CTA of 128 threads
// (LoadRBinPack, tile_based/src/include/rlebinpack_kernel.cuh:20-145): the
// runs' values and lengths are unpacked, an exchange and a block scan turn
// the lengths into run ends, the ends are marked in shared memory, a second
// block scan turns the marks into each position's run index, and the values
// are gathered.  Here one warp decodes a tile with no block-wide barrier:
//   1. lane l unpacks a contiguous chunk of the runs' lengths, and one warp
//      scan of the chunk sums gives each run's first position;
//   2. each lane writes its runs' values to shared memory and sets the bit of
//      each run's first position in a 512-bit mask (16 words);
//   3. position p = 32 j + l (row j of the tile as 32 coalesced words) is in
//      run popc(mask bits 0..p) - 1: one broadcast word, one popc and a prefix
//      count per row; the value is gathered from shared memory.
// A tile whose block is inconsistent is skipped and flagged, never read past
// its stream.
#include "fls_pipeline.cuh"

namespace fls {
namespace {

constexpr uint32_t kTile      = FLS_RFOR_TILE;
constexpr uint32_t kRforWarps = 8;

struct RforParams {
	const uint32_t *vals, *rls, *val_off, *rl_off;
	uint64_t        n_values, n_tiles, n_val_words, n_rl_words;
	uint32_t*       out;
	unsigned long long* sum;
	uint32_t*       err;
};

__device__ __forceinline__ uint32_t packed_words(uint32_t count, uint32_t bw) {
	const uint32_t bits = count * bw; // count <= 512, bw <= 32
	return bits == 0 ? 1u : (bits + 31u) >> 5;
}

// Field k of a sequentially packed block (bit k*bw, LSB first); never reads
// past the block's last packed word.
__device__ __forceinline__ uint32_t field(const uint32_t* __restrict__ p, uint32_t k, uint32_t bw) {
	if (bw == 0) { return 0u; }
	const uint32_t bit = k * bw, w = bit >> 5, sh = bit & 31u;
	const uint32_t lo  = __ldg(p + w);
	const uint32_t hi  = (sh + bw > 32u) ? __ldg(p + w + 1) : 0u;
	const uint32_t m   = bw >= 32 ? 0xffffffffu : ((1u << bw) - 1u);
	return __funnelshift_r(lo, hi, sh) & m;
}

// The run index and value of position 32 j + lane for the 16 rows of a tile,
// handed to f(p, v); pre = run starts before mask word `lane`, minus one.
template <bool FULL, class F>
__device__ __forceinline__ void expand_rows(const uint32_t* bits, const uint32_t* vals, uint32_t pre, uint32_t lane,
                                            uint32_t live, F&& f) {
	const uint32_t upto = 0xffffffffu >> (31u - lane);
#pragma unroll
	for (uint32_t j = 0; j < kTile / 32; ++j) {
		const uint32_t w   = bits[j];
		const uint32_t idx = __shfl_sync(0xffffffffu, pre, j) + __popc(w & upto);
		const uint32_t p   = 32u * j + lane;
		if (FULL || p < live) { f(p, vals[idx]); }
	}
}

template <bool SUM>
__global__ void __launch_bounds__(kRforWarps * 32, 5) rfor_kernel(const __grid_constant__ RforParams P) {
	__shared__ uint32_t s_vals[kRforWarps][kTile];
	__shared__ uint16_t s_lens[kRforWarps][kTile];
	__shared__ uint32_t s_bits[kRforWarps][kTile / 32];
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	uint32_t*      vals = s_vals[warp];
	uint16_t*      lens = s_lens[warp];
	uint32_t*      bits = s_bits[warp];
	unsigned long long acc = 0;
	const uint64_t stride = static_cast<uint64_t>(gridDim.x) * kRforWarps;
	uint64_t       t      = static_cast<uint64_t>(blockIdx.x) * kRforWarps + warp;
	// block extents of the next tile, loaded one tile ahead
	uint32_t nvo = 0, nve = 0, nro = 0, nre = 0;
	if (t < P.n_tiles) {
		nvo = __ldg(P.val_off + t);
		nve = __ldg(P.val_off + t + 1);
		nro = __ldg(P.rl_off + t);
		nre = __ldg(P.rl_off + t + 1);
	}
	for (; t < P.n_tiles; t += stride) {
		// the tile's blocks: {minimum, bit width per byte, count, fields}
		const uint64_t vo = nvo, ve = nve, ro = nro, re = nre; // 32-bit word offsets
		if (t + stride < P.n_tiles) {
			nvo = __ldg(P.val_off + t + stride);
			nve = __ldg(P.val_off + t + stride + 1);
			nro = __ldg(P.rl_off + t + stride);
			nre = __ldg(P.rl_off + t + stride + 1);
		}
		bool     ok = vo + 3u <= ve && ve <= P.n_val_words && ro + 3u <= re && re <= P.n_rl_words;
		uint32_t vmin = 0, vbw = 0, cnt = 0, rmin = 0, rbw = 0;
		if (ok) {
			vmin = __ldg(P.vals + vo);
			vbw  = __ldg(P.vals + vo + 1) & 0xffu;
			cnt  = __ldg(P.vals + vo + 2);
			rmin = __ldg(P.rls + ro);
			rbw  = __ldg(P.rls + ro + 1) & 0xffu;
			ok   = vbw <= 32u && rbw <= 32u && cnt >= 1u && cnt <= kTile && __ldg(P.rls + ro + 2) == cnt &&
			     vo + 3u + packed_words(cnt, vbw) <= ve && ro + 3u + packed_words(cnt, rbw) <= re;
		}
		if (!ok) { // warp-uniform: every lane read the same words
			if (lane == 0) { raise_err(P.err, kErrBadMeta); }
			continue;
		}
		const uint32_t* vf = P.vals + vo + 3u;
		const uint32_t* rf = P.rls + ro + 3u;
		// 1. this lane's chunk of runs: values and lengths to shared memory,
		//    and where the chunk starts
		const uint32_t chunk = (cnt + 31u) >> 5;
		const uint32_t k0 = min(cnt, lane * chunk), k1 = min(cnt, k0 + chunk);
		uint32_t       len = 0;
		for (uint32_t k = k0; k < k1; ++k) {
			const uint32_t l = rmin + field(rf, k, rbw);
			vals[k] = vmin + field(vf, k, vbw);
			lens[k] = static_cast<uint16_t>(min(l, kTile)); // a longer run fails the cover check below
			len += l;
		}
		uint32_t incl = len;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
			if (lane >= static_cast<uint32_t>(o)) { incl += x; }
		}
		if (__shfl_sync(0xffffffffu, incl, 31) != kTile) { // the runs must cover the tile exactly
			if (lane == 0) { raise_err(P.err, kErrBadMeta); }
			continue;
		}
		// 2. run starts into the mask (each lane reads back its own lengths)
		if (lane < kTile / 32) { bits[lane] = 0u; }
		__syncwarp();
		uint32_t pos = incl - len;
		for (uint32_t k = k0; k < k1; ++k) {
			if (pos < kTile) { atomicOr(&bits[pos >> 5], 1u << (pos & 31u)); } // runs of length 0 end at the tile's end
			pos += lens[k];
		}
		__syncwarp();
		// 3. run index of position 32 j + lane from prefix counts of the mask words
		const uint32_t own = lane < kTile / 32 ? __popc(bits[lane]) : 0u;
		uint32_t       c   = own;
#pragma unroll
		for (int o = 1; o < 16; o <<= 1) {
			const uint32_t x = __shfl_up_sync(0xffffffffu, c, o);
			if (lane >= static_cast<uint32_t>(o)) { c += x; }
		}
		const uint32_t pre  = c - own - 1u; // starts before word lane, minus one
		const uint64_t row0 = t * kTile;
		const uint32_t live = static_cast<uint32_t>(min(static_cast<uint64_t>(kTile), P.n_values - row0));
		if constexpr (SUM) {
			auto add = [&](uint32_t, uint32_t v) { acc += v; };
			if (live == kTile) {
				expand_rows<true>(bits, vals, pre, lane, live, add);
			} else {
				expand_rows<false>(bits, vals, pre, lane, live, add);
			}
		} else {
			uint32_t* out = P.out + row0;
			auto      put = [&](uint32_t p, uint32_t v) { __stcs(out + p, v); };
			if (live == kTile) {
				expand_rows<true>(bits, vals, pre, lane, live, put);
			} else {
				expand_rows<false>(bits, vals, pre, lane, live, put);
			}
		}
		__syncwarp();
	}
	if constexpr (SUM) {
		const unsigned long long s = warp_sum_u64(acc);
		if (lane == 0 && s) { atomicAdd(P.sum, s); }
	}
}

fls_status rfor_launch(const fls_rfor_column* col, uint32_t* d_out, uint64_t* d_sum, fls_stream_t stream,
                       const char* who) {
	if (!col || !col->values || !col->run_lengths || !col->val_offsets || !col->rl_offsets || (!d_out && !d_sum)) {
		return set_error(FLS_ERR_INVALID_ARG, std::string(who) + ": null pointer");
	}
	if (col->n_values == 0 || col->n_values > 0xffffffffull) {
		return set_error(FLS_ERR_INVALID_ARG, std::string(who) + ": 1..2^32-1 values");
	}
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	RforParams   P {};
	P.vals        = col->values;
	P.rls         = col->run_lengths;
	P.val_off     = col->val_offsets;
	P.rl_off      = col->rl_offsets;
	P.n_values    = col->n_values;
	P.n_tiles     = (col->n_values + kTile - 1) / kTile;
	P.n_val_words = col->n_val_words;
	P.n_rl_words  = col->n_rl_words;
	P.out         = d_out;
	P.sum         = reinterpret_cast<unsigned long long*>(d_sum);
	P.err         = device_error_word(st);
	if (d_sum && (s = cuda_check(cudaMemsetAsync(d_sum, 0, sizeof(uint64_t), st), "cudaMemsetAsync")) != FLS_OK) {
		return s;
	}
	const uint32_t grid = static_cast<uint32_t>(
	    std::min<uint64_t>((P.n_tiles + kRforWarps - 1) / kRforWarps, static_cast<uint64_t>(di.sms) * 8u));
	if (d_sum) {
		rfor_kernel<true><<<grid, kRforWarps * 32, 0, st>>>(P);
	} else {
		rfor_kernel<false><<<grid, kRforWarps * 32, 0, st>>>(P);
	}
	count_launch();
	return cuda_check(cudaGetLastError(), "rfor_kernel launch");
}

} // namespace
} // namespace fls

using namespace fls;

extern "C" {

fls_status fls_rfor_decode_u32(const fls_rfor_column* col, uint32_t* d_out, fls_stream_t stream) {
	if (!d_out) { return set_error(FLS_ERR_INVALID_ARG, "fls_rfor_decode_u32: null output"); }
	return rfor_launch(col, d_out, nullptr, stream, "fls_rfor_decode_u32");
}

fls_status fls_rfor_decode_sum_u32(const fls_rfor_column* col, uint64_t* d_sum, fls_stream_t stream) {
	if (!d_sum) { return set_error(FLS_ERR_INVALID_ARG, "fls_rfor_decode_sum_u32: null output"); }
	return rfor_launch(col, nullptr, d_sum, stream, "fls_rfor_decode_sum_u32");
}

} // extern "C"
