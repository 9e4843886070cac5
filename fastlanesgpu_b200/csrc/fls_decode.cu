// fls_decode.cu -- decode-to-HBM and decode-fused-sum operators.
//
// Reference counterparts: unpack_global (fastlanes/src/include/fls_gen/unpack/
// unpack.cuh:3436), QueryKernel of bitpack_shared_memory.cu:21 /
// bitpack_register.cu:21 (decode + sum), delta_shared_memory.cu:24 (delta +
// sum) and delta_global_memory.cu:24 (delta to global memory).
#include "fls_pipeline.cuh"

namespace fls {
namespace {

struct NoState {};

// Decode to HBM.  Values of a vector are written as 32 coalesced 128-byte rows
// with streaming stores; transposed columns can instead be reordered through a
// padded shared-memory tile (33 words per chunk, conflict-free) into original
// order.
struct DecodeOp {
	using State = NoState;
	uint32_t* out;
	uint32_t  original;
	__device__ void cta_setup(State&, uint32_t*, const StageCfg&) const {}
	__device__ void process(State&, uint64_t v, const WarpStage& ws, uint32_t st, uint32_t i, uint32_t lane,
	                        const StageCfg&) const {
		const StagedVec sv = staged(ws, st, i, 0);
		if (sv.bad()) { return; }
		uint32_t vals[32];
		dev::decode_vals(sv.s, sv.vi, ws.dict(), lane, vals);
		uint32_t* dst = out + v * 1024u;
		if (original) {
			uint32_t*      tb = ws.extra();
			const uint32_t cb = 33u * dev::chunk_of_lane(lane);
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) { tb[cb + dev::step_of_row(r)] = vals[r]; }
			__syncwarp();
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) { dev::st_stream(dst + 32u * r + lane, tb[33u * r + lane]); }
			__syncwarp();
		} else {
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) { dev::st_stream(dst + 32u * r + lane, vals[r]); }
		}
	}
	__device__ void finish(State&, uint32_t, const StageCfg&) const {}
};

struct AccState {
	unsigned long long acc;
};

// Decode fused with a uint64 sum; four independent partial sums per lane, one
// atomic per warp at the end.
struct DecodeSumOp {
	using State = AccState;
	unsigned long long* sum;
	__device__ void cta_setup(State&, uint32_t*, const StageCfg&) const {}
	__device__ void process(State& S, uint64_t v, const WarpStage& ws, uint32_t st, uint32_t i, uint32_t lane,
	                        const StageCfg& cfg) const {
		const StagedVec sv = staged(ws, st, i, 0);
		if (sv.bad()) { return; }
		uint32_t vals[32];
		// Values are summed as uint32 (base added per value: it may wrap).
		dev::decode_vals(sv.s, sv.vi, ws.dict(), lane, vals);
		const uint32_t     m = valid_rows(cfg, v, lane);
		unsigned long long p[4] = {0, 0, 0, 0};
		if (m == 0xffffffffu) { // every vector but the column's last
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) { p[r & 3] += vals[r]; }
		} else {
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) { p[r & 3] += ((m >> r) & 1u) ? vals[r] : 0u; }
		}
		S.acc += (p[0] + p[1]) + (p[2] + p[3]);
	}
	__device__ void finish(State& S, uint32_t lane, const StageCfg&) const {
		const unsigned long long s = warp_sum_u64(S.acc);
		if (lane == 0 && s) { atomicAdd(sum, s); }
	}
};

// ------------------------------------------------------------------------
// Decode fused with a sum for columns whose vectors all share one scheme
// (DELTA, RLE or DICT; scheme_mask has one bit), as the encoder produces for
// sorted keys, runs and dictionaries.  The scheme is a template parameter, so
// the per-vector scheme switch and the value array of the general operator
// disappear: each decoded value goes straight into the lane's sum.  The bit
// width stays a warp-uniform switch per vector (vectors of one column differ
// in width).  Values whose 32-row lane sum cannot exceed 32 bits (every value
// below 2^27, known from the vector's base and width) are summed in 32 bits.
//
// The reference times delta decode + sum as delta_shared_memory.cu:24-61
// (unpack to shared memory, d_rsum_32, BlockLoad, BlockSum per 1024 values).

template <int BW>
__device__ __forceinline__ unsigned long long delta_lane_sum(const uint32_t* __restrict__ s, uint32_t lane,
                                                             uint32_t rows) {
	dev::LaneWords<BW> lw;
	dev::load_words<BW>(s + 32, lane, lw);
	uint32_t           x   = s[lane];
	unsigned long long acc = 0;
	if constexpr (BW <= 22) {
		if (rows == 0xffffffffu) {
			// Value s is base + p_s with p_s the running sum of the deltas.
			// For BW <= 22, p_31 < 2^27 and the sum of the 32 p_s < 2^32, so
			// the p_s sum in 32 bits and the base is added once -- exact
			// unless base + p_31 wraps (then the full path below runs).
			uint32_t p = 0, ps = 0;
#pragma unroll
			for (int st = 0; st < 32; ++st) {
				p += dev::extract<BW>(lw, static_cast<int>(dev::rsum_row(st)));
				ps += p;
			}
			if (static_cast<uint64_t>(x) + p < (1ull << 32)) {
				return 32ull * x + ps;
			}
		}
	}
	if (rows == 0xffffffffu) {
#pragma unroll
		for (int st = 0; st < 32; ++st) {
			x += dev::extract<BW>(lw, static_cast<int>(dev::rsum_row(st)));
			acc += x;
		}
	} else {
#pragma unroll
		for (int st = 0; st < 32; ++st) {
			const int r = static_cast<int>(dev::rsum_row(st));
			x += dev::extract<BW>(lw, r);
			acc += ((rows >> r) & 1u) ? x : 0u;
		}
	}
	return acc;
}

// The rows `rows` of a column's last, partial vector, any code width (one
// vector per column: a plain loop).
__device__ __noinline__ unsigned long long dict_lane_sum_rows(const uint32_t* __restrict__ s,
                                                             const uint32_t* __restrict__ dict, uint32_t lane,
                                                             uint32_t cbw, uint32_t rows) {
	unsigned long long acc = 0;
	const uint32_t     m   = cbw >= 32 ? 0xffffffffu : ((1u << cbw) - 1u);
	for (uint32_t r = 0; r < 32; ++r) {
		if (cbw == 0 || !((rows >> r) & 1u)) {
			acc += ((rows >> r) & 1u) ? dict[0] : 0u;
			continue;
		}
		const uint32_t bit = r * cbw, w = bit >> 5, sh = bit & 31u;
		const uint32_t lo = s[32u * w + lane], hi = sh + cbw > 32u ? s[32u * (w + 1u) + lane] : 0u;
		acc += dict[(__funnelshift_r(lo, hi, sh) & m) & 1023u];
	}
	return acc;
}

// True when every value of the vector (base + a bw-bit field) is below 2^27.
__device__ __forceinline__ bool small_values(const VecInfo& m) {
	const uint64_t top = static_cast<uint64_t>(static_cast<uint32_t>(m.base)) +
	                     (m.bw >= 32 ? 0xffffffffull : ((1ull << m.bw) - 1ull));
	return top < (1ull << 27);
}

// FULL: every row of the lane holds a value (all vectors but a column's
// last), so no row is tested.
template <bool Small, bool FULL>
__device__ __forceinline__ unsigned long long rle_lane_sum(const uint32_t* __restrict__ s,
                                                           const uint32_t* __restrict__ dict, uint32_t lane,
                                                           uint32_t rows) {
	uint32_t           idx  = reinterpret_cast<const uint16_t*>(s)[lane];
	const uint32_t     bits = s[16 + lane];
	uint32_t           s32  = 0;
	unsigned long long s64  = 0;
#pragma unroll
	for (int st = 0; st < 32; ++st) {
		const int r = static_cast<int>(dev::rsum_row(st));
		idx += (bits >> r) & 1u;
		const uint32_t v = (FULL || ((rows >> r) & 1u)) ? dict[idx & 1023u] : 0u;
		if constexpr (Small) {
			s32 += v;
		} else {
			s64 += v;
		}
	}
	return Small ? static_cast<unsigned long long>(s32) : s64;
}

// A whole vector (every row holds a value) at code width CBW.
template <int CBW, bool Small>
__device__ __forceinline__ unsigned long long dict_lane_sum(const uint32_t* __restrict__ s,
                                                            const uint32_t* __restrict__ dict, uint32_t lane) {
	dev::LaneWords<CBW> lw;
	dev::load_words<CBW>(s, lane, lw);
	uint32_t           s32 = 0;
	unsigned long long s64 = 0;
#pragma unroll
	for (int r = 0; r < 32; ++r) {
		const uint32_t v = dict[dev::extract<CBW>(lw, r) & 1023u];
		if constexpr (Small) {
			s32 += v;
		} else {
			s64 += v;
		}
	}
	return Small ? static_cast<unsigned long long>(s32) : s64;
}

// Sequentially FOR-packed dictionary of n entries at bit width BW into dst
// (base added), lanes striding over the entries.
template <int BW>
__device__ __forceinline__ void unpack_dict_bw(const uint32_t* __restrict__ src, uint32_t n, int32_t base,
                                               uint32_t* __restrict__ dst, uint32_t lane) {
	const uint32_t b = static_cast<uint32_t>(base);
	for (uint32_t k = lane; k < n; k += 32) {
		uint32_t v = 0;
		if constexpr (BW == 32) {
			v = src[k];
		} else if constexpr (BW > 0) {
			const uint32_t bit = k * BW, w = bit >> 5, sh = bit & 31u;
			const uint32_t hi  = (sh + BW > 32u) ? src[w + 1] : 0u; // never past the dictionary
			v                  = __funnelshift_r(src[w], hi, sh) & ((1u << BW) - 1u);
		}
		dst[k] = v + b;
	}
	__syncwarp();
}

__device__ __forceinline__ void unpack_dict_any(const uint32_t* __restrict__ src, uint32_t n, uint32_t bw,
                                                int32_t base, uint32_t* __restrict__ dst, uint32_t lane) {
	switch (bw) {
#define FLS_DICT_UNPACK(B)                                                                                             \
	case B: unpack_dict_bw<B>(src, n, base, dst, lane); break;
		FLS_BW_CASES_0_32(FLS_DICT_UNPACK)
#undef FLS_DICT_UNPACK
	default: break;
	}
}

template <uint32_t SCHEME>
struct SchemeSumOp {
	using State = AccState;
	unsigned long long* sum;
	__device__ void cta_setup(State&, uint32_t*, const StageCfg&) const {}
	__device__ void process(State& S, uint64_t v, const WarpStage& ws, uint32_t st, uint32_t i, uint32_t lane,
	                        const StageCfg& cfg) const {
		const StagedVec sv = staged(ws, st, i, 0);
		if (sv.bad()) { return; }
		const uint32_t rows = valid_rows(cfg, v, lane);
		if (sv.vi.scheme != SCHEME) { // the host saw one scheme; any other vector is flagged, not read
			if (lane == 0) { raise_err(cfg.err, kErrBadMeta); }
			return;
		}
		if constexpr (SCHEME == FLS_SCHEME_DELTA) {
			switch (sv.vi.bw) {
#define FLS_DELTA_SUM(B)                                                                                               \
	case B: S.acc += delta_lane_sum<B>(sv.s, lane, rows); break;
				FLS_BW_CASES_0_32(FLS_DELTA_SUM)
#undef FLS_DELTA_SUM
			default: break;
			}
		} else if constexpr (SCHEME == FLS_SCHEME_RLE) {
			uint32_t* dict = ws.dict();
			unpack_dict_any(sv.s + 48, sv.vi.aux, sv.vi.bw, sv.vi.base, dict, lane);
			if (__all_sync(0xffffffffu, rows == 0xffffffffu)) {
				S.acc += small_values(sv.vi) ? rle_lane_sum<true, true>(sv.s, dict, lane, rows)
				                             : rle_lane_sum<false, true>(sv.s, dict, lane, rows);
			} else {
				S.acc += small_values(sv.vi) ? rle_lane_sum<true, false>(sv.s, dict, lane, rows)
				                             : rle_lane_sum<false, false>(sv.s, dict, lane, rows);
			}
			__syncwarp();
		} else {
			uint32_t*      dict = ws.dict();
			const uint32_t cbw  = dev::bits_of(sv.vi.aux - 1u);
			unpack_dict_any(sv.s + 32u * cbw, sv.vi.aux, sv.vi.bw, sv.vi.base, dict, lane);
			const bool small = small_values(sv.vi);
			if (!__all_sync(0xffffffffu, rows == 0xffffffffu)) {
				S.acc += dict_lane_sum_rows(sv.s, dict, lane, cbw, rows);
			} else {
				switch (cbw) {
#define FLS_DICT_SUM(B)                                                                                                \
	case B: S.acc += small ? dict_lane_sum<B, true>(sv.s, dict, lane) : dict_lane_sum<B, false>(sv.s, dict, lane); break;
					FLS_BW_CASES_0_10(FLS_DICT_SUM)
#undef FLS_DICT_SUM
				default: break;
				}
			}
			__syncwarp();
		}
	}
	__device__ void finish(State& S, uint32_t lane, const StageCfg&) const {
		const unsigned long long s = warp_sum_u64(S.acc);
		if (lane == 0 && s) { atomicAdd(sum, s); }
	}
};

// The single scheme of a per-vector column that has a specialised sum, or
// FLS_N_SCHEMES.
uint32_t single_scheme(const fls_column& c) {
	if (!c.meta) { return FLS_N_SCHEMES; }
	const uint32_t m = c.scheme_mask;
	if (m == (1u << FLS_SCHEME_DELTA)) { return FLS_SCHEME_DELTA; }
	if (m == (1u << FLS_SCHEME_RLE)) { return FLS_SCHEME_RLE; }
	if (m == (1u << FLS_SCHEME_DICT)) { return FLS_SCHEME_DICT; }
	return FLS_N_SCHEMES;
}

} // namespace
} // namespace fls

using namespace fls;

extern "C" {

fls_status fls_decode_u32(const fls_column* col, uint32_t* d_out, uint32_t order, fls_stream_t stream) {
	if (!col || !d_out) { return set_error(FLS_ERR_INVALID_ARG, "fls_decode_u32: null pointer"); }
	if (order > FLS_ORDER_ORIGINAL) { return set_error(FLS_ERR_INVALID_ARG, "fls_decode_u32: bad order"); }
	StageCfg   cfg;
	uint32_t   grid, threads;
	size_t     smem;
	const bool orig = order == FLS_ORDER_ORIGINAL && col->layout == FLS_LAYOUT_TRANSPOSED;
	fls_status s    = plan_stages(col, 1, orig ? kTBufWords : 0u, 0u, cfg, grid, threads, smem);
	if (s != FLS_OK) { return s; }
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	if (tuning_jit() && !orig) {
		bool used = false;
		s         = jit_decode(col, 1, d_out, nullptr, st, used);
		if (s != FLS_OK || used) { return s; }
	}
	DecodeOp op {};
	op.out      = d_out;
	op.original = orig ? 1u : 0u;
	return launch_staged(cfg, op, grid, threads, smem, st);
}

fls_status fls_decode_sum_u32(const fls_column* col, uint64_t* d_sum, fls_stream_t stream) {
	if (!col || !d_sum) { return set_error(FLS_ERR_INVALID_ARG, "fls_decode_sum_u32: null pointer"); }
	StageCfg   cfg;
	uint32_t   grid, threads;
	size_t     smem;
	fls_status s = plan_stages(col, 1, 0u, 0u, cfg, grid, threads, smem);
	if (s != FLS_OK) { return s; }
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	if ((s = cuda_check(cudaMemsetAsync(d_sum, 0, sizeof(uint64_t), st), "cudaMemsetAsync")) != FLS_OK) { return s; }
	if (tuning_jit()) {
		bool used = false;
		s         = jit_decode(col, 0, nullptr, d_sum, st, used);
		if (s != FLS_OK || used) { return s; }
	}
	if (tuning_jit()) {
		auto* sum = reinterpret_cast<unsigned long long*>(d_sum);
		switch (single_scheme(*col)) {
		case FLS_SCHEME_DELTA: return launch_staged(cfg, SchemeSumOp<FLS_SCHEME_DELTA> {sum}, grid, threads, smem, st);
		case FLS_SCHEME_RLE: return launch_staged(cfg, SchemeSumOp<FLS_SCHEME_RLE> {sum}, grid, threads, smem, st);
		case FLS_SCHEME_DICT: return launch_staged(cfg, SchemeSumOp<FLS_SCHEME_DICT> {sum}, grid, threads, smem, st);
		default: break;
		}
	}
	DecodeSumOp op {};
	op.sum = reinterpret_cast<unsigned long long*>(d_sum);
	return launch_staged(cfg, op, grid, threads, smem, st);
}

} // extern "C"
