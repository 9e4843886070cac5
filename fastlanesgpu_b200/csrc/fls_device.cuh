// fls_device.cuh -- sm_100a device building blocks of the FastLanes decoders.
//
//  * bulk-copy staging: cp.async.bulk global->shared completing on per-warp
//    mbarriers, with bounded waits (no unbounded spin anywhere);
//  * lane decoders for every vector scheme.  A warp decodes one 1024-value
//    vector; lane l produces the 32 values of its rows r = 0..31 and hands each
//    (r, value) to a callback.  Bit widths are template parameters so every
//    shift and mask is a constant (the reference's generated unpack_{bw}bw_*
//    functions, unpack.cuh:8-3329, get the same effect by code generation);
//    a warp-uniform switch per vector picks the instance.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fls_gpu.h"

namespace fls {
namespace dev {

// ------------------------------------------------------------ PTX helpers

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make mbarrier initialisation visible to the async (bulk-copy) proxy.
__device__ __forceinline__ void fence_mbar_init() {
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this thread's prior generic-proxy shared-memory accesses before
// subsequent async-proxy accesses (slot reuse by the next bulk copy).
__device__ __forceinline__ void fence_proxy_async_smem() {
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
	asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
	             : "memory");
}

// L2 policy for data read exactly once (the streamed column payloads): evict
// first, so it does not displace hash tables and group arrays kept in L2.
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
	uint64_t pol;
	asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
	return pol;
}

// 1-D bulk copy global -> shared (no multicast); size and both addresses are
// multiples of 16 bytes.  Completion is signalled on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar, uint64_t pol) {
	asm volatile(
	    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
	        smem_u32(dst)),
	    "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
	    : "memory");
}

// One poll of the stage barrier.  The thread may be suspended in hardware until
// the phase completes or `hint_ns` elapses, so waiting warps do not spin on the
// issue slots that decoding warps need.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
	uint32_t ok;
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
	    "selp.u32 %0, 1, 0, p;\n\t}"
	    : "=r"(ok)
	    : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
	    : "memory");
	return ok != 0;
}

// Bounded wait: gives up after `limit` polls of at most ~20 us each.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
	for (uint32_t i = 0; i < limit; ++i) {
		if (mbar_try_wait(bar, parity, 20000u)) { return true; }
	}
	return false;
}

__device__ __forceinline__ void st_stream(uint32_t* p, uint32_t v) { __stcs(p, v); }

// ----------------------------------------------------------- layout maps

// Row visited at step s of a lane's running sum (rsum.cuh:4-107 order).
__host__ __device__ constexpr uint32_t rsum_row(uint32_t s) {
	return 4u * (s & 7u) + ((s >> 3) == 0 ? 0u : (s >> 3) == 1 ? 2u : (s >> 3) == 2 ? 1u : 3u);
}
// Inverse of rsum_row ({0,2,1,3} is its own inverse).
__host__ __device__ constexpr uint32_t step_of_row(uint32_t r) {
	return 8u * ((r & 3u) == 0 ? 0u : (r & 3u) == 1 ? 2u : (r & 3u) == 2 ? 1u : 3u) + (r >> 2);
}
// Chunk of 32 consecutive original values held by a lane in transposed order.
__host__ __device__ constexpr uint32_t chunk_of_lane(uint32_t lane) { return ((lane & 15u) << 1) | (lane >> 4); }

// Original index (within the vector) of lane `lane`, row `r`.
__device__ __forceinline__ uint32_t orig_index(uint32_t layout, uint32_t lane, uint32_t r) {
	return layout == FLS_LAYOUT_NORMAL ? 32u * r + lane : 32u * chunk_of_lane(lane) + step_of_row(r);
}

// Rows of this lane that hold real values in a vector with `cnt` (<1024) values.
__device__ __forceinline__ uint32_t tail_rows(uint32_t layout, uint32_t lane, uint32_t cnt) {
	uint32_t m = 0;
#pragma unroll
	for (uint32_t r = 0; r < 32; ++r) { m |= (orig_index(layout, lane, r) < cnt ? 1u : 0u) << r; }
	return m;
}

// -------------------------------------------------------- bit extraction

template <int BW>
struct LaneWords {
	uint32_t w[BW > 0 ? BW : 1];
};

template <int BW>
__device__ __forceinline__ void load_words(const uint32_t* __restrict__ s, uint32_t lane, LaneWords<BW>& lw) {
#pragma unroll
	for (int k = 0; k < BW; ++k) { lw.w[k] = s[32 * k + lane]; }
}

// Value of row r (a compile-time constant after unrolling) of one lane stream.
template <int BW>
__device__ __forceinline__ uint32_t extract(const LaneWords<BW>& lw, int r) {
	if constexpr (BW == 0) {
		return 0u;
	} else if constexpr (BW == 32) {
		return lw.w[r];
	} else {
		const int      bit = r * BW, k = bit >> 5, sh = bit & 31;
		const uint32_t m   = (1u << BW) - 1u;
		if (sh + BW == 32) { return lw.w[k] >> sh; }
		if (sh + BW < 32) { return (lw.w[k] >> sh) & m; }
		return __funnelshift_r(lw.w[k], lw.w[k + 1], sh) & m;
	}
}

// FOR / DICT codes: f(r, packed value) for r = 0..31.
template <int BW, class F>
__device__ __forceinline__ void unpack_rows(const uint32_t* __restrict__ s, uint32_t lane, F&& f) {
	LaneWords<BW> lw;
	load_words<BW>(s, lane, lw);
#pragma unroll
	for (int r = 0; r < 32; ++r) { f(r, extract<BW>(lw, r)); }
}

// Rows 16 H .. 16 H + 15 of a lane stream: f(r, packed value).  `s` is the
// stream's base as unpack_rows takes it; only the word rows that hold these
// rows are read (rows 0..15 end in word row ceil(BW/2) - 1, rows 16..31 start
// in word row floor(BW/2)), so for H = 1 `s` may point below the staged half.
template <int BW, int H, class F>
__device__ __forceinline__ void unpack_half_rows(const uint32_t* __restrict__ s, uint32_t lane, F&& f) {
	static_assert(H == 0 || H == 1, "half 0 or 1");
	constexpr int k0 = H ? BW / 2 : 0, k1 = H ? BW : (BW + 1) / 2;
	LaneWords<BW> lw;
#pragma unroll
	for (int k = k0; k < k1; ++k) { lw.w[k] = s[32 * k + lane]; }
#pragma unroll
	for (int r = 16 * H; r < 16 * H + 16; ++r) { f(r, extract<BW>(lw, r)); }
}

// DELTA: 32 lane bases then packed deltas; running sum in rsum order.
template <int BW, class F>
__device__ __forceinline__ void rsum_rows(const uint32_t* __restrict__ s, uint32_t lane, F&& f) {
	LaneWords<BW> lw;
	load_words<BW>(s + 32, lane, lw);
	uint32_t acc = s[lane];
#pragma unroll
	for (int st = 0; st < 32; ++st) {
		const int r = static_cast<int>(rsum_row(st));
		acc += extract<BW>(lw, r);
		f(r, acc);
	}
}

// Warp-cooperative unpack of a sequentially packed dictionary into `dst`,
// adding the FOR base.  Must be called by all 32 lanes.
__device__ __forceinline__ void unpack_dict(const uint32_t* __restrict__ src, uint32_t n, uint32_t bw, int32_t base,
                                            uint32_t* __restrict__ dst, uint32_t lane) {
	const uint32_t m = bw >= 32 ? 0xffffffffu : ((1u << bw) - 1u);
	for (uint32_t k = lane; k < n; k += 32) {
		uint32_t v = 0;
		if (bw) {
			const uint32_t bit = k * bw, w = bit >> 5, sh = bit & 31u;
			const uint32_t hi  = (sh + bw > 32) ? src[w + 1] : 0u;
			v                  = __funnelshift_r(src[w], hi, sh) & m;
		}
		dst[k] = v + static_cast<uint32_t>(base);
	}
	__syncwarp();
}

// RLE: 16-bit lane bases, one word of 1-bit run-index deltas per lane, then the
// dictionary (already unpacked into `dict`).
template <class F>
__device__ __forceinline__ void rle_rows(const uint32_t* __restrict__ s, uint32_t lane,
                                         const uint32_t* __restrict__ dict, F&& f) {
	uint32_t       idx  = reinterpret_cast<const uint16_t*>(s)[lane];
	const uint32_t bits = s[16 + lane];
#pragma unroll
	for (int st = 0; st < 32; ++st) {
		const int r = static_cast<int>(rsum_row(st));
		idx += (bits >> r) & 1u;
		f(r, dict[idx & 1023u]);
	}
}

// ----------------------------------------------------------- vector info

struct VecInfo {
	uint64_t offset;
	int32_t  base;
	uint32_t scheme, bw, aux, words;
};

__host__ __device__ __forceinline__ uint32_t bits_of(uint32_t v) {
#ifdef __CUDA_ARCH__
	return 32u - static_cast<uint32_t>(__clz(v));
#else
	return v ? 32u - static_cast<uint32_t>(__builtin_clz(v)) : 0u;
#endif
}

__host__ __device__ __forceinline__ uint32_t payload_words(uint32_t scheme, uint32_t bw, uint32_t aux) {
	switch (scheme) {
	case FLS_SCHEME_FOR: return 32u * bw;
	case FLS_SCHEME_DELTA: return 32u + 32u * bw;
	case FLS_SCHEME_RLE: return 48u + (((aux * bw + 31u) / 32u + 3u) & ~3u);
	case FLS_SCHEME_CONST: return 0u;
	case FLS_SCHEME_DICT: return 32u * bits_of(aux - 1u) + (((aux * bw + 31u) / 32u + 3u) & ~3u);
	default: return 0u;
	}
}

// Kernel-side copy of an fls_column.
struct DevCol {
	const uint32_t*     data;
	const fls_vec_meta* meta;
	uint64_t            n_words;
	uint32_t            scheme, bw;
	int32_t             base;
	uint32_t            slot_words; // staging slot (multiple of 4, >= largest vector)
	uint32_t            layout;
	uint32_t            vec_words; // uniform columns: payload words of every vector
};

// Raw metadata for vector v (one 16-byte load; uniform columns need none).
__device__ __forceinline__ uint4 load_meta(const DevCol& c, uint64_t v) {
	if (c.meta == nullptr) { return make_uint4(0, 0, 0, 0); }
	return __ldg(reinterpret_cast<const uint4*>(c.meta) + v);
}

// Decodes the metadata and validates it against the buffer; false = bad.
__device__ __forceinline__ bool vec_info(const DevCol& c, uint64_t v, uint4 raw, VecInfo& i) {
	if (c.meta == nullptr) {
		i.scheme = c.scheme;
		i.bw     = c.bw;
		i.base   = c.base;
		i.aux    = 0;
		i.words  = payload_words(c.scheme, c.bw, 0);
		i.offset = v * i.words;
	} else {
		i.offset = (static_cast<uint64_t>(raw.y) << 32) | raw.x;
		i.base   = static_cast<int32_t>(raw.z);
		i.scheme = raw.w & 0xffu;
		i.bw     = (raw.w >> 8) & 0xffu;
		i.aux    = raw.w >> 16;
		i.words  = payload_words(i.scheme, i.bw, i.aux);
	}
	bool ok = i.scheme < FLS_N_SCHEMES && i.bw <= 32u;
	if (i.scheme == FLS_SCHEME_RLE || i.scheme == FLS_SCHEME_DICT) { ok = ok && i.aux >= 1u && i.aux <= 1024u; }
	if (!ok) { return false; }
	return (i.offset & 3u) == 0 && i.offset + i.words <= c.n_words && i.words <= c.slot_words;
}

// Decodes this lane's 32 rows of a staged vector into vals[r] (base added).
// `dict` is a 1024-word per-warp scratch used by RLE and DICT vectors.  Must be
// called by all 32 lanes (dictionary unpack).  Every operator decodes through
// this one function and then works on the register array, so the 79 unrolled
// scheme/bit-width cases are generated once per call site with a trivial body.
#define FLS_BW_CASES_0_32(X)                                                                                           \
	X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) X(19)      \
	    X(20) X(21) X(22) X(23) X(24) X(25) X(26) X(27) X(28) X(29) X(30) X(31) X(32)
#define FLS_BW_CASES_0_10(X) X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)

// With AddBase = false, FOR vectors yield the packed value p (the caller adds
// value_offset(m) = base, or folds it into its constants); every other scheme
// always yields final values.
__host__ __device__ __forceinline__ uint32_t value_offset(const VecInfo& m) {
	return m.scheme == FLS_SCHEME_FOR ? static_cast<uint32_t>(m.base) : 0u;
}

template <bool AddBase = true>
__device__ __forceinline__ void decode_vals(const uint32_t* __restrict__ s, const VecInfo& m,
                                            uint32_t* __restrict__ dict, uint32_t lane, uint32_t (&vals)[32]) {
	const uint32_t base = static_cast<uint32_t>(m.base);
	const uint32_t fadd = AddBase ? base : 0u;
	switch (m.scheme) {
	case FLS_SCHEME_FOR:
		switch (m.bw) {
#define FLS_FOR_CASE(B)                                                                                                \
	case B: unpack_rows<B>(s, lane, [&](int r, uint32_t p) { vals[r] = p + fadd; }); break;
			FLS_BW_CASES_0_32(FLS_FOR_CASE)
#undef FLS_FOR_CASE
		default: break;
		}
		break;
	case FLS_SCHEME_DELTA:
		switch (m.bw) {
#define FLS_DELTA_CASE(B)                                                                                              \
	case B: rsum_rows<B>(s, lane, [&](int r, uint32_t x) { vals[r] = x; }); break;
			FLS_BW_CASES_0_32(FLS_DELTA_CASE)
#undef FLS_DELTA_CASE
		default: break;
		}
		break;
	case FLS_SCHEME_RLE:
		unpack_dict(s + 48, m.aux, m.bw, m.base, dict, lane);
		rle_rows(s, lane, dict, [&](int r, uint32_t x) { vals[r] = x; });
		__syncwarp();
		break;
	case FLS_SCHEME_CONST:
#pragma unroll
		for (int r = 0; r < 32; ++r) { vals[r] = base; }
		break;
	case FLS_SCHEME_DICT: {
		const uint32_t cbw = bits_of(m.aux - 1u);
		unpack_dict(s + 32u * cbw, m.aux, m.bw, m.base, dict, lane);
		switch (cbw) {
#define FLS_DICT_CASE(B)                                                                                               \
	case B: unpack_rows<B>(s, lane, [&](int r, uint32_t c) { vals[r] = dict[c & 1023u]; }); break;
			FLS_BW_CASES_0_10(FLS_DICT_CASE)
#undef FLS_DICT_CASE
		default: break;
		}
		__syncwarp();
		break;
	}
	default: break;
	}
}

// Callback form of decode_vals: f(r, value) for r = 0..31, with the consumer
// inlined into each unrolled scheme / bit-width case so no value array is
// materialised.  Use it only with cheap consumers (the code is replicated once
// per case).
template <bool AddBase, class F>
__device__ __forceinline__ void decode_each(const uint32_t* __restrict__ s, const VecInfo& m,
                                            uint32_t* __restrict__ dict, uint32_t lane, F&& f) {
	const uint32_t base = static_cast<uint32_t>(m.base);
	const uint32_t fadd = AddBase ? base : 0u;
	switch (m.scheme) {
	case FLS_SCHEME_FOR:
		switch (m.bw) {
#define FLS_FOR_CASE(B)                                                                                                \
	case B: unpack_rows<B>(s, lane, [&](int r, uint32_t p) { f(r, p + fadd); }); break;
			FLS_BW_CASES_0_32(FLS_FOR_CASE)
#undef FLS_FOR_CASE
		default: break;
		}
		break;
	case FLS_SCHEME_DELTA:
		switch (m.bw) {
#define FLS_DELTA_CASE(B)                                                                                              \
	case B: rsum_rows<B>(s, lane, f); break;
			FLS_BW_CASES_0_32(FLS_DELTA_CASE)
#undef FLS_DELTA_CASE
		default: break;
		}
		break;
	case FLS_SCHEME_RLE:
		unpack_dict(s + 48, m.aux, m.bw, m.base, dict, lane);
		rle_rows(s, lane, dict, f);
		__syncwarp();
		break;
	case FLS_SCHEME_CONST:
#pragma unroll
		for (int r = 0; r < 32; ++r) { f(r, base); }
		break;
	case FLS_SCHEME_DICT: {
		const uint32_t cbw = bits_of(m.aux - 1u);
		unpack_dict(s + 32u * cbw, m.aux, m.bw, m.base, dict, lane);
		switch (cbw) {
#define FLS_DICT_CASE(B)                                                                                               \
	case B: unpack_rows<B>(s, lane, [&](int r, uint32_t c) { f(r, dict[c & 1023u]); }); break;
			FLS_BW_CASES_0_10(FLS_DICT_CASE)
#undef FLS_DICT_CASE
		default: break;
		}
		__syncwarp();
		break;
	}
	default: break;
	}
}

// ------------------------------------------------- single-row extraction

// A FOR vector prepared for reading single rows: the lane's word column in
// shared memory, bit width, mask and base.  get(r) reads two words (the second
// may lie up to 31 words past the payload: the pipeline leaves 32 words of
// slack after the stages, and the bits read from it are masked off unless the
// field straddles).  A 0-bit vector has no payload: both reads then fall on
// the slot's first word row (within the slack) and the mask drops them.
struct ForRows {
	const uint32_t* s;
	uint32_t        bw, mask, base, next;
	__device__ __forceinline__ void init(const uint32_t* slot, const VecInfo& m, uint32_t lane) {
		s    = slot + lane;
		bw   = m.bw;
		mask = m.bw >= 32 ? 0xffffffffu : ((1u << m.bw) - 1u);
		base = static_cast<uint32_t>(m.base);
		next = m.bw ? 32u : 0u;
	}
	__device__ __forceinline__ uint32_t get(uint32_t r) const {
		const uint32_t bit = r * bw, w = bit >> 5, sh = bit & 31u;
		const uint32_t* p  = s + 32u * w;
		return (__funnelshift_r(p[0], p[next], sh) & mask) + base;
	}
};

// Schemes whose rows can be read at random (no running sum): FOR, CONST, DICT.
__device__ __forceinline__ bool random_access(uint32_t scheme) {
	return scheme == FLS_SCHEME_FOR || scheme == FLS_SCHEME_CONST || scheme == FLS_SCHEME_DICT;
}

// Field of row r (runtime) of this lane's bit-packed stream.
__device__ __forceinline__ uint32_t extract_rt(const uint32_t* __restrict__ s, uint32_t bw, uint32_t lane, uint32_t r) {
	if (bw == 0) { return 0u; }
	const uint32_t bit = r * bw, w = bit >> 5, sh = bit & 31u;
	const uint32_t lo  = s[32u * w + lane];
	const uint32_t hi  = (sh + bw > 32u) ? s[32u * (w + 1u) + lane] : 0u;
	const uint32_t m   = bw >= 32 ? 0xffffffffu : ((1u << bw) - 1u);
	return __funnelshift_r(lo, hi, sh) & m;
}

// Entry k of a sequentially packed dictionary.
__device__ __forceinline__ uint32_t dict_entry(const uint32_t* __restrict__ d, uint32_t bw, uint32_t k) {
	if (bw == 0) { return 0u; }
	const uint32_t bit = k * bw, w = bit >> 5, sh = bit & 31u;
	const uint32_t hi  = (sh + bw > 32u) ? d[w + 1u] : 0u;
	const uint32_t m   = bw >= 32 ? 0xffffffffu : ((1u << bw) - 1u);
	return __funnelshift_r(d[w], hi, sh) & m;
}

// Final value of row r of a random-access (FOR / CONST / DICT) vector.
__device__ __forceinline__ uint32_t value_at(const uint32_t* __restrict__ s, const VecInfo& m, uint32_t lane,
                                             uint32_t r) {
	const uint32_t base = static_cast<uint32_t>(m.base);
	if (m.scheme == FLS_SCHEME_FOR) { return extract_rt(s, m.bw, lane, r) + base; }
	if (m.scheme == FLS_SCHEME_DICT) {
		const uint32_t cbw  = bits_of(m.aux - 1u);
		const uint32_t code = extract_rt(s, cbw, lane, r);
		return dict_entry(s + 32u * cbw, m.bw, code < m.aux ? code : 0u) + base;
	}
	return base; // CONST
}

} // namespace dev
} // namespace fls
