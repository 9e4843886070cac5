// fls_fixed.cuh -- query kernels specialised to one query shape.
//
// For queries whose columns are all uniform FOR columns (the reference's
// column format: one bit width and base per column, fls_q11.cu:202-223), the
// library compiles these templates at first use with NVRTC for the exact shape
// and caches the kernel (fls_jit.cu).  Everything the general operators decide
// per vector at run time -- which decoder, how many filters or probes, where
// the aggregate columns are, which table lives in shared memory, which
// predicates remain for the row-at-a-time loop -- becomes a compile-time
// constant here.  Results are identical to the general operators.
//
//  * filter-aggregate (FilterQuery): columns staged in filter order (column f
//    holds filter f), then aggregate columns no filter reads;
//  * probe + group-by (ProbeQuery): columns staged in probe order (column q
//    holds the key of probe q), then the measure column if no probe reads it;
//  * decode fused with a sum, and decode to HBM (DecodeQuery): one column.
#pragma once

#include "fls_device.cuh"

namespace fls {
namespace fixed {

constexpr uint32_t kSlack         = 32;      // words after the stages (row reads look one word row ahead)
constexpr uint32_t kWaitPolls     = 1u << 17; // bounded stage waits (each <= ~20 us)
constexpr uint32_t kErrTimeoutBit = 1u << 2;
constexpr uint32_t kErrHashBit    = 1u << 3;
constexpr int      kDenseAggRows  = 16; // above this many rows in some lane, aggregate whole vectors
constexpr int      kRowBatch      = 4;  // selected rows per lane whose table reads are in flight together
constexpr uint32_t kFreeSlot      = 0xffffffffu; // tag of an unclaimed group-sum slot
constexpr int      kMaxDenseProbes = 2; // probes compiled for whole-vector evaluation (each unrolls 32 rows)
constexpr uint32_t kRowList       = 256; // entries of a join warp's list of selected rows (16 bits each)
constexpr uint32_t kRowListWords  = kRowList / 2;

// The staged pipeline's parameters (shared by both operators).
struct StageParams {
	const uint32_t* data[FLS_MAX_QUERY_COLS];
	uint64_t        n_values, n_vec, n_tiles;
	uint32_t        tile, stages, warps, warp_smem_words, stage_words, bar_off;
	uint32_t*       err;
	uint32_t        cta_off;  // words: CTA-wide scratch (hash tables) after the warps' areas
	uint32_t        list_off; // words into a warp's area: its row list (join kernels), after the barriers
};

struct FilterParams {
	StageParams         S;
	uint32_t            base[FLS_MAX_QUERY_COLS]; // FOR base of each staged column
	uint32_t            lo[FLS_MAX_FILTERS];      // filter lower bound (unsigned wrap)
	uint32_t            range[FLS_MAX_FILTERS];   // hi - lo
	uint32_t            field_lo[FLS_MAX_FILTERS]; // SWAR filters: bounds on the packed field, in [0, 2^bw]
	uint32_t            field_hi[FLS_MAX_FILTERS]; //   (an empty range is (1, 0))
	int32_t             sparse_rows;
	uint32_t            pad_;
	unsigned long long* result;
};

struct ProbeParams {
	StageParams    S;
	uint32_t       base[FLS_MAX_QUERY_COLS];
	const int32_t* ht[FLS_MAX_PROBES];
	int32_t        len[FLS_MAX_PROBES];
	int32_t        kmin[FLS_MAX_PROBES];
	uint32_t       smem_off[FLS_MAX_PROBES]; // words into the CTA scratch (tables flagged as shared)
	int32_t        key_mul[FLS_MAX_GROUP_KEYS];
	int32_t        key_slot[FLS_MAX_GROUP_KEYS]; // word of each key in the group record, -1 = not written
	int32_t        sub, n_groups, sparse_rows;
	uint32_t       stride, sum_slot; // group record: int32 words, word of the int64 sum
	uint32_t       gsum_off;         // GSM: words into the CTA scratch of the group-sum slots
	uint32_t       gslot_mask;       // GSM: slots - 1 (a power of two)
	uint32_t       sum32;            // 1: wrapping int32 sum in one record word, 0: int64 in two
	const uint32_t* bits;            // presence bitmaps at the tables' shared-memory offsets
	int32_t*       res;
	const uint32_t* gcol[2];         // columns kNS, kNS + 1 (not staged): packed words in global memory
};

struct DecodeParams {
	StageParams         S;
	uint32_t            base; // FOR base of the column
	uint32_t            pad_;
	unsigned long long* sum;  // decode-sum: uint64 total
	uint32_t*           out;  // decode to HBM: n_vec * 1024 values
};

// The host (nvcc + host compiler) and NVRTC must agree on the parameter
// blocks.  Every field is naturally aligned and padded explicitly, so equal
// sizes mean equal offsets.
static_assert(sizeof(StageParams) == 128 && alignof(StageParams) == 8, "StageParams layout");
static_assert(sizeof(FilterParams) == 240, "FilterParams layout");
static_assert(sizeof(ProbeParams) == 328, "ProbeParams layout");
static_assert(sizeof(DecodeParams) == 152, "DecodeParams layout");

// Bit widths of the staged columns and where they sit in a stage.
template <int LAYOUT, int... BWS>
struct Shape {
	static constexpr int NC      = sizeof...(BWS);
	static constexpr int kNS     = NC; // columns staged in shared memory (the first kNS)
	static constexpr int kLayout = LAYOUT;
	__host__ __device__ static constexpr int bw(int c) {
		int i = 0, r = 0;
		((r = (i++ == c ? BWS : r)), ...);
		return r;
	}
	__host__ __device__ static constexpr int vec_words(int c) { return 32 * bw(c); }
	__host__ __device__ static constexpr int prefix(int c) {
		int s = 0;
		for (int i = 0; i < c; ++i) { s += 32 * bw(i); }
		return s;
	}
	// Half-vector tiles: a tile holds rows 0..15 or rows 16..31 of every lane,
	// ceil(bw/2) word rows of each column (half 1 starts at word row
	// floor(bw/2)).
	static constexpr bool kHalf = false;
	__host__ __device__ static constexpr int half_words(int c) { return 32 * ((bw(c) + 1) / 2); }
	__host__ __device__ static constexpr int half_skip(int c) { return 32 * (bw(c) / 2); }
	__host__ __device__ static constexpr int half_prefix(int c) {
		int s = 0;
		for (int i = 0; i < c; ++i) { s += half_words(i); }
		return s;
	}
	static_assert(NC >= 1 && NC <= FLS_MAX_QUERY_COLS, "1..8 staged columns");
};

// SWAR bit f: filter f may test packed fields several at a time against
// field_lo/field_hi (the host proved base + 2^bw - 1 <= INT32_MAX, so the
// decoded values do not wrap and value in [lo, hi] <=> field in
// [lo - base, hi - base] clamped to the field's domain).
template <int LAYOUT, int NF, int AGG_A, int AGG_B, int SWAR, int... BWS>
struct FilterQuery : Shape<LAYOUT, BWS...> {
	static constexpr int kNF   = NF;
	static constexpr int kAggA = AGG_A;
	static constexpr int kAggB = AGG_B;
	__host__ __device__ static constexpr bool swar(int f) { return (SWAR >> f) & 1; }
	static_assert(NF >= 0 && NF <= FLS_MAX_FILTERS, "0..4 filters");
	static_assert(AGG_B < 0 || AGG_A >= 0, "sum(a*b) needs a");
};

// AGG / SUB: staged columns of the measure and of the column subtracted from
// it (-1: none).  NK group keys, the payloads of probes K0, K1, K2.  KINDS bit
// q: probe q is PHT_2; SMEM bit q: probe q's table is in shared memory (PHT_1
// as a presence bitmap, PHT_2 verbatim); PBIT bit q: a PHT_2 table too large
// for shared memory has its presence bitmap there (a slot hits when its 64-bit
// entry is not zero), its payloads stay in global memory; DIRECT bit q: the
// host proved every key of probe q's column lands in [keys_min, keys_min +
// len) (from the column's base and bit width), so its slot is key - keys_min;
// DIRECT bit 8 + q: also base == keys_min, so the slot is the packed field.
// GSM: each CTA sums its groups in a direct-mapped cache of group-sum slots
// in shared memory (a group claims its slot, or else adds to its record
// directly) and adds the slots' non-zero sums to the records once, at its end.
// HALF: tiles are half vectors (rows 0..15 or 16..31 of every lane), so a
// stage takes half the shared memory and twice the warps fit beside the
// tables.
template <int LAYOUT, int NP, int AGG, int SUB, int NK, int K0, int K1, int K2, int KINDS, int SMEM, int PBIT,
          int DIRECT, int GSM, int HALF, int NS, int... BWS>
struct ProbeQuery : Shape<LAYOUT, BWS...> {
	static constexpr bool kHalf = HALF != 0;
	static constexpr int kNP  = NP;
	static constexpr int kAgg = AGG;
	static constexpr int kSub = SUB;
	static constexpr int kNK  = NK;
	static constexpr bool kGroupSmem = GSM != 0;
	static constexpr int  kNS        = NS; // staged columns; the measure columns past them stay in global memory
	__host__ __device__ static constexpr int key_probe(int k) { return k == 0 ? K0 : k == 1 ? K1 : K2; }
	__host__ __device__ static constexpr bool pht2(int q) { return (KINDS >> q) & 1; }
	__host__ __device__ static constexpr bool in_smem(int q) { return (SMEM >> q) & 1; }
	__host__ __device__ static constexpr bool pbit(int q) { return (PBIT >> q) & 1; }
	// Probes whose hit test reads shared memory only (or a PHT_1 array).
	__host__ __device__ static constexpr bool dense_ok(int q) { return !pht2(q) || in_smem(q) || pbit(q); }
	__host__ __device__ static constexpr bool direct(int q) { return (DIRECT >> q) & 1; }
	__host__ __device__ static constexpr bool field_slot(int q) { return direct(q) && ((DIRECT >> (8 + q)) & 1); }
	// Probes whose hit test is one bit of a shared-memory bitmap.
	__host__ __device__ static constexpr bool smem_bits(int q) { return (in_smem(q) && !pht2(q)) || pbit(q); }
	static_assert(NP >= 1 && NP <= FLS_MAX_PROBES, "1..4 probes");
	static_assert(NS >= NP && NS <= static_cast<int>(sizeof...(BWS)) && static_cast<int>(sizeof...(BWS)) - NS <= 2,
	              "probe columns staged; at most two columns in global memory");
};

// MODE 0: decode fused with a uint64 sum; MODE 1: decode to HBM in stored
// order.  NOWRAP: the host proved base + (2^BW - 1) < 2^32, so no decoded
// value wraps and the base can be added once per vector (sum of x + base =
// sum of x + count * base).
template <int LAYOUT, int BW, int MODE, bool NOWRAP>
struct DecodeQuery : Shape<LAYOUT, BW> {
	static constexpr int  kMode   = MODE;
	static constexpr bool kNoWrap = NOWRAP;
};

// Row r of this lane's stream at compile-time bit width (runtime row).
template <int BW>
__device__ __forceinline__ uint32_t row_field(const uint32_t* __restrict__ s, uint32_t lane, uint32_t r) {
	if constexpr (BW == 0) {
		return 0u;
	} else {
		const uint32_t  bit = r * BW;
		const uint32_t* p   = s + 32u * (bit >> 5) + lane;
		if constexpr (BW == 32) {
			return p[0];
		} else {
			return __funnelshift_r(p[0], p[32], bit & 31u) & ((1u << BW) - 1u);
		}
	}
}

__device__ __forceinline__ int max_rows(uint32_t mask) { return __reduce_max_sync(0xffffffffu, __popc(mask)); }

// Where the columns of tile vector i sit in the stage.  Half-vector tiles
// (h = the half): the base of column C's lane streams such that word row k
// is at 32 k + lane, for the word rows the half holds (for h = 1 this lies
// below the staged words, which start at word row floor(bw/2)).
template <class Q>
struct Vec {
	const uint32_t* stage;
	uint32_t        k, i, h;
	template <int C>
	__device__ __forceinline__ const uint32_t* col() const {
		if constexpr (Q::kHalf) {
			return stage + Q::half_prefix(C) - (h ? Q::half_skip(C) : 0);
		} else {
			constexpr uint32_t pre = Q::prefix(C), vw = Q::vec_words(C);
			return stage + k * pre + i * vw;
		}
	}
};

// f(r, packed field of column C) for the rows of this lane the tile holds:
// all 32, or the 16 of a half-vector tile.
template <class Q, int C, class F>
__device__ __forceinline__ void unpack_tile_rows(const Vec<Q>& V, uint32_t lane, F&& f) {
	if constexpr (Q::kHalf) {
		if (V.h) {
			dev::unpack_half_rows<Q::bw(C), 1>(V.template col<C>(), lane, f);
		} else {
			dev::unpack_half_rows<Q::bw(C), 0>(V.template col<C>(), lane, f);
		}
	} else {
		dev::unpack_rows<Q::bw(C)>(V.template col<C>(), lane, f);
	}
}

__device__ __forceinline__ uint32_t valid_rows(const StageParams& S, int layout, uint64_t v, uint32_t lane) {
	const uint64_t start = v * 1024u;
	if (start + 1024u <= S.n_values) { return 0xffffffffu; }
	return dev::tail_rows(static_cast<uint32_t>(layout), lane, static_cast<uint32_t>(S.n_values - start));
}

// ------------------------------------------------------------ filter-aggregate

// Row r's field of a lane stream, unmasked above the field (one shift).
template <int BW>
__device__ __forceinline__ uint32_t field_raw(const dev::LaneWords<BW>& lw, int r) {
	const int bit = r * BW, k = bit >> 5, sh = bit & 31;
	if (sh + BW <= 32) { return lw.w[k] >> sh; }
	return __funnelshift_r(lw.w[k], lw.w[k + 1], sh);
}

// In-range row mask of a 4-bit column, eight rows per word: even and odd
// nibbles go to bytes below a guard bit 0x80, so (x + 0x80 - lo) and
// (hi + 0x80 - x) keep the guard exactly when lo <= x and x <= hi, with no
// borrow across bytes; a multiply gathers the eight flags of a word.
__device__ __forceinline__ uint32_t swar_mask_bw4(const dev::LaneWords<4>& lw, uint32_t L, uint32_t H) {
	const uint32_t c1 = 0x80808080u - L * 0x01010101u, c2 = (H | 0x80u) * 0x01010101u;
	uint32_t       y[4];
#pragma unroll
	for (int k = 0; k < 4; ++k) {
		const uint32_t e  = lw.w[k] & 0x0F0F0F0Fu, o = (lw.w[k] >> 4) & 0x0F0F0F0Fu;
		const uint32_t re = (e + c1) & (c2 - e) & 0x80808080u;
		const uint32_t ro = (o + c1) & (c2 - o) & 0x80808080u;
		// bits 8j, 8j+1 = rows 8k+2j, 8k+2j+1; the multiply packs them into byte 3
		y[k] = ((re >> 7) | (ro >> 6)) * 0x01041040u;
	}
	return __byte_perm(__byte_perm(y[0], y[1], 0x0073), __byte_perm(y[2], y[3], 0x0073), 0x5410);
}

// In-range row mask of an even width <= 14: rows p and p + 16 share their bit
// offset, so both fields are tested at once in two 16-bit halves below guard
// bits 0x8000.
template <int BW>
__device__ __forceinline__ uint32_t swar_mask_pairs(const dev::LaneWords<BW>& lw, uint32_t L, uint32_t H) {
	constexpr uint32_t M2 = ((1u << BW) - 1u) * 0x00010001u, G = 0x80008000u;
	const uint32_t     c1 = G - L * 0x00010001u, c2 = (H | 0x8000u) * 0x00010001u;
	uint32_t           acc = 0;
#pragma unroll
	for (int p = 15; p >= 0; --p) {
		const uint32_t f = __byte_perm(field_raw<BW>(lw, p), field_raw<BW>(lw, p + 16), 0x5410) & M2;
		acc              = acc * 2u + (((f + c1) & (c2 - f) & G) >> 15); // bits p and 16 + p after the loop
	}
	return acc;
}

template <class Q, int F>
__device__ __forceinline__ void dense_filter(const FilterParams& P, const Vec<Q>& V, uint32_t lane, uint32_t& mask) {
	constexpr int BW = Q::bw(F);
	if constexpr (Q::swar(F) && BW == 4) {
		dev::LaneWords<4> lw;
		dev::load_words<4>(V.template col<F>(), lane, lw);
		mask &= swar_mask_bw4(lw, P.field_lo[F], P.field_hi[F]);
	} else if constexpr (Q::swar(F) && BW % 2 == 0 && BW >= 2 && BW <= 14) {
		dev::LaneWords<BW> lw;
		dev::load_words<BW>(V.template col<F>(), lane, lw);
		mask &= swar_mask_pairs<BW>(lw, P.field_lo[F], P.field_hi[F]);
	} else {
		const uint32_t lo = P.lo[F] - P.base[F], range = P.range[F];
		uint32_t       m[4] = {0, 0, 0, 0};
		dev::unpack_rows<BW>(V.template col<F>(), lane,
		                     [&](int r, uint32_t p) { m[r & 3] |= (p - lo <= range ? 1u : 0u) << r; });
		mask &= (m[0] | m[1]) | (m[2] | m[3]);
	}
}

// Dense filters F, F+1, ... while some lane keeps more than sparse_rows rows;
// f0 receives the first filter left to the row loop (NF if none).
template <class Q, int F>
__device__ __forceinline__ void dense_filters(const FilterParams& P, const Vec<Q>& V, uint32_t lane, uint32_t& mask,
                                              int& f0) {
	if constexpr (F < Q::kNF) {
		if (max_rows(mask) <= P.sparse_rows) {
			f0 = F;
			return;
		}
		dense_filter<Q, F>(P, V, lane, mask);
		dense_filters<Q, F + 1>(P, V, lane, mask, f0);
	} else {
		f0 = Q::kNF;
	}
}

template <class Q, int F>
__device__ __forceinline__ bool row_pass(const FilterParams& P, const Vec<Q>& V, uint32_t lane, uint32_t r) {
	if constexpr (F < Q::kNF) {
		const bool ok = (row_field<Q::bw(F)>(V.template col<F>(), lane, r) - (P.lo[F] - P.base[F])) <= P.range[F];
		return ok & row_pass<Q, F + 1>(P, V, lane, r);
	} else {
		return true;
	}
}

template <class Q, int C>
__device__ __forceinline__ int32_t row_value(const uint32_t* base, const Vec<Q>& V, uint32_t lane, uint32_t r) {
	return static_cast<int32_t>(row_field<Q::bw(C)>(V.template col<C>(), lane, r) + base[C]);
}

// Field of row r of `lane` in vector v of a column left in global memory
// (uniform FOR: vector v at word 32*BW*v, word k of the lane at 32k + lane);
// the second word is read only when the field straddles, so every read stays
// inside the vector.
template <int BW>
__device__ __forceinline__ uint32_t global_field(const uint32_t* __restrict__ col, uint64_t v, uint32_t lane,
                                                 uint32_t r) {
	if constexpr (BW == 0) {
		return 0u;
	} else {
		const uint32_t* p   = col + v * (32u * BW);
		const uint32_t  bit = r * BW, k = bit >> 5, s = bit & 31u;
		const uint32_t  lo  = __ldg(p + 32u * k + lane);
		if constexpr (BW == 32) {
			return lo;
		} else {
			const uint32_t hi = s + BW > 32u ? __ldg(p + 32u * (k + 1u) + lane) : 0u;
			return __funnelshift_r(lo, hi, s) & ((1u << BW) - 1u);
		}
	}
}

// Filters F0.. and the aggregate, one selected row at a time (warp-uniform
// trip count, branch-free body).
template <class Q, int F0>
__device__ __forceinline__ long long row_loop(const FilterParams& P, const Vec<Q>& V, uint32_t lane, uint32_t mask) {
	const int n_it = max_rows(mask);
	long long acc  = 0;
	for (int it = 0; it < n_it; ++it) {
		const bool     have = mask != 0u;
		const uint32_t r    = have ? static_cast<uint32_t>(__ffs(mask)) - 1u : 0u;
		mask &= mask - 1u;
		const bool pass = have & row_pass<Q, F0>(P, V, lane, r);
		long long  x;
		if constexpr (Q::kAggA < 0) {
			x = 1;
		} else if constexpr (Q::kAggB < 0) {
			x = row_value<Q, Q::kAggA>(P.base, V, lane, r);
		} else {
			x = static_cast<long long>(row_value<Q, Q::kAggA>(P.base, V, lane, r)) *
			    row_value<Q, Q::kAggB>(P.base, V, lane, r);
		}
		acc += pass ? x : 0ll;
	}
	return acc;
}

template <class Q, int F0>
__device__ __forceinline__ long long row_loop_from(const FilterParams& P, const Vec<Q>& V, uint32_t lane,
                                                   uint32_t mask, int f0) {
	if constexpr (F0 <= Q::kNF) {
		if (f0 == F0) { return row_loop<Q, F0>(P, V, lane, mask); }
		return row_loop_from<Q, F0 + 1>(P, V, lane, mask, f0);
	} else {
		return 0;
	}
}

template <class Q>
__device__ __forceinline__ long long dense_agg(const FilterParams& P, const Vec<Q>& V, uint32_t lane, uint32_t mask) {
	if constexpr (Q::kAggA < 0) {
		return __popc(mask);
	} else {
		constexpr int  A  = Q::kAggA;
		long long      p[4] = {0, 0, 0, 0};
		const uint32_t ba   = P.base[A];
		if constexpr (Q::kAggB < 0) {
			dev::unpack_rows<Q::bw(A)>(V.template col<A>(), lane, [&](int r, uint32_t x) {
				p[r & 3] += ((mask >> r) & 1u) ? static_cast<long long>(static_cast<int32_t>(x + ba)) : 0ll;
			});
		} else {
			constexpr int  B  = Q::kAggB;
			const uint32_t bb = P.base[B];
			int32_t        bv[32];
			dev::unpack_rows<Q::bw(B)>(V.template col<B>(), lane, [&](int r, uint32_t x) {
				bv[r] = ((mask >> r) & 1u) ? static_cast<int32_t>(x + bb) : 0;
			});
			dev::unpack_rows<Q::bw(A)>(V.template col<A>(), lane, [&](int r, uint32_t x) {
				p[r & 3] += static_cast<long long>(static_cast<int32_t>(x + ba)) * static_cast<long long>(bv[r]);
			});
		}
		return (p[0] + p[1]) + (p[2] + p[3]);
	}
}

template <class Q>
struct FilterBody {
	static constexpr bool kCtaSetup = false;
	const FilterParams&   P;
	long long             acc = 0;

	__device__ __forceinline__ void cta_setup(uint32_t*) {}

	__device__ __forceinline__ void operator()(const Vec<Q>& V, uint64_t v, uint32_t lane) {
		uint32_t mask = valid_rows(P.S, Q::kLayout, v, lane);
		int      f0   = Q::kNF;
		dense_filters<Q, 0>(P, V, lane, mask, f0);
		if (!__any_sync(0xffffffffu, mask)) { return; }
		if (f0 < Q::kNF) {
			acc += row_loop_from<Q, 0>(P, V, lane, mask, f0);
		} else if (Q::kAggA < 0 || max_rows(mask) > kDenseAggRows) {
			// Every filter ran dense: the aggregate reads the selected rows one
			// at a time unless most rows are selected.
			acc += dense_agg<Q>(P, V, lane, mask);
		} else {
			acc += row_loop<Q, Q::kNF>(P, V, lane, mask);
		}
	}

	__device__ __forceinline__ void finish(uint32_t lane) {
		unsigned long long s = static_cast<unsigned long long>(acc);
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) { s += __shfl_xor_sync(0xffffffffu, s, o); }
		if (lane == 0 && s) { atomicAdd(P.result, s); }
	}
};

// -------------------------------------------------------- probe + group-by

// Signed remainder, kept out of line: it runs only for keys outside the
// table's range, and inlined copies at every row would crowd the
// instruction cache.
__device__ __noinline__ int32_t rem_slow(int32_t x, int32_t n) { return x % n; }

// HASH(X,Y,Z) = (X-Z) % Y (crystal-opt/join.cuh:26) of d = key - keys_min:
// in-range keys skip the division; a negative remainder is flagged and misses.
template <bool DIRECT>
__device__ __forceinline__ bool hash_slot(uint32_t d, int32_t len, uint32_t& h, uint32_t* err) {
	h = d;
	if constexpr (!DIRECT) {
		if (d >= static_cast<uint32_t>(len)) {
			const int32_t m = rem_slow(static_cast<int32_t>(d), len);
			if (m < 0) {
				atomicOr(err, kErrHashBit);
				h = 0;
				return false;
			}
			h = static_cast<uint32_t>(m);
		}
	}
	return true;
}

// One probe's result for a row: hit, and the PHT_2 payload.
template <class Q, int q>
__device__ __forceinline__ uint2 table_entry(const ProbeParams& P, const uint32_t* tables, uint32_t h) {
	if constexpr (Q::pht2(q)) {
		if constexpr (Q::in_smem(q)) { return reinterpret_cast<const uint2*>(tables + P.smem_off[q])[h]; }
		return __ldg(reinterpret_cast<const uint2*>(P.ht[q]) + h);
	} else {
		if constexpr (Q::in_smem(q)) { return make_uint2((tables[P.smem_off[q] + (h >> 5)] >> (h & 31u)) & 1u, 0u); }
		return make_uint2(static_cast<uint32_t>(__ldg(P.ht[q] + h)), 0u);
	}
}

// Whether slot h of probe q's table hits, from the cheapest copy.
template <class Q, int q>
__device__ __forceinline__ bool table_hit(const ProbeParams& P, const uint32_t* tables, uint32_t h) {
	if constexpr (Q::pht2(q) && Q::pbit(q)) {
		return ((tables[P.smem_off[q] + (h >> 5)] >> (h & 31u)) & 1u) != 0u;
	} else {
		const uint2 e = table_entry<Q, q>(P, tables, h);
		return (e.x | e.y) != 0u;
	}
}

// Hit bits of this lane's rows `far` (slot key - keys_min >= len) for probe
// q: the remainder (crystal-opt/join.cuh:26), a negative one flagged and
// missing.  Out of line: such keys are rare.
template <class Q, int q>
__device__ __noinline__ uint32_t far_hits(const ProbeParams& P, const uint32_t* tables, const Vec<Q> V, uint32_t lane,
                                          uint32_t far) {
	const uint32_t kb = P.base[q] - static_cast<uint32_t>(P.kmin[q]);
	uint32_t       hits = 0;
	while (far) {
		const uint32_t r = static_cast<uint32_t>(__ffs(far)) - 1u;
		far &= far - 1u;
		uint32_t h;
		if (hash_slot<false>(row_field<Q::bw(q)>(V.template col<q>(), lane, r) + kb, P.len[q], h, P.S.err) &&
		    table_hit<Q, q>(P, tables, h)) {
			hits |= 1u << r;
		}
	}
	return hits;
}

// Dense probes q, q+1, ... over the whole vector (probes whose hit test reads
// shared memory: PHT_1 bitmaps, PHT_2 tables or their presence bitmaps) while
// some lane keeps more than sparse_rows rows; f0 receives the first probe left
// to the row phase.  At most kMaxDenseProbes: after two selective probes few
// rows are left, and each dense probe adds a fully unrolled unpack to the
// kernel (instruction-cache misses cost more than the rare dense third probe
// would save).
template <class Q, int q>
__device__ __forceinline__ void dense_probes(const ProbeParams& P, const uint32_t* tables, const Vec<Q>& V,
                                             uint32_t lane, uint32_t& mask, int& f0) {
	if constexpr (q < Q::kNP && q < kMaxDenseProbes && Q::dense_ok(q)) {
		if (max_rows(mask) <= P.sparse_rows) {
			f0 = q;
			return;
		}
		const uint32_t kb  = P.base[q] - static_cast<uint32_t>(P.kmin[q]);
		const int32_t  len = P.len[q];
		uint32_t       hit[4] = {0, 0, 0, 0};
		if constexpr (Q::direct(q) && Q::smem_bits(q)) {
			// slot h's bit: word h / 32, shifted right by h mod 32 (the funnel
			// shift takes the amount mod 32), moved to bit r
			const uint32_t* bm = tables + P.smem_off[q];
			unpack_tile_rows<Q, q>(V, lane, [&](int r, uint32_t x) {
				const uint32_t h = Q::field_slot(q) ? x : x + kb;
				hit[r & 3] |= (__funnelshift_r(bm[h >> 5], 0u, h) << r) & (1u << r);
			});
		} else {
			// Keys past the table (slot key - keys_min >= len) take the
			// remainder, rarely: they are collected in `far` and tested after
			// the unrolled rows, out of line, so that the hot loop holds no
			// call of the remainder (32 call sites per probe overflowed the
			// instruction cache on SSB's own data, whose probes are not direct).
			uint32_t far = 0;
			unpack_tile_rows<Q, q>(V, lane, [&](int r, uint32_t x) {
				const uint32_t d = x + kb;
				bool           b;
				if constexpr (Q::direct(q)) {
					b = table_hit<Q, q>(P, tables, d);
				} else {
					const bool in = d < static_cast<uint32_t>(len);
					b             = in && table_hit<Q, q>(P, tables, in ? d : 0u);
					far |= (in ? 0u : 1u) << r;
				}
				hit[r & 3] |= (b ? 1u : 0u) << r;
			});
			if constexpr (!Q::direct(q)) {
				if (far) { hit[0] |= far_hits<Q, q>(P, tables, V, lane, far); }
			}
		}
		mask &= (hit[0] | hit[1]) | (hit[2] | hit[3]);
		dense_probes<Q, q + 1>(P, tables, V, lane, mask, f0);
	} else {
		f0 = q;
	}
}

// Probe q of a batch of selected rows: hit test and group-key payload.
template <class Q, int q>
__device__ __forceinline__ void probe_rows_one(const ProbeParams& P, const uint32_t* tables, const Vec<Q>& V,
                                               const uint32_t (&src)[kRowBatch], const uint32_t (&rows)[kRowBatch],
                                               bool (&pass)[kRowBatch], int32_t (&kv)[FLS_MAX_GROUP_KEYS][kRowBatch],
                                               int rem) {
	const uint32_t kb  = P.base[q] - static_cast<uint32_t>(P.kmin[q]);
	const int32_t  len = P.len[q];
	uint2          e[kRowBatch];
#pragma unroll
	for (int j = 0; j < kRowBatch; ++j) {
		e[j] = make_uint2(0u, 0u);
		if (j < rem) {
			const uint32_t d = row_field<Q::bw(q)>(V.template col<q>(), src[j], rows[j]) + kb;
			uint32_t       h;
			if (pass[j] && hash_slot<Q::direct(q)>(d, len, h, P.S.err)) {
				e[j] = table_entry<Q, q>(P, tables, h);
			}
		}
	}
#pragma unroll
	for (int j = 0; j < kRowBatch; ++j) {
		pass[j] = pass[j] & ((e[j].x | e[j].y) != 0u);
#pragma unroll
		for (int k = 0; k < Q::kNK; ++k) {
			if (Q::key_probe(k) == q) { kv[k][j] = static_cast<int32_t>(e[j].y); }
		}
	}
}

// Probes of a batch of selected rows (row rows[j] of lane src[j]): those
// from f0 on (warp-uniform), and the group-key probes before f0 for their
// payloads (a row selected there hits that table already, so testing it again
// changes nothing).  The table reads of all rows of the batch are issued
// before any is consumed.  One instance serves every f0, which keeps the
// kernel small enough for the instruction cache.
template <class Q, int q>
__device__ __forceinline__ void probe_rows(const ProbeParams& P, const uint32_t* tables, const Vec<Q>& V,
                                           const uint32_t (&src)[kRowBatch], const uint32_t (&rows)[kRowBatch],
                                           bool (&pass)[kRowBatch], int32_t (&kv)[FLS_MAX_GROUP_KEYS][kRowBatch],
                                           int rem, int f0) {
	if constexpr (q < Q::kNP) {
		constexpr bool key = (Q::key_probe(0) == q && Q::kNK > 0) || (Q::key_probe(1) == q && Q::kNK > 1) ||
		                     (Q::key_probe(2) == q && Q::kNK > 2);
		if (key || q >= f0) {
			probe_rows_one<Q, q>(P, tables, V, src, rows, pass, kv, rem);
		}
		probe_rows<Q, q + 1>(P, tables, V, src, rows, pass, kv, rem, f0);
	}
}

// Adds v (an int64 sum, or a measure widened to one) to a group record: the
// int64 at word sum_slot, or its low 32 bits to the wrapping int32 there.
__device__ __forceinline__ void add_record_sum(const ProbeParams& P, int32_t* rec, unsigned long long v) {
	if (P.sum32) {
		atomicAdd(reinterpret_cast<unsigned int*>(rec + P.sum_slot), static_cast<unsigned int>(v));
	} else {
		atomicAdd(reinterpret_cast<unsigned long long*>(rec + P.sum_slot), v);
	}
}

// Group-by epilogue of one selected row (fls_q21.cu:67-77, fls_q31.cu:82-91,
// fls_q41.cu:96-104): the group of the keys in wrapping 32-bit arithmetic,
// the key values into their words of the group record, the measure into its
// int64 sum.  With GSM a group owns slot g & gslot_mask of the CTA's cache
// once it has claimed the slot's tag (its claimer writes the key words);
// rows of a group that lost its slot to another group go to the record as
// without GSM.  A slot sums as two 32-bit words: the low word by atomic add,
// the high word by the measure's sign extension plus the carry out of that
// add (the carry follows from the low word's value just before it, so the
// pair sums modulo 2^64 in any order).
template <class Q>
__device__ __forceinline__ void emit(const ProbeParams& P, uint32_t* tables,
                                     const int32_t (&kv)[FLS_MAX_GROUP_KEYS][kRowBatch], int j, int32_t measure) {
	uint32_t key = 0u - static_cast<uint32_t>(P.sub);
#pragma unroll
	for (int k = 0; k < Q::kNK; ++k) { key += static_cast<uint32_t>(kv[k][j]) * static_cast<uint32_t>(P.key_mul[k]); }
	const int32_t g = key < static_cast<uint32_t>(P.n_groups) ? static_cast<int32_t>(key)
	                                                          : rem_slow(static_cast<int32_t>(key), P.n_groups);
	if (g < 0) {
		atomicOr(P.S.err, kErrHashBit);
		return;
	}
	int32_t* rec = P.res + static_cast<int64_t>(g) * P.stride;
	bool cached = false, claimed = false;
	if constexpr (Q::kGroupSmem) {
		const uint32_t slot = static_cast<uint32_t>(g) & P.gslot_mask;
		uint32_t*      tag  = tables + P.gsum_off + 2u * (P.gslot_mask + 1u) + slot;
		uint32_t       t    = *tag; // a claimed tag never changes
		if (t == kFreeSlot) {
			t       = atomicCAS(tag, kFreeSlot, static_cast<uint32_t>(g));
			claimed = t == kFreeSlot;
		}
		cached = claimed || t == static_cast<uint32_t>(g);
		if (cached) {
			uint32_t*      sum = tables + P.gsum_off + 2u * slot;
			const uint32_t lo  = static_cast<uint32_t>(measure);
			const uint32_t old = atomicAdd(sum, lo);
			const uint32_t hi  = (measure < 0 ? 0xffffffffu : 0u) + (old + lo < old ? 1u : 0u);
			if (hi != 0u) { atomicAdd(sum + 1, hi); }
		}
	}
	if (!cached || claimed) {
#pragma unroll
		for (int k = 0; k < Q::kNK; ++k) {
			if (P.key_slot[k] >= 0) { rec[P.key_slot[k]] = kv[k][j]; }
		}
	}
	if (!cached) { add_record_sum(P, rec, static_cast<unsigned long long>(static_cast<long long>(measure))); }
}

// Value of measure column C for a selected row: from the stage, or (column
// past the staged ones) from global memory.
template <class Q, int C>
__device__ __forceinline__ uint32_t measure_value(const ProbeParams& P, const Vec<Q>& V, uint64_t v, uint32_t lane,
                                                  uint32_t r) {
	if constexpr (C < Q::kNS) {
		return static_cast<uint32_t>(row_value<Q, C>(P.base, V, lane, r));
	} else {
		return global_field<Q::bw(C)>(P.gcol[C - Q::kNS], v, lane, r) + P.base[C];
	}
}

// One batch of selected rows (row rows[j] of lane src[j], slots j < rem):
// the probes left, then each passing row's measure into its group.
template <class Q>
__device__ __forceinline__ void row_batch(const ProbeParams& P, uint32_t* tables, const Vec<Q>& V, uint64_t v,
                                          const uint32_t (&src)[kRowBatch], const uint32_t (&rows)[kRowBatch],
                                          bool (&pass)[kRowBatch], int rem, int f0) {
	int32_t kv[FLS_MAX_GROUP_KEYS][kRowBatch];
#pragma unroll
	for (int j = 0; j < kRowBatch; ++j) {
#pragma unroll
		for (int k = 0; k < FLS_MAX_GROUP_KEYS; ++k) { kv[k][j] = 0; }
	}
	probe_rows<Q, 0>(P, tables, V, src, rows, pass, kv, rem, f0);
	if constexpr (Q::kAgg >= Q::kNS || Q::kSub >= Q::kNS) {
		// measures in global memory: the batch's reads first, all in flight
		uint32_t m[kRowBatch];
#pragma unroll
		for (int j = 0; j < kRowBatch; ++j) {
			m[j] = 0u;
			if (j < rem && pass[j]) {
				m[j] = measure_value<Q, Q::kAgg>(P, V, v, src[j], rows[j]);
				if constexpr (Q::kSub >= 0) { m[j] -= measure_value<Q, Q::kSub>(P, V, v, src[j], rows[j]); }
			}
		}
#pragma unroll
		for (int j = 0; j < kRowBatch; ++j) {
			if (j < rem && pass[j]) { emit<Q>(P, tables, kv, j, static_cast<int32_t>(m[j])); }
		}
	} else {
#pragma unroll
		for (int j = 0; j < kRowBatch; ++j) {
			if (j < rem && pass[j]) {
				uint32_t m = static_cast<uint32_t>(row_value<Q, Q::kAgg>(P.base, V, src[j], rows[j]));
				if constexpr (Q::kSub >= 0) {
					m -= static_cast<uint32_t>(row_value<Q, Q::kSub>(P.base, V, src[j], rows[j]));
				}
				emit<Q>(P, tables, kv, j, static_cast<int32_t>(m));
			}
		}
	}
}

// The rows that passed the dense probes.  Each lane holds its own rows, and
// a warp-uniform loop over them runs as many times as the busiest lane has
// rows.  When the warp's rows are few and unevenly spread, they go to the
// warp's row list first (entry = lane * 32 + row, in lane order) and every
// lane takes the list's entries 32 apart: ceil(rows / 32) slots per lane
// instead of the busiest lane's count.  Any lane may read any lane's fields,
// since the whole tile is staged.
template <class Q>
__device__ __forceinline__ void row_phase(const ProbeParams& P, uint32_t* tables, uint16_t* list, const Vec<Q>& V,
                                          uint64_t v, uint32_t lane, uint32_t mask, int f0) {
	const int n_it = max_rows(mask);
	// A slot without a row reads the tile's first row (its fields are staged).
	const uint32_t idle = Q::kHalf ? 16u * V.h : 0u;
	const uint32_t cnt  = static_cast<uint32_t>(__popc(mask));
	uint32_t       incl = cnt;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= static_cast<uint32_t>(o)) { incl += x; }
	}
	const uint32_t total  = __shfl_sync(0xffffffffu, incl, 31);
	const int      n_comp = static_cast<int>((total + 31u) / 32u);
	if (total <= kRowList && n_comp < n_it) { // warp-uniform
		uint32_t pos = incl - cnt, m = mask;
		for (int it = 0; it < n_it; ++it) {
			if (m != 0u) {
				list[pos++] = static_cast<uint16_t>((lane << 5) | (static_cast<uint32_t>(__ffs(m)) - 1u));
				m &= m - 1u;
			}
		}
		__syncwarp();
		for (int it0 = 0; it0 < n_comp; it0 += kRowBatch) {
			const int rem = n_comp - it0; // warp-uniform
			uint32_t  src[kRowBatch], rows[kRowBatch];
			bool      pass[kRowBatch];
#pragma unroll
			for (int j = 0; j < kRowBatch; ++j) {
				const uint32_t k = static_cast<uint32_t>(it0 + j) * 32u + lane;
				pass[j]          = k < total;
				const uint32_t e = pass[j] ? list[k] : ((lane << 5) | idle);
				src[j]           = e >> 5;
				rows[j]          = e & 31u;
			}
			row_batch<Q>(P, tables, V, v, src, rows, pass, rem, f0);
		}
		__syncwarp(); // the list is read before the next tile writes it
		return;
	}
	for (int it0 = 0; it0 < n_it; it0 += kRowBatch) {
		const int rem = n_it - it0; // warp-uniform
		uint32_t  src[kRowBatch], rows[kRowBatch];
		bool      pass[kRowBatch];
#pragma unroll
		for (int j = 0; j < kRowBatch; ++j) {
			src[j]  = lane;
			pass[j] = mask != 0u;
			rows[j] = pass[j] ? static_cast<uint32_t>(__ffs(mask)) - 1u : idle;
			mask &= mask - 1u;
		}
		row_batch<Q>(P, tables, V, v, src, rows, pass, rem, f0);
	}
}

template <class Q>
struct ProbeBody {
	static constexpr bool kCtaSetup = true;
	const ProbeParams&    P;
	uint32_t*             tables = nullptr;
	uint16_t*             list   = nullptr; // this warp's row list

	// Shared-memory tables, staged once per CTA by all its threads: presence
	// bitmaps (of PHT_1 tables, whose probe only tests slot != 0, crystal-opt/
	// join.cuh:42-47, and of PHT_2 tables too large to stage, whose slot hits
	// when its 64-bit entry is not zero) copied from P.bits when a prepass
	// built them there at the same offsets, else built here from the tables;
	// small PHT_2 tables verbatim.  GSM: every slot of the group-sum cache
	// starts free.
	__device__ void cta_setup(uint32_t* cta) {
		extern __shared__ __align__(128) uint32_t smem[];
		tables = cta;
		list   = reinterpret_cast<uint16_t*>(smem + (threadIdx.x >> 5) * P.S.warp_smem_words + P.S.list_off);
#pragma unroll 1
		for (int q = 0; q < Q::kNP; ++q) {
			if (!Q::in_smem(q) && !Q::pbit(q)) { continue; }
			const uint32_t len = static_cast<uint32_t>(P.len[q]);
			if ((!Q::pht2(q) || Q::pbit(q)) && P.bits == nullptr) {
				// No prebuilt bitmaps: one ballot per 32 slots, 8 words per warp
				// in flight.
				const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
				const uint32_t n_words = (len + 31u) / 32u;
				uint32_t*      dst     = cta + P.smem_off[q];
				for (uint32_t w0 = warp * 8u; w0 < n_words; w0 += nw * 8u) {
					int32_t x[8];
#pragma unroll
					for (uint32_t j = 0; j < 8; ++j) {
						const uint32_t idx = 32u * (w0 + j) + lane;
						x[j]               = 0;
						if (w0 + j < n_words && idx < len) {
							if (Q::pht2(q)) {
								const int2 e = __ldg(reinterpret_cast<const int2*>(P.ht[q]) + idx);
								x[j]         = e.x | e.y;
							} else {
								x[j] = __ldg(P.ht[q] + idx);
							}
						}
					}
#pragma unroll
					for (uint32_t j = 0; j < 8; ++j) {
						const uint32_t b = __ballot_sync(0xffffffffu, x[j] != 0);
						if (lane == 0 && w0 + j < n_words) { dst[w0 + j] = b; }
					}
				}
			} else if (!Q::pht2(q) || Q::pbit(q)) {
				// 16-byte units: offsets and slot sizes are multiples of 4 words.
				const uint32_t n4  = ((len + 31u) / 32u + 3u) / 4u;
				const uint4*   src = reinterpret_cast<const uint4*>(P.bits + P.smem_off[q]);
				uint4*         dst = reinterpret_cast<uint4*>(cta + P.smem_off[q]);
				for (uint32_t i0 = threadIdx.x; i0 < n4; i0 += 4u * blockDim.x) {
					uint4 x[4];
#pragma unroll
					for (uint32_t j = 0; j < 4; ++j) {
						const uint32_t i = i0 + j * blockDim.x;
						x[j]             = i < n4 ? __ldg(src + i) : make_uint4(0u, 0u, 0u, 0u);
					}
#pragma unroll
					for (uint32_t j = 0; j < 4; ++j) {
						const uint32_t i = i0 + j * blockDim.x;
						if (i < n4) { dst[i] = x[j]; }
					}
				}
			} else {
				uint32_t*      dst = cta + P.smem_off[q];
				const int32_t* ht  = P.ht[q];
				const uint32_t n   = 2u * len;
				for (uint32_t i0 = threadIdx.x; i0 < n; i0 += 4u * blockDim.x) {
					int32_t x[4];
#pragma unroll
					for (uint32_t j = 0; j < 4; ++j) {
						const uint32_t idx = i0 + j * blockDim.x;
						x[j]               = idx < n ? __ldg(ht + idx) : 0;
					}
#pragma unroll
					for (uint32_t j = 0; j < 4; ++j) {
						const uint32_t idx = i0 + j * blockDim.x;
						if (idx < n) { dst[idx] = static_cast<uint32_t>(x[j]); }
					}
				}
			}
		}
		if constexpr (Q::kGroupSmem) {
			const uint32_t slots = P.gslot_mask + 1u;
			for (uint32_t i = threadIdx.x; i < 3u * slots; i += blockDim.x) {
				cta[P.gsum_off + i] = i < 2u * slots ? 0u : kFreeSlot;
			}
		}
	}

	__device__ __forceinline__ void operator()(const Vec<Q>& V, uint64_t v, uint32_t lane) {
		uint32_t mask = valid_rows(P.S, Q::kLayout, v, lane);
		if constexpr (Q::kHalf) { mask &= V.h ? 0xffff0000u : 0x0000ffffu; }
		int      f0   = Q::kNP;
		dense_probes<Q, 0>(P, tables, V, lane, mask, f0);
		if (!__any_sync(0xffffffffu, mask)) { return; }
		row_phase<Q>(P, tables, list, V, v, lane, mask, f0);
	}

	// GSM: once every warp of the CTA is done, the CTA adds each claimed
	// slot's non-zero sum to its group's record.
	__device__ __forceinline__ void finish(uint32_t) {
		if constexpr (Q::kGroupSmem) {
			__syncthreads();
			const uint32_t  slots = P.gslot_mask + 1u;
			const uint32_t* sum   = tables + P.gsum_off;
			const uint32_t* tag   = sum + 2u * slots;
			for (uint32_t i = threadIdx.x; i < slots; i += blockDim.x) {
				const uint32_t           g = tag[i];
				const unsigned long long v =
				    static_cast<unsigned long long>(sum[2u * i]) | (static_cast<unsigned long long>(sum[2u * i + 1u]) << 32);
				if (g != kFreeSlot && v != 0ull) { add_record_sum(P, P.res + static_cast<int64_t>(g) * P.stride, v); }
			}
		}
	}
};

// ------------------------------------------------------------------ decode

template <class Q>
struct DecodeBody {
	static constexpr bool kCtaSetup = false;
	const DecodeParams&   P;
	unsigned long long    acc = 0;

	__device__ __forceinline__ void cta_setup(uint32_t*) {}

	__device__ __forceinline__ void operator()(const Vec<Q>& V, uint64_t v, uint32_t lane) {
		constexpr int  BW   = Q::bw(0);
		const uint32_t base = P.base;
		if constexpr (Q::kMode == 1) {
			uint32_t* dst = P.out + v * 1024u + lane;
			dev::unpack_rows<BW>(V.template col<0>(), lane, [&](int r, uint32_t x) { __stcs(dst + 32 * r, x + base); });
		} else {
			const uint32_t m = valid_rows(P.S, Q::kLayout, v, lane);
			if constexpr (Q::kNoWrap && BW <= 27) {
				// 32 values of at most 27 bits: the lane's sum fits 32 bits.
				uint32_t s = 0;
				if (m == 0xffffffffu) {
					dev::unpack_rows<BW>(V.template col<0>(), lane, [&](int, uint32_t x) { s += x; });
				} else {
					dev::unpack_rows<BW>(V.template col<0>(), lane,
					                     [&](int r, uint32_t x) { s += ((m >> r) & 1u) ? x : 0u; });
				}
				acc += static_cast<unsigned long long>(s) +
				       static_cast<unsigned long long>(__popc(m)) * static_cast<unsigned long long>(base);
			} else {
				unsigned long long p[4] = {0, 0, 0, 0};
				dev::unpack_rows<BW>(V.template col<0>(), lane, [&](int r, uint32_t x) {
					p[r & 3] += ((m >> r) & 1u) ? static_cast<unsigned long long>(x + base) : 0ull;
				});
				acc += (p[0] + p[1]) + (p[2] + p[3]);
			}
		}
	}

	__device__ __forceinline__ void finish(uint32_t lane) {
		if constexpr (Q::kMode == 0) {
			unsigned long long s = acc;
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) { s += __shfl_xor_sync(0xffffffffu, s, o); }
			if (lane == 0 && s) { atomicAdd(P.sum, s); }
		}
	}
};

// ---------------------------------------------------------------- pipeline

// Words per vector and stage offset (in vectors' words) of column `lane`.
template <class Q, int C>
__device__ __forceinline__ void lane_column(uint32_t lane, uint32_t& vw, uint32_t& pre) {
	if constexpr (C < Q::kNS) {
		constexpr uint32_t w = Q::vec_words(C), p = Q::prefix(C);
		if (lane == C) {
			vw  = w;
			pre = p;
		}
		lane_column<Q, C + 1>(lane, vw, pre);
	}
}

// Word rows of column `lane` in a half-vector tile: its words, its stage
// offset, the words it skips in half 1, and its words per vector.
template <class Q, int C>
__device__ __forceinline__ void lane_half_column(uint32_t lane, uint32_t& hw, uint32_t& pre, uint32_t& skip,
                                                 uint32_t& vw) {
	if constexpr (C < Q::kNS) {
		if (lane == C) {
			hw   = Q::half_words(C);
			pre  = Q::half_prefix(C);
			skip = Q::half_skip(C);
			vw   = Q::vec_words(C);
		}
		lane_half_column<Q, C + 1>(lane, hw, pre, skip, vw);
	}
}

// Issue tile t into a stage: lane c copies column c (k vectors, contiguous;
// or, for half-vector tiles, the word rows of half t mod 2 of vector t / 2).
template <class Q>
__device__ __forceinline__ void issue(const StageParams& S, uint32_t* stage, uint64_t* bar, uint64_t t, uint32_t lane,
                                      uint64_t pol) {
	if constexpr (Q::kHalf) {
		if (lane < static_cast<uint32_t>(Q::kNS)) {
			uint32_t hw = 0, pre = 0, skip = 0, vw = 0;
			lane_half_column<Q, 0>(lane, hw, pre, skip, vw);
			const uint64_t v = t >> 1;
			if (hw) {
				dev::mbar_expect_tx(bar, 4u * hw);
				dev::bulk_g2s(stage + pre, S.data[lane] + v * vw + ((t & 1u) ? skip : 0u), 4u * hw, bar, pol);
			}
		}
		__syncwarp();
		if (lane == 0) { dev::mbar_arrive(bar); }
		__syncwarp();
		return;
	}
	const uint64_t v0 = t * S.tile;
	const uint64_t kk = S.n_vec - v0 < S.tile ? S.n_vec - v0 : S.tile;
	if (lane < static_cast<uint32_t>(Q::kNS)) {
		uint32_t vw = 0, pre = 0;
		lane_column<Q, 0>(lane, vw, pre);
		const uint32_t bytes = static_cast<uint32_t>(kk) * vw * 4u;
		if (bytes) {
			dev::mbar_expect_tx(bar, bytes);
			dev::bulk_g2s(stage + S.tile * pre, S.data[lane] + v0 * vw, bytes, bar, pol);
		}
	}
	__syncwarp();
	if (lane == 0) { dev::mbar_arrive(bar); }
	__syncwarp();
}

// Persistent loop: each warp stages its tiles (tile t = first + j*total) into
// its own ring of S stages and hands every vector to body(V, v, lane).
template <class Q, class Body>
__device__ __forceinline__ void run(const StageParams& S, Body& body) {
	extern __shared__ __align__(128) uint32_t smem[];
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	uint32_t*      base = smem + warp * S.warp_smem_words;
	uint64_t*      bars = reinterpret_cast<uint64_t*>(base + S.bar_off);
	if (lane == 0) {
		for (uint32_t s = 0; s < S.stages; ++s) { dev::mbar_init(bars + s, 1); }
		dev::fence_mbar_init();
	}
	__syncwarp();
	const uint64_t pol   = dev::l2_evict_first_policy();
	const uint64_t total = static_cast<uint64_t>(gridDim.x) * S.warps;
	const uint64_t first = static_cast<uint64_t>(blockIdx.x) * S.warps + warp;
	for (uint32_t s = 0; s < S.stages; ++s) {
		const uint64_t t = first + s * total;
		if (t >= S.n_tiles) { break; }
		issue<Q>(S, base + s * S.stage_words, bars + s, t, lane, pol);
	}
	if constexpr (Body::kCtaSetup) {
		body.cta_setup(smem + S.cta_off); // overlaps the first stages' copies
		__syncthreads();
	}
	uint64_t next = first + static_cast<uint64_t>(S.stages) * total;
	uint32_t st = 0, phase = 0;
	for (uint64_t t = first; t < S.n_tiles; t += total) {
		if (!dev::mbar_wait_bounded(bars + st, phase, kWaitPolls)) {
			// Copies that did not land: flag, drain (bounded) and leave the
			// loop; finish() still runs so that CTA-wide barriers there see
			// every warp.
			atomicOr(S.err, kErrTimeoutBit);
			for (uint32_t s = 0; s < S.stages; ++s) {
				dev::mbar_wait_bounded(bars + s, phase, 1u << 10);
				dev::mbar_wait_bounded(bars + s, phase ^ 1u, 1u << 10);
			}
			break;
		}
		if constexpr (Q::kHalf) {
			body(Vec<Q> {base + st * S.stage_words, 1u, 0u, static_cast<uint32_t>(t & 1u)}, t >> 1, lane);
		} else {
			const uint64_t v0 = t * S.tile;
			const uint32_t kk = static_cast<uint32_t>(S.n_vec - v0 < S.tile ? S.n_vec - v0 : S.tile);
			for (uint32_t i = 0; i < kk; ++i) { body(Vec<Q> {base + st * S.stage_words, S.tile, i, 0u}, v0 + i, lane); }
		}
		__syncwarp();
		if (next < S.n_tiles) {
			dev::fence_proxy_async_smem();
			issue<Q>(S, base + st * S.stage_words, bars + st, next, lane, pol);
			next += total;
		}
		if (++st == S.stages) {
			st    = 0;
			phase ^= 1u;
		}
	}
	body.finish(lane);
}

template <class Q>
__device__ __forceinline__ void filter_kernel(const FilterParams& P) {
	FilterBody<Q> body {P};
	run<Q>(P.S, body);
}

template <class Q>
__device__ __forceinline__ void probe_kernel(const ProbeParams& P) {
	ProbeBody<Q> body {P};
	run<Q>(P.S, body);
}

template <class Q>
__device__ __forceinline__ void decode_kernel(const DecodeParams& P) {
	DecodeBody<Q> body {P};
	run<Q>(P.S, body);
}

} // namespace fixed
} // namespace fls
