// fls_fixed.cuh -- filter-aggregate kernel specialised to one query shape.
//
// For queries whose columns are all uniform FOR columns (the reference's
// column format: one bit width and base per column, fls_q11.cu:202-223), the
// library compiles this template at first use with NVRTC for the exact shape
// (bit width of every column, number of filters, aggregate kind) and caches
// the kernel (fls_jit.cu).  Everything that the generic operator decides per
// vector at run time -- which decoder, how many filters, where the aggregate
// columns are, which filters remain in the row-at-a-time loop -- becomes a
// compile-time constant here.  Results are identical to the generic operator.
//
// Columns are staged in filter order (column f holds filter f), followed by
// aggregate columns that are not filter columns; Query's template arguments
// name the aggregate columns by staged index (-1 = none).
#pragma once

#include "fls_device.cuh"

namespace fls {
namespace fixed {

constexpr uint32_t kSlack     = 32;       // words after the stages (row reads look one word row ahead)
constexpr uint32_t kWaitPolls = 1u << 17; // bounded stage waits (each <= ~20 us)
constexpr uint32_t kErrTimeoutBit = 1u << 2;
constexpr int      kDenseAggRows  = 16;      // above this many rows in some lane, aggregate whole vectors

struct FixedParams {
	const uint32_t*     data[FLS_MAX_QUERY_COLS];
	uint32_t            base[FLS_MAX_QUERY_COLS]; // FOR base of each staged column
	uint32_t            lo[FLS_MAX_FILTERS];      // filter lower bound (unsigned wrap)
	uint32_t            range[FLS_MAX_FILTERS];   // hi - lo
	uint64_t            n_values, n_vec, n_tiles;
	uint32_t            tile, stages, warps, warp_smem_words, stage_words, bar_off;
	int32_t             sparse_rows;
	uint32_t            pad_;
	unsigned long long* result;
	uint32_t*           err;
};

// The host (nvcc + host compiler) and NVRTC must agree on the parameter block.
// Every field is naturally aligned and padded explicitly, so equal sizes mean
// equal offsets.
static_assert(sizeof(FixedParams) == 200 && alignof(FixedParams) == 8, "FixedParams layout");

template <int LAYOUT, int NF, int AGG_A, int AGG_B, int... BWS>
struct Query {
	static constexpr int NC     = sizeof...(BWS);
	static constexpr int kNF    = NF;
	static constexpr int kAggA  = AGG_A;
	static constexpr int kAggB  = AGG_B;
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
	static_assert(NF >= 0 && NF <= FLS_MAX_FILTERS && NC <= FLS_MAX_QUERY_COLS, "query shape");
	static_assert(AGG_B < 0 || AGG_A >= 0, "sum(a*b) needs a");
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

// Where the columns of tile vector i sit in the stage.
template <class Q>
struct Vec {
	const uint32_t* stage;
	uint32_t        k, i;
	template <int C>
	__device__ __forceinline__ const uint32_t* col() const {
		constexpr uint32_t pre = Q::prefix(C), vw = Q::vec_words(C);
		return stage + k * pre + i * vw;
	}
};

template <class Q, int F>
__device__ __forceinline__ void dense_filter(const FixedParams& P, const Vec<Q>& V, uint32_t lane, uint32_t& mask) {
	const uint32_t lo = P.lo[F] - P.base[F], range = P.range[F];
	uint32_t       m[4] = {0, 0, 0, 0};
	dev::unpack_rows<Q::bw(F)>(V.template col<F>(), lane,
	                           [&](int r, uint32_t p) { m[r & 3] |= (p - lo <= range ? 1u : 0u) << r; });
	mask &= (m[0] | m[1]) | (m[2] | m[3]);
}

// Dense filters F, F+1, ... while some lane keeps more than sparse_rows rows;
// f0 receives the first filter left to the row loop (NF if none).
template <class Q, int F>
__device__ __forceinline__ void dense_filters(const FixedParams& P, const Vec<Q>& V, uint32_t lane, uint32_t& mask,
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

template <class Q, int F, int F0>
__device__ __forceinline__ bool row_pass(const FixedParams& P, const Vec<Q>& V, uint32_t lane, uint32_t r) {
	if constexpr (F < Q::kNF) {
		const bool ok = (row_field<Q::bw(F)>(V.template col<F>(), lane, r) - (P.lo[F] - P.base[F])) <= P.range[F];
		return ok & row_pass<Q, F + 1, F0>(P, V, lane, r);
	} else {
		return true;
	}
}

template <class Q, int C>
__device__ __forceinline__ long long row_value(const FixedParams& P, const Vec<Q>& V, uint32_t lane, uint32_t r) {
	return static_cast<int32_t>(row_field<Q::bw(C)>(V.template col<C>(), lane, r) + P.base[C]);
}

// Filters F0.. and the aggregate, one selected row at a time (warp-uniform
// trip count, branch-free body).
template <class Q, int F0>
__device__ __forceinline__ long long row_loop(const FixedParams& P, const Vec<Q>& V, uint32_t lane, uint32_t mask) {
	const int n_it = max_rows(mask);
	long long acc  = 0;
	for (int it = 0; it < n_it; ++it) {
		const bool     have = mask != 0u;
		const uint32_t r    = have ? static_cast<uint32_t>(__ffs(mask)) - 1u : 0u;
		mask &= mask - 1u;
		const bool pass = have & row_pass<Q, F0, F0>(P, V, lane, r);
		long long  x;
		if constexpr (Q::kAggA < 0) {
			x = 1;
		} else if constexpr (Q::kAggB < 0) {
			x = row_value<Q, Q::kAggA>(P, V, lane, r);
		} else {
			x = row_value<Q, Q::kAggA>(P, V, lane, r) * row_value<Q, Q::kAggB>(P, V, lane, r);
		}
		acc += pass ? x : 0ll;
	}
	return acc;
}

template <class Q, int F0>
__device__ __forceinline__ long long row_loop_from(const FixedParams& P, const Vec<Q>& V, uint32_t lane,
                                                   uint32_t mask, int f0) {
	if constexpr (F0 <= Q::kNF) {
		if (f0 == F0) { return row_loop<Q, F0>(P, V, lane, mask); }
		return row_loop_from<Q, F0 + 1>(P, V, lane, mask, f0);
	} else {
		return 0;
	}
}

template <class Q>
__device__ __forceinline__ long long dense_agg(const FixedParams& P, const Vec<Q>& V, uint32_t lane, uint32_t mask) {
	if constexpr (Q::kAggA < 0) {
		return __popc(mask);
	} else {
		constexpr int A = Q::kAggA;
		long long     p[4] = {0, 0, 0, 0};
		const uint32_t ba = P.base[A];
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
__device__ __forceinline__ long long process(const FixedParams& P, const Vec<Q>& V, uint64_t v, uint32_t lane) {
	uint32_t       mask  = 0xffffffffu;
	const uint64_t start = v * 1024u;
	if (start + 1024u > P.n_values) { mask = dev::tail_rows(Q::kLayout, lane, static_cast<uint32_t>(P.n_values - start)); }
	int f0 = Q::kNF;
	dense_filters<Q, 0>(P, V, lane, mask, f0);
	if (!__any_sync(0xffffffffu, mask)) { return 0; }
	if (f0 < Q::kNF) { return row_loop_from<Q, 0>(P, V, lane, mask, f0); }
	// Every filter ran dense: the aggregate reads the selected rows one at a
	// time unless most rows are selected.
	if (Q::kAggA < 0 || max_rows(mask) > kDenseAggRows) { return dense_agg<Q>(P, V, lane, mask); }
	return row_loop<Q, Q::kNF>(P, V, lane, mask);
}

// Words per vector and stage offset (in vectors' words) of column `lane`.
template <class Q, int C>
__device__ __forceinline__ void lane_column(uint32_t lane, uint32_t& vw, uint32_t& pre) {
	if constexpr (C < Q::NC) {
		constexpr uint32_t w = Q::vec_words(C), p = Q::prefix(C);
		if (lane == C) {
			vw  = w;
			pre = p;
		}
		lane_column<Q, C + 1>(lane, vw, pre);
	}
}

// Issue tile t into stage st: lane c copies column c (k vectors, contiguous).
template <class Q>
__device__ __forceinline__ void issue(const FixedParams& P, uint32_t* stage, uint64_t* bar, uint64_t t, uint32_t lane,
                                      uint64_t pol) {
	const uint64_t v0 = t * P.tile;
	const uint64_t kk = P.n_vec - v0 < P.tile ? P.n_vec - v0 : P.tile;
	if (lane < static_cast<uint32_t>(Q::NC)) {
		uint32_t vw = 0, pre = 0;
		lane_column<Q, 0>(lane, vw, pre);
		const uint32_t bytes = static_cast<uint32_t>(kk) * vw * 4u;
		if (bytes) {
			dev::mbar_expect_tx(bar, bytes);
			dev::bulk_g2s(stage + P.tile * pre, P.data[lane] + v0 * vw, bytes, bar, pol);
		}
	}
	__syncwarp();
	if (lane == 0) { dev::mbar_arrive(bar); }
	__syncwarp();
}

template <class Q>
__device__ __forceinline__ void run(const FixedParams& P) {
	extern __shared__ __align__(128) uint32_t smem[];
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	uint32_t*      base = smem + warp * P.warp_smem_words;
	uint64_t*      bars = reinterpret_cast<uint64_t*>(base + P.bar_off);
	if (lane == 0) {
		for (uint32_t s = 0; s < P.stages; ++s) { dev::mbar_init(bars + s, 1); }
		dev::fence_mbar_init();
	}
	__syncwarp();
	const uint64_t pol   = dev::l2_evict_first_policy();
	const uint64_t total = static_cast<uint64_t>(gridDim.x) * P.warps;
	const uint64_t first = static_cast<uint64_t>(blockIdx.x) * P.warps + warp;
	for (uint32_t s = 0; s < P.stages; ++s) {
		const uint64_t t = first + s * total;
		if (t >= P.n_tiles) { break; }
		issue<Q>(P, base + s * P.stage_words, bars + s, t, lane, pol);
	}
	uint64_t  next  = first + static_cast<uint64_t>(P.stages) * total;
	uint32_t  st = 0, phase = 0;
	long long acc = 0;
	for (uint64_t t = first; t < P.n_tiles; t += total) {
		if (!dev::mbar_wait_bounded(bars + st, phase, kWaitPolls)) {
			atomicOr(P.err, kErrTimeoutBit);
			for (uint32_t s = 0; s < P.stages; ++s) {
				dev::mbar_wait_bounded(bars + s, phase, 1u << 10);
				dev::mbar_wait_bounded(bars + s, phase ^ 1u, 1u << 10);
			}
			return;
		}
		const uint64_t v0 = t * P.tile;
		const uint32_t kk = static_cast<uint32_t>(P.n_vec - v0 < P.tile ? P.n_vec - v0 : P.tile);
		for (uint32_t i = 0; i < kk; ++i) {
			const Vec<Q> V {base + st * P.stage_words, P.tile, i};
			acc += process<Q>(P, V, v0 + i, lane);
		}
		__syncwarp();
		if (next < P.n_tiles) {
			dev::fence_proxy_async_smem();
			issue<Q>(P, base + st * P.stage_words, bars + st, next, lane, pol);
			next += total;
		}
		if (++st == P.stages) {
			st = 0;
			phase ^= 1u;
		}
	}
	unsigned long long s = static_cast<unsigned long long>(acc);
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) { s += __shfl_xor_sync(0xffffffffu, s, o); }
	if (lane == 0 && s) { atomicAdd(P.result, s); }
}

} // namespace fixed
} // namespace fls
