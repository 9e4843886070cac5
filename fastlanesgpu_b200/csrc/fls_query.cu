// fls_query.cu -- fused decode + query operators: filter-aggregate, selective
// perfect-hash build, and decode + multi-probe + int64 group-by.
//
// Reference counterparts: QueryKernel_v1/_v2 (fastlanes/src/ssb/fls_q11.cu:29-135),
// build_hashtable_{s,p,d} and probe_v1..v3 (fls_q21.cu:21-263), with the tile
// primitives of fastlanes/src/include/crystal-opt/{pred,load,reduce,join}.cuh.
#include <algorithm>
#include <cmath>
#include <utility>

#include "fls_pipeline.cuh"

namespace fls {
namespace {

struct AccState {
	unsigned long long acc;
};

__device__ __forceinline__ int max_rows(uint32_t mask) { return __reduce_max_sync(0xffffffffu, __popc(mask)); }

__device__ __forceinline__ bool in_range(uint32_t x, uint32_t lo, uint32_t range) { return x - lo <= range; }

// Range filters ANDed into a per-lane row mask (bit r = row r), then sum(a),
// sum(a*b) or count over the selected rows, in int64.
struct FilterAggOp {
	using State = AccState;
	uint32_t   n_filters;
	uint32_t   f_col[FLS_MAX_FILTERS];
	uint32_t   f_lo[FLS_MAX_FILTERS];
	uint32_t   f_range[FLS_MAX_FILTERS]; // hi - lo (unsigned)
	int32_t    agg_a, agg_b;
	long long* result;
	// Above this many selected rows in some lane, whole vectors are evaluated
	// (dense); at or below it a loop over the set bits of the row mask reads
	// only the selected rows' fields (FLS_TUNE_SPARSE_ROWS).
	int32_t sparse_rows;

	__device__ void cta_setup(State&, uint32_t*, const StageCfg&) const {}

	// Dense pass of filter f: whole vector, FOR base folded into the bound.
	__device__ bool dense_filter(uint32_t f, uint32_t& mask, const WarpStage& ws, uint32_t st, uint32_t i,
	                             uint32_t lane) const {
		const StagedVec sv = staged(ws, st, i, f_col[f]);
		if (sv.bad()) { return false; }
		const uint32_t lo = f_lo[f] - dev::value_offset(sv.vi), range = f_range[f];
		uint32_t       m[4] = {0, 0, 0, 0};
		dev::decode_each<false>(sv.s, sv.vi, ws.dict(), lane,
		                        [&](int r, uint32_t x) { m[r & 3] |= (in_range(x, lo, range) ? 1u : 0u) << r; });
		mask &= (m[0] | m[1]) | (m[2] | m[3]);
		return true;
	}

	__device__ void process(State& S, uint64_t v, const WarpStage& ws, uint32_t st, uint32_t i, uint32_t lane,
	                        const StageCfg& cfg) const {
		uint32_t mask = valid_rows(cfg, v, lane);
		uint32_t f    = 0;
		for (; f < n_filters; ++f) {
			if (max_rows(mask) <= sparse_rows) { break; }
			if (!dense_filter(f, mask, ws, st, i, lane)) { return; }
		}
		if (!__any_sync(0xffffffffu, mask)) { return; }
		// Can the rest be read row by row?
		bool rnd = true;
		for (uint32_t g = f; g < n_filters; ++g) { rnd = rnd && dev::random_access(staged(ws, st, i, f_col[g]).vi.scheme); }
		if (agg_a >= 0) { rnd = rnd && dev::random_access(staged(ws, st, i, static_cast<uint32_t>(agg_a)).vi.scheme); }
		if (agg_b >= 0) { rnd = rnd && dev::random_access(staged(ws, st, i, static_cast<uint32_t>(agg_b)).vi.scheme); }
		if (rnd) {
			S.acc += all_for(f, ws, st, i) ? sparse_rest_for(f, mask, ws, st, i, lane)
			                                : sparse_rest(f, mask, ws, st, i, lane);
			return;
		}
		for (; f < n_filters; ++f) {
			if (!dense_filter(f, mask, ws, st, i, lane)) { return; }
			if (!__any_sync(0xffffffffu, mask)) { return; }
		}
		S.acc += dense_agg(mask, ws, st, i, lane);
	}

	__device__ bool all_for(uint32_t f0, const WarpStage& ws, uint32_t st, uint32_t i) const {
		bool ok = true;
		for (uint32_t f = f0; f < n_filters; ++f) { ok = ok && staged(ws, st, i, f_col[f]).vi.scheme == FLS_SCHEME_FOR; }
		if (agg_a >= 0) { ok = ok && staged(ws, st, i, static_cast<uint32_t>(agg_a)).vi.scheme == FLS_SCHEME_FOR; }
		if (agg_b >= 0) { ok = ok && staged(ws, st, i, static_cast<uint32_t>(agg_b)).vi.scheme == FLS_SCHEME_FOR; }
		return ok;
	}

	// Row-at-a-time rest when every remaining column is FOR: per field two
	// shared-memory loads, a funnel shift, a mask and the base.
	__device__ unsigned long long sparse_rest_for(uint32_t f0, uint32_t mask, const WarpStage& ws, uint32_t st,
	                                              uint32_t i, uint32_t lane) const {
		dev::ForRows fr[FLS_MAX_FILTERS];
		uint32_t     lo[FLS_MAX_FILTERS], range[FLS_MAX_FILTERS];
#pragma unroll
		for (uint32_t f = 0; f < FLS_MAX_FILTERS; ++f) {
			if (f >= f0 && f < n_filters) {
				const StagedVec sv = staged(ws, st, i, f_col[f]);
				fr[f].init(sv.s, sv.vi, lane);
				// fold the base into the bound: x + base - lo = x - (lo - base)
				lo[f]        = f_lo[f] - fr[f].base;
				range[f]     = f_range[f];
				fr[f].base   = 0;
			}
		}
		dev::ForRows ra {}, rb {};
		if (agg_a >= 0) {
			const StagedVec sv = staged(ws, st, i, static_cast<uint32_t>(agg_a));
			ra.init(sv.s, sv.vi, lane);
		}
		if (agg_b >= 0) {
			const StagedVec sv = staged(ws, st, i, static_cast<uint32_t>(agg_b));
			rb.init(sv.s, sv.vi, lane);
		}
		// Warp-uniform trip count (the largest per-lane row count); the body is
		// branch-free: lanes without a row left read row 0 and discard it.
		const int n_it = max_rows(mask);
		long long acc  = 0;
		for (int it = 0; it < n_it; ++it) {
			const bool     have = mask != 0u;
			const uint32_t r    = have ? static_cast<uint32_t>(__ffs(mask)) - 1u : 0u;
			mask &= mask - 1u;
			bool pass = have;
#pragma unroll
			for (uint32_t f = 0; f < FLS_MAX_FILTERS; ++f) {
				if (f >= f0 && f < n_filters) { pass &= in_range(fr[f].get(r), lo[f], range[f]); }
			}
			long long x;
			if (agg_a < 0) {
				x = 1;
			} else if (agg_b >= 0) {
				x = static_cast<long long>(static_cast<int32_t>(ra.get(r))) *
				    static_cast<long long>(static_cast<int32_t>(rb.get(r)));
			} else {
				x = static_cast<int32_t>(ra.get(r));
			}
			acc += pass ? x : 0ll;
		}
		return static_cast<unsigned long long>(acc);
	}

	// Remaining filters and the aggregate, one selected row at a time.  The
	// staged-vector descriptors are read once; the row loop only extracts.
	__device__ unsigned long long sparse_rest(uint32_t f0, uint32_t mask, const WarpStage& ws, uint32_t st,
	                                          uint32_t i, uint32_t lane) const {
		StagedVec fv[FLS_MAX_FILTERS];
#pragma unroll
		for (uint32_t f = 0; f < FLS_MAX_FILTERS; ++f) {
			if (f >= f0 && f < n_filters) {
				fv[f] = staged(ws, st, i, f_col[f]);
				if (fv[f].bad()) { return 0; }
			}
		}
		StagedVec sa {}, sb {};
		if (agg_a >= 0) {
			sa = staged(ws, st, i, static_cast<uint32_t>(agg_a));
			if (sa.bad()) { return 0; }
		}
		if (agg_b >= 0) {
			sb = staged(ws, st, i, static_cast<uint32_t>(agg_b));
			if (sb.bad()) { return 0; }
		}
		long long acc = 0;
		while (mask) {
			const uint32_t r = static_cast<uint32_t>(__ffs(mask)) - 1u;
			mask &= mask - 1u;
			bool pass = true;
#pragma unroll
			for (uint32_t f = 0; f < FLS_MAX_FILTERS; ++f) {
				if (pass && f >= f0 && f < n_filters) {
					pass = in_range(dev::value_at(fv[f].s, fv[f].vi, lane, r), f_lo[f], f_range[f]);
				}
			}
			if (!pass) { continue; }
			if (agg_a < 0) {
				acc += 1;
			} else if (agg_b >= 0) {
				acc += static_cast<long long>(static_cast<int32_t>(dev::value_at(sa.s, sa.vi, lane, r))) *
				       static_cast<long long>(static_cast<int32_t>(dev::value_at(sb.s, sb.vi, lane, r)));
			} else {
				acc += static_cast<int32_t>(dev::value_at(sa.s, sa.vi, lane, r));
			}
		}
		return static_cast<unsigned long long>(acc);
	}

	__device__ unsigned long long dense_agg(uint32_t mask, const WarpStage& ws, uint32_t st, uint32_t i,
	                                        uint32_t lane) const {
		if (agg_a < 0) { return static_cast<unsigned long long>(__popc(mask)); }
		long long       p[4] = {0, 0, 0, 0};
		const StagedVec sa   = staged(ws, st, i, static_cast<uint32_t>(agg_a));
		if (sa.bad()) { return 0; }
		if (agg_b >= 0) {
			const StagedVec sb = staged(ws, st, i, static_cast<uint32_t>(agg_b));
			if (sb.bad()) { return 0; }
			int32_t bv[32];
			dev::decode_each<true>(sb.s, sb.vi, ws.dict(), lane, [&](int r, uint32_t x) {
				bv[r] = ((mask >> r) & 1u) ? static_cast<int32_t>(x) : 0;
			});
			dev::decode_each<true>(sa.s, sa.vi, ws.dict(), lane, [&](int r, uint32_t x) {
				p[r & 3] += static_cast<long long>(static_cast<int32_t>(x)) * static_cast<long long>(bv[r]);
			});
		} else {
			dev::decode_each<true>(sa.s, sa.vi, ws.dict(), lane, [&](int r, uint32_t x) {
				p[r & 3] += ((mask >> r) & 1u) ? static_cast<long long>(static_cast<int32_t>(x)) : 0ll;
			});
		}
		return static_cast<unsigned long long>((p[0] + p[1]) + (p[2] + p[3]));
	}

	__device__ void finish(State& S, uint32_t lane, const StageCfg&) const {
		const unsigned long long s = warp_sum_u64(S.acc);
		if (lane == 0 && s) { atomicAdd(reinterpret_cast<unsigned long long*>(result), s); }
	}
};

struct TableState {
	const uint32_t* tables;
};

// Shared parameters of the probe + group-by operators (fls_q21.cu,
// fls_q31.cu, fls_q41.cu probe_v1).
struct ProbeParams {
	uint32_t       n_probes;
	uint32_t       p_col[FLS_MAX_PROBES];
	const int32_t* p_ht[FLS_MAX_PROBES];
	int32_t        p_len[FLS_MAX_PROBES];
	int32_t        p_min[FLS_MAX_PROBES];
	int32_t        p_kind[FLS_MAX_PROBES];
	uint32_t       p_smem_off[FLS_MAX_PROBES]; // words into the CTA scratch, ~0u = probe global memory
	int32_t        n_keys;
	int32_t        key_probe[FLS_MAX_GROUP_KEYS], key_mul[FLS_MAX_GROUP_KEYS], key_slot[FLS_MAX_GROUP_KEYS];
	int32_t        sub, n_groups;
	uint32_t       stride, sum_slot; // group record: int32 words, word of the sum
	uint32_t       sum32;            // 1: wrapping int32 sum in one word, 0: int64 sum in two
	uint32_t       agg_col;
	int32_t        agg_sub; // column subtracted from the measure, or -1
	int32_t*       res;
	int32_t        sparse_rows; // see FilterAggOp

	// Payload of probe q becomes the value of every key that names it.
	__device__ __forceinline__ void take_key(uint32_t q, int32_t val, int32_t (&kv)[FLS_MAX_GROUP_KEYS]) const {
#pragma unroll
		for (int k = 0; k < FLS_MAX_GROUP_KEYS; ++k) {
			if (k < n_keys && key_probe[k] == static_cast<int32_t>(q)) { kv[k] = val; }
		}
	}

	// Small hash tables are staged into shared memory once per CTA: PHT_1 tables
	// as a presence bitmap (the probe only tests slot != 0, crystal-opt/
	// join.cuh:42-47), small PHT_2 tables verbatim.
	__device__ void stage_tables(TableState& S, uint32_t* cta_smem) const {
		S.tables            = cta_smem;
		const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
		for (uint32_t p = 0; p < n_probes; ++p) {
			if (p_smem_off[p] == ~0u) { continue; }
			uint32_t*      dst = cta_smem + p_smem_off[p];
			const int32_t* ht  = p_ht[p];
			const uint32_t len = static_cast<uint32_t>(p_len[p]);
			if (p_kind[p] == 1) {
				// Presence bitmap, 8 independent coalesced loads in flight per warp.
				const uint32_t n_words = (len + 31u) / 32u;
				for (uint32_t w0 = warp * 8u; w0 < n_words; w0 += nw * 8u) {
					int32_t x[8];
#pragma unroll
					for (uint32_t j = 0; j < 8; ++j) {
						const uint32_t idx = 32u * (w0 + j) + lane;
						x[j]               = (w0 + j < n_words && idx < len) ? __ldg(ht + idx) : 0;
					}
#pragma unroll
					for (uint32_t j = 0; j < 8; ++j) {
						const uint32_t b = __ballot_sync(0xffffffffu, x[j] != 0);
						if (lane == 0 && w0 + j < n_words) { dst[w0 + j] = b; }
					}
				}
			} else {
				const uint32_t n = 2u * len;
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
	}

	// HASH(X,Y,Z) = (X-Z) % Y (join.cuh:26): d = key - keys_min; in-range keys
	// skip the division; a negative remainder is flagged and misses.
	__device__ __forceinline__ bool slot_of(uint32_t p, uint32_t key, int32_t& h, uint32_t* err) const {
		const int32_t d = static_cast<int32_t>(key - static_cast<uint32_t>(p_min[p]));
		h               = d;
		if (static_cast<uint32_t>(d) >= static_cast<uint32_t>(p_len[p])) {
			h = d % p_len[p];
			if (h < 0) {
				raise_err(err, kErrHash);
				return false;
			}
		}
		return true;
	}

	// Probe of one key: hit?  PHT_2 hits return their value in *val.
	__device__ __forceinline__ bool probe(const TableState& S, uint32_t p, uint32_t key, int32_t* val,
	                                      uint32_t* err) const {
		int32_t h;
		if (!slot_of(p, key, h, err)) { return false; }
		const bool in_smem = p_smem_off[p] != ~0u;
		if (p_kind[p] == 1) {
			return in_smem ? ((S.tables[p_smem_off[p] + (h >> 5)] >> (h & 31)) & 1u) != 0u : __ldg(p_ht[p] + h) != 0;
		}
		const uint2 s = in_smem ? reinterpret_cast<const uint2*>(S.tables + p_smem_off[p])[h]
		                        : __ldg(reinterpret_cast<const uint2*>(p_ht[p]) + h);
		*val = static_cast<int32_t>(s.y);
		return (s.x | s.y) != 0u;
	}

	// Group-by epilogue of one selected row (fls_q21.cu:67-77, fls_q31.cu:82-91,
	// fls_q41.cu:96-104): the group of the key values in wrapping 32-bit
	// arithmetic, the key values into their words of the group record, the
	// measure (an int32, widened) into its int64 sum, or into a wrapping int32
	// sum.
	__device__ __forceinline__ void add_sum(int32_t* rec, int32_t measure) const {
		if (sum32) {
			atomicAdd(reinterpret_cast<unsigned int*>(rec + sum_slot), static_cast<unsigned int>(measure));
		} else {
			atomicAdd(reinterpret_cast<unsigned long long*>(rec + sum_slot),
			          static_cast<unsigned long long>(static_cast<long long>(measure)));
		}
	}
	__device__ __forceinline__ void emit(const int32_t (&kv)[FLS_MAX_GROUP_KEYS], uint32_t measure, uint32_t* err) const {
		uint32_t key = 0u - static_cast<uint32_t>(sub);
#pragma unroll
		for (int k = 0; k < FLS_MAX_GROUP_KEYS; ++k) {
			if (k < n_keys) { key += static_cast<uint32_t>(kv[k]) * static_cast<uint32_t>(key_mul[k]); }
		}
		const int32_t g = key < static_cast<uint32_t>(n_groups) ? static_cast<int32_t>(key)
		                                                         : static_cast<int32_t>(key) % n_groups;
		if (g < 0) {
			raise_err(err, kErrHash);
			return;
		}
		int32_t* rec = res + static_cast<int64_t>(g) * stride;
#pragma unroll
		for (int k = 0; k < FLS_MAX_GROUP_KEYS; ++k) {
			if (k < n_keys && key_slot[k] >= 0) { rec[key_slot[k]] = kv[k]; }
		}
		add_sum(rec, static_cast<int32_t>(measure));
	}
};

// Random-access form: leading PHT_1 probes run dense over the whole vector;
// from the first PHT_2 probe on (or once few rows remain) every selected row is
// probed and aggregated on its own, reading only its fields.  Used when every
// probed / summed column holds only FOR, CONST or DICT vectors.
struct ProbeGroupByRowOp : ProbeParams {
	using State = TableState;

	__device__ void cta_setup(State& S, uint32_t* cta_smem, const StageCfg&) const { stage_tables(S, cta_smem); }

	__device__ void process(State& S, uint64_t v, const WarpStage& ws, uint32_t st, uint32_t i, uint32_t lane,
	                        const StageCfg& cfg) const {
		uint32_t mask = valid_rows(cfg, v, lane);
		uint32_t p    = 0;
		for (; p < n_probes && p_kind[p] == 1; ++p) {
			if (max_rows(mask) <= sparse_rows) { break; }
			const StagedVec sv = staged(ws, st, i, p_col[p]);
			if (sv.bad() || !dev::random_access(sv.vi.scheme)) { return; }
			uint32_t vals[32];
			dev::decode_vals(sv.s, sv.vi, ws.dict(), lane, vals);
			uint32_t hit[4] = {0, 0, 0, 0};
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) {
				int32_t unused;
				hit[r & 3] |= (probe(S, p, vals[r], &unused, cfg.err) ? 1u : 0u) << r;
			}
			mask &= (hit[0] | hit[1]) | (hit[2] | hit[3]);
		}
		// Row-at-a-time rest; FOR vectors use the hoisted fast field reader.
		bool fast = staged(ws, st, i, agg_col).vi.scheme == FLS_SCHEME_FOR;
		if (agg_sub >= 0) { fast = fast && staged(ws, st, i, static_cast<uint32_t>(agg_sub)).vi.scheme == FLS_SCHEME_FOR; }
		for (uint32_t q = p; q < n_probes; ++q) { fast = fast && staged(ws, st, i, p_col[q]).vi.scheme == FLS_SCHEME_FOR; }
		if (fast) {
			dev::ForRows kr[FLS_MAX_PROBES], mr;
#pragma unroll
			for (uint32_t q = 0; q < FLS_MAX_PROBES; ++q) {
				if (q >= p && q < n_probes) {
					const StagedVec sv = staged(ws, st, i, p_col[q]);
					kr[q].init(sv.s, sv.vi, lane);
				}
			}
			{
				const StagedVec sv = staged(ws, st, i, agg_col);
				mr.init(sv.s, sv.vi, lane);
			}
			dev::ForRows sr {};
			if (agg_sub >= 0) {
				const StagedVec sv = staged(ws, st, i, static_cast<uint32_t>(agg_sub));
				sr.init(sv.s, sv.vi, lane);
			}
			const int n_it = max_rows(mask);
			for (int it = 0; it < n_it; ++it) {
				const bool     have = mask != 0u;
				const uint32_t r    = have ? static_cast<uint32_t>(__ffs(mask)) - 1u : 0u;
				mask &= mask - 1u;
				int32_t kv[FLS_MAX_GROUP_KEYS] = {0, 0, 0};
				bool    pass = have;
#pragma unroll
				for (uint32_t q = 0; q < FLS_MAX_PROBES; ++q) {
					if (q >= p && q < n_probes) {
						int32_t val = 0;
						const uint32_t key = kr[q].get(r);
						if (pass) { pass = probe(S, q, key, &val, cfg.err); }
						take_key(q, val, kv);
					}
				}
				const uint32_t m = mr.get(r) - (agg_sub >= 0 ? sr.get(r) : 0u);
				if (pass) { emit(kv, m, cfg.err); }
			}
			return;
		}
		while (mask) {
			const uint32_t r = static_cast<uint32_t>(__ffs(mask)) - 1u;
			mask &= mask - 1u;
			int32_t kv[FLS_MAX_GROUP_KEYS] = {0, 0, 0};
			bool    pass = true;
			for (uint32_t q = p; q < n_probes && pass; ++q) {
				const StagedVec sv = staged(ws, st, i, p_col[q]);
				int32_t         val = 0;
				pass = !sv.bad() && probe(S, q, dev::value_at(sv.s, sv.vi, lane, r), &val, cfg.err);
				take_key(q, val, kv);
			}
			if (!pass) { continue; }
			const StagedVec sm = staged(ws, st, i, agg_col);
			if (sm.bad()) { continue; }
			uint32_t m = dev::value_at(sm.s, sm.vi, lane, r);
			if (agg_sub >= 0) {
				const StagedVec sb = staged(ws, st, i, static_cast<uint32_t>(agg_sub));
				if (sb.bad()) { continue; }
				m -= dev::value_at(sb.s, sb.vi, lane, r);
			}
			emit(kv, m, cfg.err);
		}
	}
	__device__ void finish(State&, uint32_t, const StageCfg&) const {}
};

// General form (any scheme, including the running-sum schemes DELTA / RLE):
// every probe and the aggregate are evaluated over whole vectors.
struct ProbeGroupByDenseOp : ProbeParams {
	using State = TableState;

	__device__ void cta_setup(State& S, uint32_t* cta_smem, const StageCfg&) const { stage_tables(S, cta_smem); }

	// Decodes probe column q and, for the selected rows, looks up its payload.
	__device__ __forceinline__ void payloads(const State& S, uint32_t q, uint32_t mask, const WarpStage& ws, uint32_t st,
	                                         uint32_t i, uint32_t lane, uint32_t (&vals)[32], uint32_t* err) const {
		const StagedVec sv = staged(ws, st, i, p_col[q]);
		dev::decode_vals(sv.s, sv.vi, ws.dict(), lane, vals);
#pragma unroll
		for (uint32_t r = 0; r < 32; ++r) {
			int32_t val = 0;
			if ((mask >> r) & 1u) { probe(S, q, vals[r], &val, err); }
			vals[r] = static_cast<uint32_t>(val);
		}
	}

	__device__ void process(State& S, uint64_t v, const WarpStage& ws, uint32_t st, uint32_t i, uint32_t lane,
	                        const StageCfg& cfg) const {
		uint32_t mask = valid_rows(cfg, v, lane);
		uint32_t vals[32];
		// 1. the selection: every probe over the whole vector
		for (uint32_t p = 0; p < n_probes; ++p) {
			const StagedVec sv = staged(ws, st, i, p_col[p]);
			if (sv.bad()) { return; }
			dev::decode_vals(sv.s, sv.vi, ws.dict(), lane, vals);
			uint32_t hit = 0;
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) {
				if ((mask >> r) & 1u) {
					int32_t val = 0;
					if (probe(S, p, vals[r], &val, cfg.err)) { hit |= 1u << r; }
				}
			}
			mask &= hit;
			if (!__any_sync(0xffffffffu, mask)) { return; }
		}
		if (staged(ws, st, i, agg_col).bad() || (agg_sub >= 0 && staged(ws, st, i, static_cast<uint32_t>(agg_sub)).bad())) {
			return;
		}
		// 2. group ids: the key payloads re-read for the selected rows
		uint32_t grp[32];
#pragma unroll
		for (uint32_t r = 0; r < 32; ++r) { grp[r] = 0u - static_cast<uint32_t>(sub); }
		for (int k = 0; k < n_keys; ++k) {
			payloads(S, static_cast<uint32_t>(key_probe[k]), mask, ws, st, i, lane, vals, cfg.err);
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) { grp[r] += vals[r] * static_cast<uint32_t>(key_mul[k]); }
		}
#pragma unroll
		for (uint32_t r = 0; r < 32; ++r) {
			const int32_t key = static_cast<int32_t>(grp[r]);
			const int32_t g   = grp[r] < static_cast<uint32_t>(n_groups) ? key : key % n_groups;
			if (((mask >> r) & 1u) && g < 0) {
				raise_err(cfg.err, kErrHash);
				mask &= ~(1u << r);
			}
			grp[r] = static_cast<uint32_t>(g);
		}
		// 3. key words of the group records
		for (int k = 0; k < n_keys; ++k) {
			if (key_slot[k] < 0) { continue; }
			payloads(S, static_cast<uint32_t>(key_probe[k]), mask, ws, st, i, lane, vals, cfg.err);
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) {
				if ((mask >> r) & 1u) { res[static_cast<int64_t>(grp[r]) * stride + key_slot[k]] = static_cast<int32_t>(vals[r]); }
			}
		}
		// 4. the measure (minus the subtracted column) into the sums
		const StagedVec sm = staged(ws, st, i, agg_col);
		dev::decode_vals(sm.s, sm.vi, ws.dict(), lane, vals);
		if (agg_sub >= 0) {
			const StagedVec sb = staged(ws, st, i, static_cast<uint32_t>(agg_sub));
			dev::decode_each<true>(sb.s, sb.vi, ws.dict(), lane, [&](int r, uint32_t y) { vals[r] -= y; });
		}
#pragma unroll
		for (uint32_t r = 0; r < 32; ++r) {
			if ((mask >> r) & 1u) { add_sum(res + static_cast<int64_t>(grp[r]) * stride, static_cast<int32_t>(vals[r])); }
		}
	}
	__device__ void finish(State&, uint32_t, const StageCfg&) const {}
};

// Selective perfect-hash build (join.cuh:190-334, fls_q21.cu:197-263): rows
// whose filter value lies in [lo0, hi0] or [lo1, hi1].
__global__ void pht_build_kernel(const int32_t* __restrict__ filter, int32_t lo0, int32_t hi0, int32_t lo1,
                                 int32_t hi1, const int32_t* __restrict__ keys, const int32_t* __restrict__ vals,
                                 uint64_t n, int32_t* ht, int32_t len, int32_t keys_min, uint32_t* err) {
	const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
		if (filter) {
			const int32_t f = __ldg(filter + i);
			if (!((f >= lo0 && f <= hi0) || (f >= lo1 && f <= hi1))) { continue; }
		}
		const int32_t key = __ldg(keys + i);
		const int32_t h   = static_cast<int32_t>(static_cast<uint32_t>(key) - static_cast<uint32_t>(keys_min)) % len;
		if (h < 0) {
			raise_err(err, kErrHash);
			continue;
		}
		if (vals == nullptr) {
			atomicCAS(ht + h, 0, key);
		} else {
			atomicCAS(ht + 2 * h, 0, key);
			ht[2 * h + 1] = __ldg(vals + i);
		}
	}
}

} // namespace
} // namespace fls

using namespace fls;

namespace {

// Validates a filter-aggregate descriptor and puts its filters in evaluation
// order: most selective first (the result does not depend on the order).
// Selectivity is estimated for uniform FOR columns as the share of the
// column's value domain [base, base + 2^bw) inside the range; other columns
// keep their position.  empty: some range is empty, so nothing is selected.
fls_status order_filters(const fls_filter_agg_desc* desc, fls_filter (&order)[FLS_MAX_FILTERS], bool& empty) {
	if (!desc || !desc->cols) { return set_error(FLS_ERR_INVALID_ARG, "fls_query_filter_agg: null pointer"); }
	if (desc->n_filters > FLS_MAX_FILTERS) { return set_error(FLS_ERR_INVALID_ARG, "too many filters"); }
	const int32_t nc = static_cast<int32_t>(desc->n_cols);
	if (desc->agg_a >= nc || desc->agg_b >= nc || (desc->agg_b >= 0 && desc->agg_a < 0)) {
		return set_error(FLS_ERR_INVALID_ARG, "aggregate column out of range");
	}
	empty = false;
	double sel[FLS_MAX_FILTERS];
	for (uint32_t f = 0; f < desc->n_filters; ++f) {
		order[f] = desc->filters[f];
		sel[f]   = 1.0;
		if (order[f].col >= desc->n_cols) { return set_error(FLS_ERR_INVALID_ARG, "filter column out of range"); }
		empty               = empty || order[f].lo > order[f].hi;
		const fls_column& c = desc->cols[order[f].col];
		if (!c.meta && c.scheme == FLS_SCHEME_FOR && c.bw < 32) {
			const double lo = std::max<double>(order[f].lo, c.base);
			const double hi = std::min<double>(order[f].hi, static_cast<double>(c.base) + std::ldexp(1.0, c.bw) - 1);
			sel[f]          = hi < lo ? 0.0 : (hi - lo + 1.0) / std::ldexp(1.0, c.bw);
		}
	}
	for (uint32_t f = 1; f < desc->n_filters; ++f) { // stable insertion sort
		for (uint32_t g = f; g > 0 && sel[g] < sel[g - 1]; --g) {
			std::swap(sel[g], sel[g - 1]);
			std::swap(order[g], order[g - 1]);
		}
	}
	return FLS_OK;
}

// Validates a probe + group-by descriptor.
fls_status check_join_desc(const fls_join_agg_desc* desc) {
	if (!desc || !desc->cols) { return set_error(FLS_ERR_INVALID_ARG, "fls_query_probe_groupby: null pointer"); }
	if (desc->n_probes == 0 || desc->n_probes > FLS_MAX_PROBES) { return set_error(FLS_ERR_INVALID_ARG, "1..4 probes"); }
	if (desc->agg_col >= desc->n_cols || desc->n_groups <= 0) {
		return set_error(FLS_ERR_INVALID_ARG, "bad aggregate column or group count");
	}
	const int32_t np = static_cast<int32_t>(desc->n_probes);
	if (desc->key_a < 0 || desc->key_b < 0 || desc->key_a >= np || desc->key_b >= np ||
	    desc->probes[desc->key_a].kind != 2 || desc->probes[desc->key_b].kind != 2) {
		return set_error(FLS_ERR_INVALID_ARG, "group keys must name PHT_2 probes");
	}
	for (uint32_t p = 0; p < desc->n_probes; ++p) {
		const fls_probe& pr = desc->probes[p];
		if (pr.col >= desc->n_cols || !pr.ht || pr.ht_len <= 0 || (pr.kind != 1 && pr.kind != 2)) {
			return set_error(FLS_ERR_INVALID_ARG, "bad probe");
		}
		if (pr.kind == 2 && (reinterpret_cast<uintptr_t>(pr.ht) & 7u)) {
			return set_error(FLS_ERR_ALIGNMENT, "PHT_2 tables must be 8-byte aligned");
		}
	}
	return FLS_OK;
}

// fls_q21.cu's group-by as the general form: keys (payload of key_a) x mul and
// (payload of key_b) x 1, record {b, a, int64 sum}.
fls_join_groupby_desc groupby_of(const fls_join_agg_desc& d) {
	fls_join_groupby_desc g {};
	g.cols   = d.cols;
	g.n_cols = d.n_cols;
	for (uint32_t p = 0; p < FLS_MAX_PROBES; ++p) { g.probes[p] = d.probes[p]; }
	g.n_probes     = d.n_probes;
	g.agg_col      = d.agg_col;
	g.agg_sub_col  = -1;
	g.n_keys       = 2;
	g.key_probe[0] = d.key_a;
	g.key_probe[1] = d.key_b;
	g.key_probe[2] = -1;
	g.key_mul[0]   = d.group_mul;
	g.key_mul[1]   = 1;
	g.key_mul[2]   = 0;
	g.key_slot[0]  = 1;
	g.key_slot[1]  = 0;
	g.key_slot[2]  = -1;
	g.group_sub    = d.group_sub;
	g.n_groups     = d.n_groups;
	g.res_stride   = 4;
	g.sum_slot     = 2;
	g.sum_bits     = 64;
	return g;
}

// Validates a general join + group-by descriptor.
fls_status check_groupby_desc(const fls_join_groupby_desc* d) {
	if (!d || !d->cols) { return set_error(FLS_ERR_INVALID_ARG, "fls_query_join_groupby: null pointer"); }
	if (d->n_probes == 0 || d->n_probes > FLS_MAX_PROBES) { return set_error(FLS_ERR_INVALID_ARG, "1..4 probes"); }
	if (d->agg_col >= d->n_cols || d->agg_sub_col >= static_cast<int32_t>(d->n_cols) || d->agg_sub_col < -1 ||
	    d->n_groups <= 0) {
		return set_error(FLS_ERR_INVALID_ARG, "bad measure column or group count");
	}
	if (d->sum_bits != 0 && d->sum_bits != 32 && d->sum_bits != 64) {
		return set_error(FLS_ERR_INVALID_ARG, "sum_bits must be 32 or 64");
	}
	const bool     sum32     = d->sum_bits == 32;
	const uint32_t sum_words = sum32 ? 1u : 2u;
	if (sum32 ? (d->res_stride < 1 || d->sum_slot >= d->res_stride)
	          : (d->res_stride < 2 || (d->res_stride & 1u) || (d->sum_slot & 1u) || d->sum_slot + 1u >= d->res_stride)) {
		return set_error(FLS_ERR_INVALID_ARG,
		                 "group record: sum word inside the record (int64: even stride, even sum word)");
	}
	if (d->n_keys == 0 || d->n_keys > FLS_MAX_GROUP_KEYS) { return set_error(FLS_ERR_INVALID_ARG, "1..3 group keys"); }
	for (uint32_t k = 0; k < d->n_keys; ++k) {
		const int32_t q = d->key_probe[k], w = d->key_slot[k];
		if (q < 0 || q >= static_cast<int32_t>(d->n_probes) || d->probes[q].kind != 2) {
			return set_error(FLS_ERR_INVALID_ARG, "group keys must name PHT_2 probes");
		}
		if (w < -1 || w >= static_cast<int32_t>(d->res_stride) ||
		    (w >= static_cast<int32_t>(d->sum_slot) && w < static_cast<int32_t>(d->sum_slot + sum_words))) {
			return set_error(FLS_ERR_INVALID_ARG, "key word outside the group record or on the sum");
		}
	}
	for (uint32_t p = 0; p < d->n_probes; ++p) {
		const fls_probe& pr = d->probes[p];
		if (pr.col >= d->n_cols || !pr.ht || pr.ht_len <= 0 || (pr.kind != 1 && pr.kind != 2)) {
			return set_error(FLS_ERR_INVALID_ARG, "bad probe");
		}
		if (pr.kind == 2 && (reinterpret_cast<uintptr_t>(pr.ht) & 7u)) {
			return set_error(FLS_ERR_ALIGNMENT, "PHT_2 tables must be 8-byte aligned");
		}
	}
	return FLS_OK;
}

} // namespace

extern "C" {

fls_status fls_query_filter_agg(const fls_filter_agg_desc* desc, int64_t* d_result, fls_stream_t stream) {
	if (!d_result) { return set_error(FLS_ERR_INVALID_ARG, "fls_query_filter_agg: null pointer"); }
	fls_filter order[FLS_MAX_FILTERS];
	bool       empty = false;
	fls_status s     = order_filters(desc, order, empty);
	if (s != FLS_OK) { return s; }
	FilterAggOp op {};
	op.n_filters = desc->n_filters;
	for (uint32_t f = 0; f < desc->n_filters; ++f) {
		op.f_col[f]   = order[f].col;
		op.f_lo[f]    = static_cast<uint32_t>(order[f].lo);
		op.f_range[f] = static_cast<uint32_t>(order[f].hi) - static_cast<uint32_t>(order[f].lo);
	}
	op.agg_a       = desc->agg_a;
	op.agg_b       = desc->agg_b;
	op.result      = reinterpret_cast<long long*>(d_result);
	op.sparse_rows = tuning_sparse_rows();
	StageCfg cfg;
	uint32_t grid, threads;
	size_t   smem;
	s = plan_stages(desc->cols, desc->n_cols, 0u, 0u, cfg, grid, threads, smem);
	if (s != FLS_OK) { return s; }
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	if ((s = cuda_check(cudaMemsetAsync(d_result, 0, sizeof(int64_t), st), "cudaMemsetAsync")) != FLS_OK) { return s; }
	if (empty) { return FLS_OK; } // an empty range selects nothing
	if (tuning_jit()) {
		bool used = false;
		s = jit_filter_agg(desc->cols, order, desc->n_filters, desc->agg_a, desc->agg_b, d_result, op.sparse_rows, st,
		                   used);
		if (s != FLS_OK || used) { return s; }
	}
	return launch_staged(cfg, op, grid, threads, smem, st);
}

fls_status fls_jit_precompile(const fls_filter_agg_desc* desc) {
	fls_filter order[FLS_MAX_FILTERS];
	bool       empty = false;
	fls_status s     = order_filters(desc, order, empty);
	if (s != FLS_OK) { return s; }
	JitShape sh;
	if (!jit_shape(desc->cols, order, desc->n_filters, desc->agg_a, desc->agg_b, sh)) {
		return set_error(FLS_ERR_UNSUPPORTED, "query does not qualify for specialisation (uniform FOR columns only)");
	}
	if (!jit_compile(desc->cols, sh)) {
		return set_error(FLS_ERR_UNSUPPORTED, std::string("specialisation failed: ") + fls_jit_last_log());
	}
	return FLS_OK;
}

fls_status fls_jit_precompile_probe(const fls_join_agg_desc* desc) {
	fls_status s = check_join_desc(desc);
	if (s != FLS_OK) { return s; }
	const fls_join_groupby_desc g = groupby_of(*desc);
	return fls_jit_precompile_join(&g);
}

fls_status fls_jit_precompile_join(const fls_join_groupby_desc* desc) {
	fls_status s = check_groupby_desc(desc);
	if (s != FLS_OK) { return s; }
	JitProbeShape sh;
	if (!jit_probe_shape(desc, sh)) {
		return set_error(FLS_ERR_UNSUPPORTED, "query does not qualify for specialisation (uniform FOR columns only)");
	}
	if (!jit_compile(desc, sh)) {
		return set_error(FLS_ERR_UNSUPPORTED, std::string("specialisation failed: ") + fls_jit_last_log());
	}
	return FLS_OK;
}

fls_status fls_pht_build(const int32_t* d_filter, int32_t filter_eq, const int32_t* d_keys, const int32_t* d_vals,
                         uint64_t n, int32_t* d_ht, int32_t ht_len, int32_t keys_min, fls_stream_t stream) {
	return fls_pht_build_ranges(d_filter, filter_eq, filter_eq, 1, 0, d_keys, d_vals, n, d_ht, ht_len, keys_min,
	                            stream);
}

fls_status fls_pht_build_ranges(const int32_t* d_filter, int32_t lo0, int32_t hi0, int32_t lo1, int32_t hi1,
                                const int32_t* d_keys, const int32_t* d_vals, uint64_t n, int32_t* d_ht,
                                int32_t ht_len, int32_t keys_min, fls_stream_t stream) {
	if (!d_keys || !d_ht || ht_len <= 0) { return set_error(FLS_ERR_INVALID_ARG, "fls_pht_build: bad arguments"); }
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	if (n == 0) { return FLS_OK; }
	const uint64_t want = (n + 255u) / 256u;
	const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>(want, static_cast<uint64_t>(di.sms) * 8u));
	pht_build_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_filter, lo0, hi0, lo1, hi1, d_keys,
	                                                                           d_vals, n, d_ht, ht_len, keys_min,
	                                                                           device_error_word(reinterpret_cast<cudaStream_t>(stream)));
	count_launch();
	return cuda_check(cudaGetLastError(), "pht_build_kernel launch");
}

uint64_t fls_join_workspace_bytes(const fls_join_groupby_desc* desc) {
	return check_groupby_desc(desc) == FLS_OK ? jit_probe_workspace_bytes(desc) : 0u;
}

uint64_t fls_probe_workspace_bytes(const fls_join_agg_desc* desc) {
	if (check_join_desc(desc) != FLS_OK) { return 0u; }
	const fls_join_groupby_desc g = groupby_of(*desc);
	return fls_join_workspace_bytes(&g);
}

fls_status fls_query_join_groupby(const fls_join_groupby_desc* desc, int32_t* d_res, fls_stream_t stream) {
	return fls_query_join_groupby_ws(desc, d_res, nullptr, 0u, stream);
}

fls_status fls_query_join_groupby_ws(const fls_join_groupby_desc* desc, int32_t* d_res, void* d_workspace,
                                     uint64_t workspace_bytes, fls_stream_t stream) {
	if (!d_res) { return set_error(FLS_ERR_INVALID_ARG, "fls_query_join_groupby: null pointer"); }
	if (reinterpret_cast<uintptr_t>(d_workspace) & 15u) {
		return set_error(FLS_ERR_ALIGNMENT, "workspace must be 16-byte aligned");
	}
	if (reinterpret_cast<uintptr_t>(d_res) & 7u) { return set_error(FLS_ERR_ALIGNMENT, "result must be 8-byte aligned"); }
	fls_status s = check_groupby_desc(desc);
	if (s != FLS_OK) { return s; }
	ProbeParams op {};
	op.n_probes = desc->n_probes;
	// Small tables go to shared memory, first come first served.
	uint32_t       cta_words = 0;
	const uint32_t budget    = 48u * 1024u / 4u;
	for (uint32_t p = 0; p < desc->n_probes; ++p) {
		const fls_probe& pr = desc->probes[p];
		op.p_col[p]          = pr.col;
		op.p_ht[p]           = pr.ht;
		op.p_len[p]          = pr.ht_len;
		op.p_min[p]          = pr.keys_min;
		op.p_kind[p]         = pr.kind;
		const uint64_t words = pr.kind == 1 ? (static_cast<uint64_t>(pr.ht_len) + 31u) / 32u
		                                    : 2ull * static_cast<uint64_t>(pr.ht_len);
		if (cta_words + words <= budget) {
			op.p_smem_off[p] = cta_words;
			cta_words += static_cast<uint32_t>((words + 3u) & ~3ull);
		} else {
			op.p_smem_off[p] = ~0u;
		}
	}
	op.n_keys = static_cast<int32_t>(desc->n_keys);
	for (uint32_t k = 0; k < FLS_MAX_GROUP_KEYS; ++k) {
		op.key_probe[k] = k < desc->n_keys ? desc->key_probe[k] : -1;
		op.key_mul[k]   = k < desc->n_keys ? desc->key_mul[k] : 0;
		op.key_slot[k]  = k < desc->n_keys ? desc->key_slot[k] : -1;
	}
	op.sub         = desc->group_sub;
	op.n_groups    = desc->n_groups;
	op.stride      = desc->res_stride;
	op.sum_slot    = desc->sum_slot;
	op.sum32       = desc->sum_bits == 32 ? 1u : 0u;
	op.agg_col     = desc->agg_col;
	op.agg_sub     = desc->agg_sub_col;
	op.res         = d_res;
	op.sparse_rows = tuning_sparse_rows();
	// The row-at-a-time form needs random access to every column it reads.
	const uint32_t seq_schemes = (1u << FLS_SCHEME_DELTA) | (1u << FLS_SCHEME_RLE);
	bool           rnd         = true;
	for (uint32_t c = 0; c < desc->n_cols; ++c) {
		const fls_column& col = desc->cols[c];
		const uint32_t    mask = col.meta ? col.scheme_mask : (1u << col.scheme);
		rnd                   = rnd && !(mask & seq_schemes);
	}
	StageCfg cfg;
	uint32_t grid, threads;
	size_t   smem;
	s = plan_stages(desc->cols, desc->n_cols, 0u, cta_words, cfg, grid, threads, smem);
	if (s != FLS_OK) { return s; }
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	s = cuda_check(cudaMemsetAsync(d_res, 0,
	                               sizeof(int32_t) * static_cast<size_t>(desc->res_stride) *
	                                   static_cast<size_t>(desc->n_groups),
	                               st),
	               "cudaMemsetAsync");
	if (s != FLS_OK) { return s; }
	if (tuning_jit()) {
		bool used = false;
		s = jit_probe_groupby(desc, d_res, op.sparse_rows, d_workspace, workspace_bytes, st, used);
		if (s != FLS_OK || used) { return s; }
	}
	if (rnd) {
		ProbeGroupByRowOp rop;
		static_cast<ProbeParams&>(rop) = op;
		return launch_staged(cfg, rop, grid, threads, smem, st);
	}
	ProbeGroupByDenseOp dop;
	static_cast<ProbeParams&>(dop) = op;
	return launch_staged(cfg, dop, grid, threads, smem, st);
}

fls_status fls_query_probe_groupby(const fls_join_agg_desc* desc, int32_t* d_res, fls_stream_t stream) {
	return fls_query_probe_groupby_ws(desc, d_res, nullptr, 0u, stream);
}

fls_status fls_query_probe_groupby_ws(const fls_join_agg_desc* desc, int32_t* d_res, void* d_workspace,
                                      uint64_t workspace_bytes, fls_stream_t stream) {
	if (!d_res) { return set_error(FLS_ERR_INVALID_ARG, "fls_query_probe_groupby: null pointer"); }
	fls_status s = check_join_desc(desc);
	if (s != FLS_OK) { return s; }
	const fls_join_groupby_desc g = groupby_of(*desc);
	return fls_query_join_groupby_ws(&g, d_res, d_workspace, workspace_bytes, stream);
}
} // extern "C"
