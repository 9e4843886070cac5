// fls_query.cu -- fused decode + query operators: filter-aggregate, selective
// perfect-hash build, and decode + multi-probe + int64 group-by.
//
// Reference counterparts: QueryKernel_v1/_v2 (fastlanes/src/ssb/fls_q11.cu:29-135),
// build_hashtable_{s,p,d} and probe_v1..v3 (fls_q21.cu:21-263), with the tile
// primitives of fastlanes/src/include/crystal-opt/{pred,load,reduce,join}.cuh.
#include "fls_pipeline.cuh"

namespace fls {
namespace {

struct AccState {
	unsigned long long acc;
};

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

	__device__ void cta_setup(State&, uint32_t*, const StageCfg&) const {}
	__device__ void process(State& S, uint64_t v, const WarpStage& ws, uint32_t st, uint32_t lane,
	                        const StageCfg& cfg) const {
		uint32_t mask = valid_rows(cfg, v, lane);
		uint32_t vals[32];
		for (uint32_t f = 0; f < n_filters; ++f) {
			if (!stage_decode(ws, st, f_col[f], lane, vals)) { return; }
			const uint32_t lo = f_lo[f], range = f_range[f];
			uint32_t       fm = 0;
			// lo <= x <= hi  <=>  (x - lo) <= (hi - lo) in wrapping unsigned arithmetic.
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) { fm |= (vals[r] - lo <= range ? 1u : 0u) << r; }
			mask &= fm;
			if (!__any_sync(0xffffffffu, mask)) { return; }
		}
		if (agg_a < 0) {
			S.acc += static_cast<unsigned long long>(__popc(mask));
			return;
		}
		long long a = 0;
		if (agg_b >= 0) {
			int32_t bv[32];
			if (!stage_decode(ws, st, static_cast<uint32_t>(agg_b), lane, vals)) { return; }
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) { bv[r] = ((mask >> r) & 1u) ? static_cast<int32_t>(vals[r]) : 0; }
			if (!stage_decode(ws, st, static_cast<uint32_t>(agg_a), lane, vals)) { return; }
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) {
				a += static_cast<long long>(static_cast<int32_t>(vals[r])) * static_cast<long long>(bv[r]);
			}
		} else {
			if (!stage_decode(ws, st, static_cast<uint32_t>(agg_a), lane, vals)) { return; }
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) {
				a += ((mask >> r) & 1u) ? static_cast<long long>(static_cast<int32_t>(vals[r])) : 0ll;
			}
		}
		S.acc += static_cast<unsigned long long>(a);
	}
	__device__ void finish(State& S, uint32_t lane, const StageCfg&) const {
		const unsigned long long s = warp_sum_u64(S.acc);
		if (lane == 0 && s) { atomicAdd(reinterpret_cast<unsigned long long*>(result), s); }
	}
};

struct TableState {
	const uint32_t* tables;
};

// Probe + group-by.  Small hash tables are staged into shared memory once per
// CTA: PHT_1 tables as a presence bitmap (the probe only tests slot != 0,
// crystal-opt/join.cuh:42-47), small PHT_2 tables verbatim.
struct ProbeGroupByOp {
	using State = TableState;
	uint32_t       n_probes;
	uint32_t       p_col[FLS_MAX_PROBES];
	const int32_t* p_ht[FLS_MAX_PROBES];
	int32_t        p_len[FLS_MAX_PROBES];
	int32_t        p_min[FLS_MAX_PROBES];
	int32_t        p_kind[FLS_MAX_PROBES];
	uint32_t       p_smem_off[FLS_MAX_PROBES]; // words into the CTA scratch, ~0u = probe global memory
	int32_t        key_a, key_b, mul, sub, n_groups;
	uint32_t       agg_col;
	int32_t*       res;

	__device__ void cta_setup(State& S, uint32_t* cta_smem, const StageCfg&) const {
		S.tables            = cta_smem;
		const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
		for (uint32_t p = 0; p < n_probes; ++p) {
			if (p_smem_off[p] == ~0u) { continue; }
			uint32_t*      dst = cta_smem + p_smem_off[p];
			const int32_t* ht  = p_ht[p];
			const uint32_t len = static_cast<uint32_t>(p_len[p]);
			if (p_kind[p] == 1) {
				const uint32_t n_words = (len + 31u) / 32u;
				for (uint32_t w = warp; w < n_words; w += nw) {
					const uint32_t i   = 32u * w + lane;
					const bool     set = i < len && __ldg(ht + i) != 0;
					const uint32_t b   = __ballot_sync(0xffffffffu, set);
					if (lane == 0) { dst[w] = b; }
				}
			} else {
				for (uint32_t i = threadIdx.x; i < 2u * len; i += blockDim.x) {
					dst[i] = static_cast<uint32_t>(__ldg(ht + i));
				}
			}
		}
	}

	__device__ void process(State& S, uint64_t v, const WarpStage& ws, uint32_t st, uint32_t lane,
	                        const StageCfg& cfg) const {
		uint32_t mask = valid_rows(cfg, v, lane);
		uint32_t vals[32];
		int32_t  pa[32], pb[32];
		for (uint32_t p = 0; p < n_probes; ++p) {
			if (!stage_decode(ws, st, p_col[p], lane, vals)) { return; }
			const int32_t   len = p_len[p], kmin = p_min[p];
			const bool      one     = p_kind[p] == 1;
			const bool      in_smem = p_smem_off[p] != ~0u;
			const uint32_t* tab     = S.tables + (in_smem ? p_smem_off[p] : 0u);
			const int32_t*  ght     = p_ht[p];
			const bool      wa = static_cast<int32_t>(p) == key_a, wb = static_cast<int32_t>(p) == key_b;
			uint32_t        hit = 0;
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) {
				if ((mask >> r) & 1u) {
					// HASH(X,Y,Z) = (X-Z) % Y (join.cuh:26); in-range keys skip the division.
					const int32_t d = static_cast<int32_t>(vals[r] - static_cast<uint32_t>(kmin));
					int32_t       h = d;
					bool          ok = true;
					if (static_cast<uint32_t>(d) >= static_cast<uint32_t>(len)) {
						h  = d % len;
						ok = h >= 0;
						if (!ok) { raise_err(cfg.err, kErrHash); }
					}
					if (ok) {
						if (one) {
							const bool f = in_smem ? ((tab[h >> 5] >> (h & 31)) & 1u) != 0u : (__ldg(ght + h) != 0);
							hit |= (f ? 1u : 0u) << r;
						} else {
							const uint2 s = in_smem ? reinterpret_cast<const uint2*>(tab)[h]
							                        : __ldg(reinterpret_cast<const uint2*>(ght) + h);
							if (s.x | s.y) {
								hit |= 1u << r;
								if (wa) { pa[r] = static_cast<int32_t>(s.y); }
								if (wb) { pb[r] = static_cast<int32_t>(s.y); }
							}
						}
					}
				}
			}
			mask &= hit;
			if (!__any_sync(0xffffffffu, mask)) { return; }
		}
		if (!stage_decode(ws, st, agg_col, lane, vals)) { return; }
#pragma unroll
		for (uint32_t r = 0; r < 32; ++r) {
			if ((mask >> r) & 1u) {
				// (a*mul + (b - sub)) % n_groups in wrapping 32-bit arithmetic.
				const int32_t key = static_cast<int32_t>(static_cast<uint32_t>(pa[r]) * static_cast<uint32_t>(mul) +
				                                         (static_cast<uint32_t>(pb[r]) - static_cast<uint32_t>(sub)));
				const int32_t g   = key % n_groups;
				if (g < 0) {
					raise_err(cfg.err, kErrHash);
				} else {
					res[4 * g]     = pb[r];
					res[4 * g + 1] = pa[r];
					atomicAdd(reinterpret_cast<unsigned long long*>(res + 4 * g + 2),
					          static_cast<unsigned long long>(static_cast<long long>(static_cast<int32_t>(vals[r]))));
				}
			}
		}
	}
	__device__ void finish(State&, uint32_t, const StageCfg&) const {}
};

// Selective perfect-hash build (join.cuh:190-334, fls_q21.cu:197-263).
__global__ void pht_build_kernel(const int32_t* __restrict__ filter, int32_t filter_eq,
                                 const int32_t* __restrict__ keys, const int32_t* __restrict__ vals, uint64_t n,
                                 int32_t* ht, int32_t len, int32_t keys_min, uint32_t* err) {
	const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
		if (filter && __ldg(filter + i) != filter_eq) { continue; }
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

extern "C" {

fls_status fls_query_filter_agg(const fls_filter_agg_desc* desc, int64_t* d_result, fls_stream_t stream) {
	if (!desc || !d_result || !desc->cols) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_query_filter_agg: null pointer");
	}
	if (desc->n_filters > FLS_MAX_FILTERS) { return set_error(FLS_ERR_INVALID_ARG, "too many filters"); }
	const int32_t nc = static_cast<int32_t>(desc->n_cols);
	if (desc->agg_a >= nc || desc->agg_b >= nc || (desc->agg_b >= 0 && desc->agg_a < 0)) {
		return set_error(FLS_ERR_INVALID_ARG, "aggregate column out of range");
	}
	FilterAggOp op {};
	op.n_filters = desc->n_filters;
	bool empty   = false;
	for (uint32_t f = 0; f < desc->n_filters; ++f) {
		const fls_filter& fl = desc->filters[f];
		if (fl.col >= desc->n_cols) { return set_error(FLS_ERR_INVALID_ARG, "filter column out of range"); }
		empty         = empty || fl.lo > fl.hi;
		op.f_col[f]   = fl.col;
		op.f_lo[f]    = static_cast<uint32_t>(fl.lo);
		op.f_range[f] = static_cast<uint32_t>(fl.hi) - static_cast<uint32_t>(fl.lo);
	}
	op.agg_a  = desc->agg_a;
	op.agg_b  = desc->agg_b;
	op.result = reinterpret_cast<long long*>(d_result);
	StageCfg   cfg;
	uint32_t   grid, threads;
	size_t     smem;
	fls_status s = plan_stages(desc->cols, desc->n_cols, 0u, 0u, cfg, grid, threads, smem);
	if (s != FLS_OK) { return s; }
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	if ((s = cuda_check(cudaMemsetAsync(d_result, 0, sizeof(int64_t), st), "cudaMemsetAsync")) != FLS_OK) { return s; }
	if (empty) { return FLS_OK; } // an empty range selects nothing
	return launch_staged(cfg, op, grid, threads, smem, st);
}

fls_status fls_pht_build(const int32_t* d_filter, int32_t filter_eq, const int32_t* d_keys, const int32_t* d_vals,
                         uint64_t n, int32_t* d_ht, int32_t ht_len, int32_t keys_min, fls_stream_t stream) {
	if (!d_keys || !d_ht || ht_len <= 0) { return set_error(FLS_ERR_INVALID_ARG, "fls_pht_build: bad arguments"); }
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	if (n == 0) { return FLS_OK; }
	const uint64_t want = (n + 255u) / 256u;
	const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>(want, static_cast<uint64_t>(di.sms) * 8u));
	pht_build_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_filter, filter_eq, d_keys, d_vals, n,
	                                                                           d_ht, ht_len, keys_min,
	                                                                           device_error_word());
	count_launch();
	return cuda_check(cudaGetLastError(), "pht_build_kernel launch");
}

fls_status fls_query_probe_groupby(const fls_join_agg_desc* desc, int32_t* d_res, fls_stream_t stream) {
	if (!desc || !d_res || !desc->cols) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_query_probe_groupby: null pointer");
	}
	if (desc->n_probes == 0 || desc->n_probes > FLS_MAX_PROBES) { return set_error(FLS_ERR_INVALID_ARG, "1..4 probes"); }
	if (desc->agg_col >= desc->n_cols || desc->n_groups <= 0) {
		return set_error(FLS_ERR_INVALID_ARG, "bad aggregate column or group count");
	}
	if (reinterpret_cast<uintptr_t>(d_res) & 7u) { return set_error(FLS_ERR_ALIGNMENT, "result must be 8-byte aligned"); }
	const int32_t np = static_cast<int32_t>(desc->n_probes);
	if (desc->key_a < 0 || desc->key_b < 0 || desc->key_a >= np || desc->key_b >= np ||
	    desc->probes[desc->key_a].kind != 2 || desc->probes[desc->key_b].kind != 2) {
		return set_error(FLS_ERR_INVALID_ARG, "group keys must name PHT_2 probes");
	}
	ProbeGroupByOp op {};
	op.n_probes = desc->n_probes;
	// Small tables go to shared memory, first come first served.
	uint32_t       cta_words = 0;
	const uint32_t budget    = 48u * 1024u / 4u;
	for (uint32_t p = 0; p < desc->n_probes; ++p) {
		const fls_probe& pr = desc->probes[p];
		if (pr.col >= desc->n_cols || !pr.ht || pr.ht_len <= 0 || (pr.kind != 1 && pr.kind != 2)) {
			return set_error(FLS_ERR_INVALID_ARG, "bad probe");
		}
		if (pr.kind == 2 && (reinterpret_cast<uintptr_t>(pr.ht) & 7u)) {
			return set_error(FLS_ERR_ALIGNMENT, "PHT_2 tables must be 8-byte aligned");
		}
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
	op.key_a    = desc->key_a;
	op.key_b    = desc->key_b;
	op.mul      = desc->group_mul;
	op.sub      = desc->group_sub;
	op.n_groups = desc->n_groups;
	op.agg_col  = desc->agg_col;
	op.res      = d_res;
	StageCfg   cfg;
	uint32_t   grid, threads;
	size_t     smem;
	fls_status s = plan_stages(desc->cols, desc->n_cols, 0u, cta_words, cfg, grid, threads, smem);
	if (s != FLS_OK) { return s; }
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	s = cuda_check(cudaMemsetAsync(d_res, 0, sizeof(int32_t) * 4u * static_cast<size_t>(desc->n_groups), st),
	               "cudaMemsetAsync");
	if (s != FLS_OK) { return s; }
	return launch_staged(cfg, op, grid, threads, smem, st);
}

} // extern "C"
