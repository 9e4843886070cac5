// fls_batch.cu -- batched persistent execution of many filter-aggregate queries
// over many columns of uneven length and bit width in one launch.
//
// The host groups queries (filter lo <= x <= hi on one column, sum of another
// column of the same length) that read the same pair of columns, up to four
// per group, and cuts every group into work items of `chunk` consecutive
// vectors.  One persistent kernel runs all items: each warp pulls the next item
// from a global counter (dynamic load balancing across columns of very
// different lengths), streams the item's vectors through its own bulk-copy
// pipeline, decodes each vector once into registers, evaluates every query of
// the group on those values, and adds each query's sum and count into its
// result with one atomic each per item.  fls_batch_run only resets the counter
// and launches, so it can be captured into a CUDA graph and replayed.
//
// No reference counterpart: the reference launches one grid per query
// (fls_q11.cu:150-160).
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "fls_pipeline.cuh"

namespace fls {
// Queries sharing one (filter column, aggregated column) pair.
constexpr uint32_t kGroupQueries = 4;
struct BatchGroup {
	uint32_t col, agg_col, n_q, pad;
	uint32_t q[kGroupQueries];
};
} // namespace fls

struct fls_batch {
	std::vector<fls::DevCol>     cols;
	std::vector<fls_batch_query> queries;
	std::vector<fls::BatchGroup> groups;
	std::vector<uint4>           items; // {group, first vector, end vector, 0}
	uint32_t                     slot_words = 0;
	uint32_t                     has_dict   = 0;
	bool                         any_pair   = false; // some query aggregates another column than it filters
	void*                        ws         = nullptr; // device workspace after upload
	uint64_t                     ws_bytes   = 0;
};

namespace fls {
namespace {

constexpr uint32_t kBatchStages = 3;

struct BatchParams {
	const DevCol*          cols;
	const fls_batch_query* queries;
	const BatchGroup*      groups;
	const uint4*           items;
	uint32_t               n_items;
	uint32_t*              counter;
	long long*             results; // 2 per query: sum, count
	uint32_t               slot_words;
	uint32_t               n_slots; // staged columns per stage: 1 (filter = aggregate everywhere) or 2
	uint32_t               has_dict;
	uint32_t               warps;
	uint32_t*              err;
};

// Per warp shared memory: kBatchStages x {filter slot, aggregate slot},
// slack, dictionary scratch, stage infos and barriers.
struct BatchLayout {
	uint32_t slots, dict, info, bars, total;
	// n_slots = 1 when every query aggregates its own filter column.
	__host__ __device__ BatchLayout(uint32_t slot_words, uint32_t n_slots) {
		slots = 0;
		dict  = slots + kBatchStages * n_slots * slot_words + kSlotSlackWords;
		info  = dict + kDictWords;
		bars  = info + kBatchStages * 2u * 4u;
		total = (bars + 2u * kBatchStages + 3u) & ~3u;
	}
};

// Stages vector v of the filter column (slot 0) and, unless it is the same
// column, of the aggregated column (slot 1).
__device__ __forceinline__ bool batch_issue(const BatchParams& P, uint32_t* base, const BatchLayout& L, uint32_t st,
                                            const DevCol& cf, const DevCol& ca, bool same, uint64_t v, uint32_t lane,
                                            uint64_t pol) {
	uint4*    info = reinterpret_cast<uint4*>(base + L.info) + st * 2u;
	uint64_t* bar  = reinterpret_cast<uint64_t*>(base + L.bars) + st;
	bool      ok   = true;
	if (lane < (same ? 1u : 2u)) {
		const DevCol& c  = lane == 0 ? cf : ca;
		VecInfo       vi {};
		ok               = dev::vec_info(c, v, dev::load_meta(c, v), vi);
		if (ok && !P.has_dict && (vi.scheme == FLS_SCHEME_RLE || vi.scheme == FLS_SCHEME_DICT)) { ok = false; }
		info[lane] = ok ? make_uint4(static_cast<uint32_t>(vi.base), vi.scheme | (vi.bw << 8) | (vi.aux << 16), 0u, 0u)
		                : make_uint4(0u, kBadScheme, 0u, 0u);
		if (!ok) { raise_err(P.err, kErrBadMeta); }
		if (ok && vi.words) {
			dev::mbar_expect_tx(bar, vi.words * 4u);
			dev::bulk_g2s(base + L.slots + (st * P.n_slots + lane) * P.slot_words, c.data + vi.offset, vi.words * 4u,
			              bar, pol);
		}
	}
	__syncwarp();
	if (lane == 0) { dev::mbar_arrive(bar); }
	__syncwarp();
	return ok;
}

__global__ void __launch_bounds__(kMaxWarps * 32, 1) batch_kernel(const __grid_constant__ BatchParams P) {
	extern __shared__ __align__(128) uint32_t smem[];
	const uint32_t    lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	const BatchLayout L(P.slot_words, P.n_slots);
	uint32_t*         base = smem + warp * L.total;
	uint64_t*         bars = reinterpret_cast<uint64_t*>(base + L.bars);
	if (lane == 0) {
		for (uint32_t s = 0; s < kBatchStages; ++s) { dev::mbar_init(bars + s, 1); }
		dev::fence_mbar_init();
	}
	__syncwarp();
	const uint64_t pol   = dev::l2_evict_first_policy();
	uint32_t       phase = 0, st = 0; // running stage / phase across items
	for (;;) {
		uint32_t item = 0;
		if (lane == 0) { item = atomicAdd(P.counter, 1u); }
		item = __shfl_sync(0xffffffffu, item, 0);
		if (item >= P.n_items) { break; }
		const uint4       it = P.items[item];
		const BatchGroup  gr = P.groups[it.x];
		const DevCol&     cf = P.cols[gr.col];
		const DevCol&     ca = P.cols[gr.agg_col];
		const uint64_t    v0 = it.y, v1 = it.z;
		const bool        same = gr.col == gr.agg_col;
		const uint64_t    rows = P.queries[gr.q[0]].n_values;
		uint32_t          lo[kGroupQueries], range[kGroupQueries];
		bool              live[kGroupQueries];
#pragma unroll
		for (uint32_t j = 0; j < kGroupQueries; ++j) {
			const fls_batch_query& q = P.queries[gr.q[j < gr.n_q ? j : 0]];
			lo[j]    = static_cast<uint32_t>(q.lo);
			range[j] = static_cast<uint32_t>(q.hi) - lo[j];
			live[j]  = j < gr.n_q && q.lo <= q.hi;
		}
		// prologue
		uint32_t s_issue = st;
		for (uint32_t k = 0; k < kBatchStages && v0 + k < v1; ++k) {
			batch_issue(P, base, L, s_issue, cf, ca, same, v0 + k, lane, pol);
			s_issue = (s_issue + 1u == kBatchStages) ? 0u : s_issue + 1u;
		}
		long long          sum[kGroupQueries] = {0, 0, 0, 0};
		uint32_t           cnt[kGroupQueries] = {0, 0, 0, 0}; // at most 32 * chunk per lane
		for (uint64_t v = v0; v < v1; ++v) {
			if (!dev::mbar_wait_bounded(bars + st, phase, kWaitPolls)) {
				raise_err(P.err, kErrTimeout);
				for (uint32_t s = 0; s < kBatchStages; ++s) {
					dev::mbar_wait_bounded(bars + s, phase, 1u << 10);
					dev::mbar_wait_bounded(bars + s, phase ^ 1u, 1u << 10);
				}
				return;
			}
			const uint4* info = reinterpret_cast<const uint4*>(base + L.info) + st * 2u;
			const uint4  fi = info[0], ai = same ? info[0] : info[1];
			if ((fi.y & 0xffu) != kBadScheme && (ai.y & 0xffu) != kBadScheme) {
				VecInfo vf {}, va {};
				vf.base = static_cast<int32_t>(fi.x), vf.scheme = fi.y & 0xffu, vf.bw = (fi.y >> 8) & 0xffu;
				vf.aux  = fi.y >> 16;
				va.base = static_cast<int32_t>(ai.x), va.scheme = ai.y & 0xffu, va.bw = (ai.y >> 8) & 0xffu;
				va.aux  = ai.y >> 16;
				const uint32_t* sf = base + L.slots + (st * P.n_slots) * P.slot_words;
				const uint32_t* sa = same ? sf : sf + P.slot_words;
				// rows of a partial last vector
				uint32_t valid = 0xffffffffu;
				if ((v + 1) * 1024u > rows) {
					valid = dev::tail_rows(cf.layout, lane, static_cast<uint32_t>(rows - v * 1024u));
				}
				// Decode once; every query of the group reads the registers:
				// row masks first, then the sums (over the same values, or over
				// the aggregated column decoded row by row into the sums).
				uint32_t x[32];
				dev::decode_vals(sf, vf, base + L.dict, lane, x);
				long long p[kGroupQueries] = {0, 0, 0, 0};
				if (same && valid == 0xffffffffu) {
					// A whole vector whose sums are over the filtered values: each
					// query adds the rows in its range straight from the registers.
#pragma unroll
					for (uint32_t j = 0; j < kGroupQueries; ++j) {
						if (!live[j]) { continue; } // warp-uniform: one group per work item
						uint32_t c = 0;
#pragma unroll
						for (int r = 0; r < 32; ++r) {
							if (x[r] - lo[j] <= range[j]) {
								p[j] += static_cast<int32_t>(x[r]);
								++c;
							}
						}
						cnt[j] += c;
					}
				} else {
					uint32_t m[kGroupQueries];
#pragma unroll
					for (uint32_t j = 0; j < kGroupQueries; ++j) {
						uint32_t mj = 0;
#pragma unroll
						for (int r = 0; r < 32; ++r) { mj |= (x[r] - lo[j] <= range[j] ? 1u : 0u) << r; }
						m[j] = live[j] ? (mj & valid) : 0u;
						cnt[j] += static_cast<unsigned>(__popc(m[j]));
					}
					if (same) {
#pragma unroll
						for (int r = 0; r < 32; ++r) {
							const long long a = static_cast<int32_t>(x[r]);
#pragma unroll
							for (uint32_t j = 0; j < kGroupQueries; ++j) { p[j] += ((m[j] >> r) & 1u) ? a : 0ll; }
						}
					} else {
						dev::decode_each<true>(sa, va, base + L.dict, lane, [&](int r, uint32_t y) {
							const long long a = static_cast<int32_t>(y);
#pragma unroll
							for (uint32_t j = 0; j < kGroupQueries; ++j) { p[j] += ((m[j] >> r) & 1u) ? a : 0ll; }
						});
					}
				}
#pragma unroll
				for (uint32_t j = 0; j < kGroupQueries; ++j) { sum[j] += p[j]; }
			}
			__syncwarp();
			if (v + kBatchStages < v1) {
				dev::fence_proxy_async_smem();
				batch_issue(P, base, L, st, cf, ca, same, v + kBatchStages, lane, pol);
			}
			if (++st == kBatchStages) {
				st = 0;
				phase ^= 1u;
			}
		}
#pragma unroll
		for (uint32_t j = 0; j < kGroupQueries; ++j) {
			if (j >= gr.n_q) { break; }
			const unsigned long long s = warp_sum_u64(static_cast<unsigned long long>(sum[j]));
			const unsigned long long c = warp_sum_u64(cnt[j]);  // widened before the warp sum
			if (lane == 0) {
				if (s) { atomicAdd(reinterpret_cast<unsigned long long*>(P.results + 2u * gr.q[j]), s); }
				if (c) { atomicAdd(reinterpret_cast<unsigned long long*>(P.results + 2u * gr.q[j] + 1u), c); }
			}
		}
	}
}

size_t ws_align(size_t x) { return (x + 255u) & ~static_cast<size_t>(255u); }

struct WsLayout {
	size_t cols, queries, groups, items, counter, total;
	explicit WsLayout(const fls_batch& b) {
		cols    = 0;
		queries = cols + ws_align(b.cols.size() * sizeof(DevCol));
		groups  = queries + ws_align(b.queries.size() * sizeof(fls_batch_query));
		items   = groups + ws_align(b.groups.size() * sizeof(BatchGroup));
		counter = items + ws_align(b.items.size() * sizeof(uint4));
		total   = counter + 256;
	}
};

} // namespace

// Shared by fls_batch_run and its static-scratch variant.
fls_status batch_launch(const fls_batch* b, const DevCol* cols, const fls_batch_query* queries,
                        const BatchGroup* groups, const uint4* items, uint32_t* counter, int64_t* d_results,
                        cudaStream_t st) {
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	if ((s = cuda_check(cudaMemsetAsync(counter, 0, sizeof(uint32_t), st), "cudaMemsetAsync")) != FLS_OK) { return s; }
	if ((s = cuda_check(cudaMemsetAsync(d_results, 0, sizeof(int64_t) * 2u * b->queries.size(), st), "cudaMemsetAsync")) !=
	    FLS_OK) {
		return s;
	}
	if (b->items.empty()) { return FLS_OK; }
	uint32_t          warps, stages, ctas, tile;
	fls_get_launch_config(&warps, &stages, &ctas, &tile);
	const uint32_t    n_slots = b->any_pair ? 2u : 1u;
	const BatchLayout L(b->slot_words, n_slots);
	warps = std::min<uint32_t>(warps, static_cast<uint32_t>(di.max_smem) / (4u * L.total));
	if (warps == 0) {
		return set_error(FLS_ERR_CAPACITY, "batch vectors too large for shared-memory staging");
	}
	{
		static std::mutex mu;
		static uint64_t   configured = 0; // bit d: device d's shared-memory attribute raised
		int               dev        = 0;
		cudaGetDevice(&dev);
		std::lock_guard<std::mutex> lk(mu);
		if (dev >= 64 || !(configured & (1ull << dev))) {
			if ((s = cuda_check(cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, di.max_smem),
			                    "cudaFuncSetAttribute")) != FLS_OK) {
				return s;
			}
			if (dev < 64) { configured |= 1ull << dev; }
		}
	}
	BatchParams P;
	P.cols       = cols;
	P.queries    = queries;
	P.groups     = groups;
	P.items      = items;
	P.n_items    = static_cast<uint32_t>(b->items.size());
	P.counter    = counter;
	P.results    = reinterpret_cast<long long*>(d_results);
	P.slot_words = b->slot_words;
	P.n_slots    = n_slots;
	P.has_dict   = b->has_dict;
	// Every SM gets warps: fewer work items than SMs x warps take fewer warps
	// per CTA, not fewer CTAs (the items are pulled from one counter).
	const uint64_t n_items = b->items.size();
	uint64_t       grid64  = std::min<uint64_t>((n_items + warps - 1) / warps, static_cast<uint64_t>(di.sms) * ctas);
	if (grid64 < static_cast<uint64_t>(di.sms)) {
		grid64 = std::min<uint64_t>(n_items, static_cast<uint64_t>(di.sms));
		warps  = static_cast<uint32_t>((n_items + grid64 - 1) / grid64);
	}
	const uint32_t grid = static_cast<uint32_t>(grid64);
	P.warps      = warps;
	P.err        = device_error_word(st);
	batch_kernel<<<grid, 32u * warps, 4ull * L.total * warps, st>>>(P);
	count_launch();
	return cuda_check(cudaGetLastError(), "batch_kernel launch");
}

} // namespace fls

using namespace fls;

extern "C" {

fls_status fls_batch_create(const fls_column* cols, uint32_t n_cols, const fls_batch_query* queries,
                            uint32_t n_queries, uint32_t chunk_vectors, fls_batch** out) {
	if (!cols || !queries || !out || n_cols == 0 || chunk_vectors == 0 || chunk_vectors > (1u << 20)) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_batch_create: bad arguments (chunk_vectors in [1, 2^20])");
	}
	fls_batch* b = new (std::nothrow) fls_batch;
	if (!b) { return set_error(FLS_ERR_CAPACITY, "out of host memory"); }
	b->cols.resize(n_cols);
	uint32_t slot = 0;
	for (uint32_t c = 0; c < n_cols; ++c) {
		fls_status s = make_devcol(cols[c], b->cols[c]);
		if (s != FLS_OK) {
			delete b;
			return s;
		}
		slot = std::max(slot, b->cols[c].slot_words);
		if (cols[c].meta && (cols[c].scheme_mask & ((1u << FLS_SCHEME_RLE) | (1u << FLS_SCHEME_DICT)))) {
			b->has_dict = 1u;
		}
	}
	b->slot_words = (slot + 3u) & ~3u;
	b->queries.assign(queries, queries + n_queries);
	std::vector<int64_t> open_group(static_cast<size_t>(n_cols) * n_cols, -1); // (col, agg) -> group being filled
	for (uint32_t q = 0; q < n_queries; ++q) {
		fls_batch_query& bq = b->queries[q];
		if (bq.col >= n_cols || bq.agg_col >= n_cols || cols[bq.col].n_values != cols[bq.agg_col].n_values ||
		    cols[bq.col].layout != cols[bq.agg_col].layout) {
			delete b;
			return set_error(FLS_ERR_INVALID_ARG, "batch query names missing or mismatched columns");
		}
		bq.n_values    = cols[bq.col].n_values;
		b->any_pair    = b->any_pair || bq.col != bq.agg_col;
		int64_t& slot_g = open_group[static_cast<size_t>(bq.col) * n_cols + bq.agg_col];
		if (slot_g < 0 || b->groups[static_cast<size_t>(slot_g)].n_q == kGroupQueries) {
			slot_g = static_cast<int64_t>(b->groups.size());
			b->groups.push_back(BatchGroup {bq.col, bq.agg_col, 0u, 0u, {0u, 0u, 0u, 0u}});
		}
		BatchGroup& g    = b->groups[static_cast<size_t>(slot_g)];
		g.q[g.n_q++] = q;
	}
	for (uint32_t gi = 0; gi < b->groups.size(); ++gi) {
		const uint64_t n_vec = (cols[b->groups[gi].col].n_values + 1023u) / 1024u;
		for (uint64_t v = 0; v < n_vec; v += chunk_vectors) {
			b->items.push_back(make_uint4(gi, static_cast<uint32_t>(v),
			                              static_cast<uint32_t>(std::min<uint64_t>(n_vec, v + chunk_vectors)), 0u));
		}
	}
	*out = b;
	return FLS_OK;
}

uint64_t fls_batch_workspace_bytes(const fls_batch* b) { return b ? WsLayout(*b).total : 0; }

uint32_t fls_batch_items(const fls_batch* b) { return b ? static_cast<uint32_t>(b->items.size()) : 0u; }

fls_status fls_batch_upload(fls_batch* b, void* d_workspace, uint64_t workspace_bytes, fls_stream_t stream) {
	if (!b || !d_workspace) { return set_error(FLS_ERR_INVALID_ARG, "fls_batch_upload: bad arguments"); }
	const WsLayout L(*b);
	if (workspace_bytes < L.total) { return set_error(FLS_ERR_CAPACITY, "batch workspace too small"); }
	char*        w  = static_cast<char*>(d_workspace);
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	fls_status   s  = cuda_check(cudaMemcpyAsync(w + L.cols, b->cols.data(), b->cols.size() * sizeof(DevCol),
	                                             cudaMemcpyHostToDevice, st), "upload columns");
	if (s == FLS_OK) {
		s = cuda_check(cudaMemcpyAsync(w + L.queries, b->queries.data(), b->queries.size() * sizeof(fls_batch_query),
		                               cudaMemcpyHostToDevice, st), "upload queries");
	}
	if (s == FLS_OK && !b->groups.empty()) {
		s = cuda_check(cudaMemcpyAsync(w + L.groups, b->groups.data(), b->groups.size() * sizeof(BatchGroup),
		                               cudaMemcpyHostToDevice, st), "upload groups");
	}
	if (s == FLS_OK && !b->items.empty()) {
		s = cuda_check(cudaMemcpyAsync(w + L.items, b->items.data(), b->items.size() * sizeof(uint4),
		                               cudaMemcpyHostToDevice, st), "upload items");
	}
	if (s == FLS_OK) { s = cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize"); }
	if (s == FLS_OK) {
		b->ws       = d_workspace;
		b->ws_bytes = workspace_bytes;
	}
	return s;
}

fls_status fls_batch_run(const fls_batch* b, int64_t* d_results, fls_stream_t stream) {
	if (!b || !d_results || !b->ws) { return set_error(FLS_ERR_INVALID_ARG, "fls_batch_run: not uploaded"); }
	const WsLayout L(*b);
	char*          w = static_cast<char*>(b->ws);
	return batch_launch(b, reinterpret_cast<const DevCol*>(w + L.cols),
	                    reinterpret_cast<const fls_batch_query*>(w + L.queries),
	                    reinterpret_cast<const BatchGroup*>(w + L.groups), reinterpret_cast<const uint4*>(w + L.items),
	                    reinterpret_cast<uint32_t*>(w + L.counter), d_results, reinterpret_cast<cudaStream_t>(stream));
}

void fls_batch_destroy(fls_batch* b) { delete b; }

} // extern "C"
