// fls_pipeline.cuh -- the persistent staged-decode pipeline shared by every
// operator of the library, and the host-side planning helpers behind it.
//
// Execution model:
//   * persistent grid: ctas_per_sm CTAs per SM, W warps per CTA;
//   * each warp owns vectors w, w + total_warps, ... of the table;
//   * each warp stages its next S vectors (all referenced columns of one vector
//     form one stage) into private shared-memory slots with cp.async.bulk,
//     tracked by one mbarrier per stage, so HBM reads run S vectors ahead of
//     the decode;
//   * decode happens lane-parallel out of shared memory into registers
//     (fls_device.cuh); predicates become a 32-bit row mask per lane;
//     aggregates are warp-reduced and committed with one atomic per warp.
// Nothing spins without a bound, traps or reads outside a buffer: bad metadata
// or a timed-out wait sets a bit in the device error word and skips the vector.
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "fls_device.cuh"
#include "fls_internal.h"

namespace fls {

using dev::DevCol;
using dev::VecInfo;

constexpr uint32_t kMaxCols   = FLS_MAX_QUERY_COLS;
constexpr uint32_t kWaitPolls = 1u << 22; // bounded mbarrier waits
constexpr uint32_t kDictWords = 1024;     // per-warp dictionary scratch
constexpr uint32_t kTBufWords = 33 * 32;  // per-warp transpose buffer
constexpr uint32_t kBadScheme = 0xffu;

// ------------------------------------------------------------ parameters

struct StageCfg {
	DevCol    cols[kMaxCols];
	uint32_t  col_off[kMaxCols]; // word offset of column c's slot inside a stage
	uint32_t  n_cols;
	uint32_t  stage_words;     // words per stage (multiple of 4)
	uint32_t  stages;          // S
	uint32_t  warps;           // W
	uint32_t  warp_smem_words; // per-warp region (multiple of 4)
	uint32_t  dict_off;        // per-warp dictionary scratch (words)
	uint32_t  extra_off;       // per-warp kernel-specific scratch (words)
	uint32_t  info_off;        // per-warp stage info (uint2 per stage per column)
	uint32_t  bar_off;         // per-warp mbarriers (uint64 per stage)
	uint32_t  cta_extra_off;   // CTA-level scratch after all warp regions (words)
	uint64_t  n_vec, n_values;
	uint32_t  layout;
	uint32_t  has_dict; // per-warp dictionary scratch planned (RLE / DICT allowed)
	uint32_t* err;      // device error word
};

__device__ __forceinline__ void raise_err(uint32_t* err, uint32_t bits) { atomicOr(err, bits); }

// ------------------------------------------------------- staged pipeline

// Per-warp view of its shared-memory region.
struct WarpStage {
	uint32_t*       base;
	const StageCfg* cfg;
	__device__ uint32_t* slot(uint32_t st, uint32_t c) const { return base + st * cfg->stage_words + cfg->col_off[c]; }
	__device__ uint2*    info(uint32_t st) const { return reinterpret_cast<uint2*>(base + cfg->info_off) + st * kMaxCols; }
	__device__ uint64_t* bar(uint32_t st) const { return reinterpret_cast<uint64_t*>(base + cfg->bar_off) + st; }
	__device__ uint32_t* dict() const { return base + cfg->dict_off; }
	__device__ uint32_t* extra() const { return base + cfg->extra_off; }
};

// Issues the bulk copies of vector v into stage st.  All lanes participate:
// lane c handles column c; `raw` is lane c's metadata entry for v.
__device__ __forceinline__ void issue_stage(const StageCfg& cfg, const WarpStage& ws, uint32_t st, uint64_t v,
                                            uint4 raw, uint32_t lane) {
	uint32_t bytes = 0;
	VecInfo  vi {};
	bool     ok = true;
	if (lane < cfg.n_cols) {
		ok = dev::vec_info(cfg.cols[lane], v, raw, vi);
		// RLE / DICT vectors need the dictionary scratch; reject them otherwise.
		if (ok && !cfg.has_dict && (vi.scheme == FLS_SCHEME_RLE || vi.scheme == FLS_SCHEME_DICT)) { ok = false; }
		uint2 x;
		if (ok) {
			bytes = vi.words * 4u;
			x     = make_uint2(static_cast<uint32_t>(vi.base), vi.scheme | (vi.bw << 8) | (vi.aux << 16));
		} else {
			x = make_uint2(0u, kBadScheme);
			raise_err(cfg.err, kErrBadMeta);
		}
		ws.info(st)[lane] = x;
	}
	const uint32_t total = __reduce_add_sync(0xffffffffu, bytes);
	if (lane == 0) { dev::mbar_arrive_expect_tx(ws.bar(st), total); }
	__syncwarp();
	if (lane < cfg.n_cols && ok && bytes) {
		dev::bulk_g2s(ws.slot(st, lane), cfg.cols[lane].data + vi.offset, bytes, ws.bar(st));
	}
}

__device__ __forceinline__ VecInfo stage_info(const WarpStage& ws, uint32_t st, uint32_t c) {
	const uint2 x = ws.info(st)[c];
	VecInfo     vi;
	vi.offset = 0;
	vi.base   = static_cast<int32_t>(x.x);
	vi.scheme = x.y & 0xffu;
	vi.bw     = (x.y >> 8) & 0xffu;
	vi.aux    = x.y >> 16;
	vi.words  = 0;
	return vi;
}

// Decodes column c of the staged vector in stage st into vals; false if the
// vector's metadata was rejected at issue time.
__device__ __forceinline__ bool stage_decode(const WarpStage& ws, uint32_t st, uint32_t c, uint32_t lane,
                                             uint32_t (&vals)[32]) {
	const VecInfo vi = stage_info(ws, st, c);
	if (vi.scheme == kBadScheme) { return false; }
	dev::decode_vals(ws.slot(st, c), vi, ws.dict(), lane, vals);
	return true;
}

__device__ __forceinline__ uint32_t valid_rows(const StageCfg& cfg, uint64_t v, uint32_t lane) {
	const uint64_t start = v * 1024u;
	if (start + 1024u <= cfg.n_values) { return 0xffffffffu; }
	return dev::tail_rows(cfg.layout, lane, static_cast<uint32_t>(cfg.n_values - start));
}

// The persistent staged loop.  Op provides
//   struct State                                                    (per-thread mutable state)
//   __device__ void cta_setup(State&, uint32_t* cta_smem, const StageCfg&) const   (all threads)
//   __device__ void process(State&, uint64_t v, const WarpStage&, uint32_t st, uint32_t lane,
//                           const StageCfg&) const
//   __device__ void finish(State&, uint32_t lane, const StageCfg&) const
// The Op itself is a read-only kernel parameter.
template <class Op>
__global__ void __launch_bounds__(256, 1)
    staged_kernel(const __grid_constant__ StageCfg cfg, const __grid_constant__ Op op) {
	extern __shared__ __align__(128) uint32_t smem[];
	const uint32_t     lane = threadIdx.x & 31u;
	const uint32_t     warp = threadIdx.x >> 5;
	typename Op::State state {};
	op.cta_setup(state, smem + cfg.cta_extra_off, cfg);
	__syncthreads();

	WarpStage      ws {smem + warp * cfg.warp_smem_words, &cfg};
	const uint64_t total = static_cast<uint64_t>(gridDim.x) * cfg.warps;
	const uint64_t first = static_cast<uint64_t>(blockIdx.x) * cfg.warps + warp;

	if (lane == 0) {
		for (uint32_t s = 0; s < cfg.stages; ++s) { dev::mbar_init(ws.bar(s), 1); }
		dev::fence_mbar_init();
	}
	__syncwarp();

	// Prologue: fill the pipeline.
	for (uint32_t s = 0; s < cfg.stages; ++s) {
		const uint64_t v = first + s * total;
		if (v >= cfg.n_vec) { break; }
		const uint4 raw = lane < cfg.n_cols ? dev::load_meta(cfg.cols[lane], v) : make_uint4(0, 0, 0, 0);
		issue_stage(cfg, ws, s, v, raw, lane);
	}
	// Metadata of the next vector to issue, fetched one iteration early.
	uint64_t next_issue = first + static_cast<uint64_t>(cfg.stages) * total;
	uint4    next_raw   = (lane < cfg.n_cols && next_issue < cfg.n_vec) ? dev::load_meta(cfg.cols[lane], next_issue)
	                                                                   : make_uint4(0, 0, 0, 0);

	uint32_t st = 0, phase = 0;
	for (uint64_t v = first; v < cfg.n_vec; v += total) {
		if (!dev::mbar_wait_bounded(ws.bar(st), phase, kWaitPolls)) {
			raise_err(cfg.err, kErrTimeout);
			// Give the copies still in flight a bounded chance to land before exit.
			for (uint32_t s = 0; s < cfg.stages; ++s) {
				dev::mbar_wait_bounded(ws.bar(s), phase, 1u << 10);
				dev::mbar_wait_bounded(ws.bar(s), phase ^ 1u, 1u << 10);
			}
			return;
		}
		op.process(state, v, ws, st, lane, cfg);
		__syncwarp();
		if (next_issue < cfg.n_vec) {
			dev::fence_proxy_async_smem();
			issue_stage(cfg, ws, st, next_issue, next_raw, lane);
			next_issue += total;
			next_raw = (lane < cfg.n_cols && next_issue < cfg.n_vec) ? dev::load_meta(cfg.cols[lane], next_issue)
			                                                         : make_uint4(0, 0, 0, 0);
		}
		if (++st == cfg.stages) {
			st = 0;
			phase ^= 1u;
		}
	}
	op.finish(state, lane, cfg);
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) { x += __shfl_xor_sync(0xffffffffu, x, o); }
	return x;
}

// ------------------------------------------------------------ host side

struct DeviceInfo {
	int sms = 0, max_smem = 0, major = 0;
};

fls_status device_info(DeviceInfo& di);
fls_status cuda_check(cudaError_t e, const char* what);
uint32_t*  device_error_word(); // device address of this device's error word
void       count_launch(uint64_t n = 1);

// Lays out shared memory for a set of columns; extra_words per warp and
// cta_words per CTA are operator-specific scratch.
fls_status plan_stages(const fls_column* cols, uint32_t n_cols, uint32_t extra_words, uint32_t cta_words,
                       StageCfg& cfg, uint32_t& grid, uint32_t& threads, size_t& smem_bytes);

template <class Op>
fls_status launch_staged(const StageCfg& cfg, const Op& op, uint32_t grid, uint32_t threads, size_t smem,
                         cudaStream_t stream) {
	DeviceInfo di;
	fls_status ds = device_info(di);
	if (ds != FLS_OK) { return ds; }
	static std::mutex mu;
	static uint64_t   configured = 0; // bit d set once device d's smem attribute is raised
	auto              kern       = staged_kernel<Op>;
	int               dev        = 0;
	cudaGetDevice(&dev);
	{
		std::lock_guard<std::mutex> lk(mu);
		if (dev >= 64 || !(configured & (1ull << dev))) {
			fls_status s = cuda_check(
			    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, di.max_smem), "cudaFuncSetAttribute");
			if (s != FLS_OK) { return s; }
			if (dev < 64) { configured |= 1ull << dev; }
		}
	}
	if (grid == 0) { return FLS_OK; }
	kern<<<grid, threads, smem, stream>>>(cfg, op);
	count_launch();
	return cuda_check(cudaGetLastError(), "staged kernel launch");
}

} // namespace fls
