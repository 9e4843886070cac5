// fls_pipeline.cuh -- the persistent staged-decode pipeline shared by every
// operator of the library, and the host-side planning helpers behind it.
//
// Execution model:
//   * persistent grid: ctas_per_sm CTAs per SM, W warps per CTA;
//   * the table is cut into tiles of k consecutive 1024-value vectors (k is
//     chosen so a tile is a few KB: 32 vectors at bit width 1, one vector for
//     a 4-column 46-bit row); warp w owns tiles w, w + total_warps, ...;
//   * each warp stages its next S tiles into private shared-memory slots, one
//     cp.async.bulk per column per tile, tracked by one mbarrier per stage, so
//     HBM reads run S tiles ahead of the decode;
//   * decode happens lane-parallel out of shared memory into registers
//     (fls_device.cuh); predicates become a 32-bit row mask per lane;
//     aggregates are warp-reduced and committed with one atomic per warp.
// Nothing spins without a bound, traps or reads outside a buffer: bad metadata
// or a timed-out wait sets a bit in the device error word and skips the tile.
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

constexpr uint32_t kMaxCols    = FLS_MAX_QUERY_COLS;
constexpr uint32_t kMaxTile    = 32;       // vectors per tile (one lane per vector at issue)
constexpr uint32_t kMaxWarps   = 16;       // warps per CTA (general kernels)
// Warps per CTA of the specialised join kernels unless the caller set a
// launch configuration: their launch bounds follow the shape, and joins whose
// tables leave room for more than 16 warps run faster with them (Q2.1: 0.230
// ms at 20, 0.210 ms at 24; the filter and decode kernels measured faster at
// 16).
constexpr uint32_t kJitDefaultWarps = 24;
// With half-vector stages (FLS_TUNE_HALF_VECTORS): 28 warps fit at the
// joins' 66-72 registers per thread.
constexpr uint32_t kJitHalfWarps = 28;
constexpr uint32_t kWaitPolls  = 1u << 17; // bounded mbarrier waits (x <= 20 us each)
constexpr uint32_t kDictWords  = 1024;     // per-warp dictionary scratch
constexpr uint32_t kTBufWords  = 33 * 32;  // per-warp transpose buffer
constexpr uint32_t kBadScheme  = 0xffu;

// ------------------------------------------------------------ parameters

struct StageCfg {
	DevCol    cols[kMaxCols];
	uint32_t  col_off[kMaxCols]; // word offset of column c's slot inside a stage
	uint32_t  n_cols;
	uint32_t  tile;            // k vectors per tile
	uint32_t  stage_words;     // words per stage (multiple of 4)
	uint32_t  stages;          // S
	uint32_t  warps;           // W
	uint32_t  warp_smem_words; // per-warp region (multiple of 4)
	uint32_t  dict_off;        // per-warp dictionary scratch (words)
	uint32_t  extra_off;       // per-warp operator scratch (words)
	uint32_t  info_off;        // per-warp vector info: uint4 per (stage, vector, column)
	uint32_t  bar_off;         // per-warp mbarriers (uint64 per stage)
	uint32_t  cta_extra_off;   // CTA-level scratch after all warp regions (words)
	uint64_t  n_vec, n_values, n_tiles;
	uint32_t  layout;
	uint32_t  has_dict;    // per-warp dictionary scratch planned (RLE / DICT allowed)
	uint32_t  all_uniform; // every column uniform (no metadata): host-validated, no per-vector info
	uint32_t* err;         // device error word
};

// Words of slack after the staged slots of a warp (single-row reads may look
// one word row past a vector's payload).
constexpr uint32_t kSlotSlackWords = 32;

__device__ __forceinline__ void raise_err(uint32_t* err, uint32_t bits) { atomicOr(err, bits); }

// ------------------------------------------------------- staged pipeline

// Per-warp view of its shared-memory region.  Vector info entries are
// {base, scheme | bw<<8 | aux<<16, word offset inside the column's slot, 0}.
struct WarpStage {
	uint32_t*       base;
	const StageCfg* cfg;
	__device__ uint32_t* slot(uint32_t st, uint32_t c) const { return base + st * cfg->stage_words + cfg->col_off[c]; }
	__device__ uint4*    info(uint32_t st, uint32_t i, uint32_t c) const {
        return reinterpret_cast<uint4*>(base + cfg->info_off) + (st * cfg->tile + i) * cfg->n_cols + c;
	}
	__device__ uint64_t* bar(uint32_t st) const { return reinterpret_cast<uint64_t*>(base + cfg->bar_off) + st; }
	__device__ uint32_t* dict() const { return base + cfg->dict_off; }
	__device__ uint32_t* extra() const { return base + cfg->extra_off; }
};

// Issues the bulk copies of tile t into stage st.  All lanes participate in
// one pass: lane l handles vector l / n_cols of the tile for column
// l % n_cols (the planner keeps tile * n_cols <= 32).  The lane holding a
// column's first vector issues one bulk copy covering the tile's payload range
// of that column, after adding its byte count to the stage barrier's
// transaction count; lane 0 arrives last.
struct LaneRole {
	uint32_t i, c;     // tile vector and column of this lane
	uint32_t col_mask; // lanes that work on column c
};

__device__ __forceinline__ LaneRole lane_role(const StageCfg& cfg, uint32_t lane) {
	LaneRole role;
	role.i        = lane / cfg.n_cols;
	role.c        = lane - role.i * cfg.n_cols;
	uint32_t m    = 0;
	for (uint32_t l = role.c; l < 32; l += cfg.n_cols) { m |= 1u << l; }
	role.col_mask = m;
	return role;
}

__device__ __forceinline__ void issue_stage(const StageCfg& cfg, const WarpStage& ws, uint32_t st, uint64_t t,
                                            uint32_t lane, const LaneRole& role, uint64_t pol) {
	const uint64_t v0     = t * cfg.tile;
	const uint32_t kk     = static_cast<uint32_t>(min(static_cast<uint64_t>(cfg.tile), cfg.n_vec - v0));
	if (cfg.all_uniform) {
		// Uniform columns: vector v sits at v * vec_words; the host checked that
		// the data buffer covers every vector.  Lane c copies column c.
		if (lane < cfg.n_cols) {
			const DevCol&  col   = cfg.cols[lane];
			const uint32_t bytes = kk * col.vec_words * 4u;
			if (bytes) {
				dev::mbar_expect_tx(ws.bar(st), bytes);
				dev::bulk_g2s(ws.slot(st, lane), col.data + v0 * col.vec_words, bytes, ws.bar(st), pol);
			}
		}
		__syncwarp();
		if (lane == 0) { dev::mbar_arrive(ws.bar(st)); }
		__syncwarp();
		return;
	}
	const uint32_t active = kk * cfg.n_cols; // lanes with a (vector, column) pair
	const bool     mine   = lane < active;
	const DevCol&  col    = cfg.cols[mine ? role.c : 0];
	VecInfo        vi {};
	bool           ok = true;
	if (mine) {
		const uint4 raw = dev::load_meta(col, v0 + role.i);
		ok              = dev::vec_info(col, v0 + role.i, raw, vi);
		// RLE / DICT vectors need the dictionary scratch; reject them otherwise.
		if (ok && !cfg.has_dict && (vi.scheme == FLS_SCHEME_RLE || vi.scheme == FLS_SCHEME_DICT)) { ok = false; }
	}
	// The column's payload range [start, end) over the tile.
	const uint32_t first_lane = role.c;
	const uint32_t last_lane  = (kk - 1u) * cfg.n_cols + role.c;
	const uint64_t start      = __shfl_sync(0xffffffffu, vi.offset, first_lane);
	const uint64_t end        = __shfl_sync(0xffffffffu, vi.offset + vi.words, last_lane);
	if (mine) { ok = ok && vi.offset >= start && vi.offset + vi.words <= end && end - start <= col.slot_words; }
	const uint32_t bad   = __ballot_sync(0xffffffffu, !ok);
	const bool     good  = (bad & role.col_mask & ((active >= 32u) ? 0xffffffffu : ((1u << active) - 1u))) == 0u;
	if (mine) {
		*ws.info(st, role.i, role.c) = good ? make_uint4(static_cast<uint32_t>(vi.base),
		                                                 vi.scheme | (vi.bw << 8) | (vi.aux << 16),
		                                                 static_cast<uint32_t>(vi.offset - start), 0u)
		                                    : make_uint4(0u, kBadScheme, 0u, 0u);
		if (role.i == 0) {
			if (!good) {
				raise_err(cfg.err, kErrBadMeta);
			} else if (end > start) {
				const uint32_t bytes = static_cast<uint32_t>(end - start) * 4u;
				dev::mbar_expect_tx(ws.bar(st), bytes);
				dev::bulk_g2s(ws.slot(st, role.c), col.data + start, bytes, ws.bar(st), pol);
			}
		}
	}
	__syncwarp();
	if (lane == 0) { dev::mbar_arrive(ws.bar(st)); }
	__syncwarp();
}

__device__ __forceinline__ VecInfo stage_info(const WarpStage& ws, uint32_t st, uint32_t i, uint32_t c,
                                              uint32_t& rel_off) {
	const uint4 x = *ws.info(st, i, c);
	VecInfo     vi;
	vi.offset = 0;
	vi.base   = static_cast<int32_t>(x.x);
	vi.scheme = x.y & 0xffu;
	vi.bw     = (x.y >> 8) & 0xffu;
	vi.aux    = x.y >> 16;
	vi.words  = 0;
	rel_off   = x.z;
	return vi;
}

// A staged vector of one column: its info and where its payload sits.
struct StagedVec {
	VecInfo         vi;
	const uint32_t* s;
	__device__ bool bad() const { return vi.scheme == kBadScheme; }
};

__device__ __forceinline__ StagedVec staged(const WarpStage& ws, uint32_t st, uint32_t i, uint32_t c) {
	StagedVec sv;
	if (ws.cfg->all_uniform) {
		const DevCol& col = ws.cfg->cols[c];
		sv.vi.offset      = 0;
		sv.vi.base        = col.base;
		sv.vi.scheme      = col.scheme;
		sv.vi.bw          = col.bw;
		sv.vi.aux         = 0;
		sv.vi.words       = col.vec_words;
		sv.s              = ws.slot(st, c) + i * col.vec_words;
		return sv;
	}
	uint32_t rel;
	sv.vi = stage_info(ws, st, i, c, rel);
	sv.s  = ws.slot(st, c) + rel;
	return sv;
}

__device__ __forceinline__ uint32_t valid_rows(const StageCfg& cfg, uint64_t v, uint32_t lane) {
	const uint64_t start = v * 1024u;
	if (start + 1024u <= cfg.n_values) { return 0xffffffffu; }
	return dev::tail_rows(cfg.layout, lane, static_cast<uint32_t>(cfg.n_values - start));
}

// The persistent staged loop.  Op provides
//   struct State                                                    (per-thread mutable state)
//   __device__ void cta_setup(State&, uint32_t* cta_smem, const StageCfg&) const   (all threads)
//   __device__ void process(State&, uint64_t v, const WarpStage&, uint32_t st, uint32_t i, uint32_t lane,
//                           const StageCfg&) const      (vector v = tile vector i in stage st)
//   __device__ void finish(State&, uint32_t lane, const StageCfg&) const
// The Op itself is a read-only kernel parameter.
template <class Op>
__global__ void __launch_bounds__(kMaxWarps * 32, 1)
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
	const LaneRole role = lane_role(cfg, lane);
	const uint64_t pol  = dev::l2_evict_first_policy();

	// Prologue: fill the pipeline.
	for (uint32_t s = 0; s < cfg.stages; ++s) {
		const uint64_t t = first + s * total;
		if (t >= cfg.n_tiles) { break; }
		issue_stage(cfg, ws, s, t, lane, role, pol);
	}
	uint64_t next_issue = first + static_cast<uint64_t>(cfg.stages) * total;

	uint32_t st = 0, phase = 0;
	for (uint64_t t = first; t < cfg.n_tiles; t += total) {
		if (!dev::mbar_wait_bounded(ws.bar(st), phase, kWaitPolls)) {
			raise_err(cfg.err, kErrTimeout);
			// Give the copies still in flight a bounded chance to land before exit.
			for (uint32_t s = 0; s < cfg.stages; ++s) {
				dev::mbar_wait_bounded(ws.bar(s), phase, 1u << 10);
				dev::mbar_wait_bounded(ws.bar(s), phase ^ 1u, 1u << 10);
			}
			return;
		}
		const uint64_t v0 = t * cfg.tile;
		const uint32_t kk = static_cast<uint32_t>(min(static_cast<uint64_t>(cfg.tile), cfg.n_vec - v0));
		for (uint32_t i = 0; i < kk; ++i) { op.process(state, v0 + i, ws, st, i, lane, cfg); }
		__syncwarp();
		if (next_issue < cfg.n_tiles) {
			dev::fence_proxy_async_smem();
			issue_stage(cfg, ws, st, next_issue, lane, role, pol);
			next_issue += total;
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
// Device address of the error word that kernels launched on `stream` record
// errors in: the word bound to the stream (fls_bind_error_word), else the
// device's default word.
uint32_t*  device_error_word(cudaStream_t stream);
void       count_launch(uint64_t n = 1);
int        tuning_sparse_rows();
int        tuning_jit();
int        tuning_group_smem();
int        tuning_late_measure();
int        tuning_half_vectors();
uint32_t   tuning_table_words(); // table budget in 4-byte words
uint32_t   jit_max_warps(); // most warps per CTA of the specialised join kernels

// Validates one column descriptor and converts it for a kernel.
fls_status make_devcol(const fls_column& c, DevCol& d);

// Query specialisation of filter-aggregate (fls_jit.cu).  A shape: the staged
// columns (filter columns in evaluation order, then aggregate-only columns),
// the aggregate columns' staged slots and the key naming the kernel.
struct JitShape {
	uint32_t    staged[FLS_MAX_QUERY_COLS];
	uint32_t    n_staged = 0;
	int         agg_a = -1, agg_b = -1;
	uint32_t    swar = 0; // filters tested several packed fields at a time
	std::string key;
};
// False when the query does not qualify (a non-FOR or non-uniform column,
// two ranges on one column, no column read).
bool jit_shape(const fls_column* cols, const fls_filter* filters, uint32_t n_filters, int32_t agg_a, int32_t agg_b,
               JitShape& sh);
// NVRTC compile of a shape as the current device (or, with none, a B200)
// would launch it (cached; no device needed).  False on failure.
bool jit_compile(const fls_column* cols, const JitShape& sh);
// Filter-aggregate through the specialised kernel (filters in evaluation
// order).  used = false, with FLS_OK, when the shape does not qualify or its
// specialisation is unavailable: run the general kernel then.
fls_status jit_filter_agg(const fls_column* cols, const fls_filter* filters, uint32_t n_filters, int32_t agg_a,
                          int32_t agg_b, int64_t* d_result, int32_t sparse_rows, cudaStream_t stream, bool& used);

// Probe + group-by shapes: staged columns (probe keys in probe order, then the
// measure column if no probe reads it), which tables live in shared memory.
constexpr uint32_t kJitTableKB    = 72u;  // default shared-memory budget for hash tables
constexpr uint32_t kJitMaxTableKB = 144u; // largest budget: 144 KB of tables + 24 KB of group slots
                                          // leave room for one warp of the widest staged row
constexpr uint32_t kJitGroupSlots = 2048u;            // most group-sum slots per CTA in shared memory
struct JitProbeShape {
	uint32_t    staged[FLS_MAX_QUERY_COLS];
	uint32_t    n_staged = 0;
	int         agg      = -1;
	int         sub      = -1; // staged column subtracted from the measure
	uint32_t    smem_off[FLS_MAX_PROBES];
	uint32_t    cta_words = 0;
	uint32_t    tables_words = 0;  // words of the tables (the presence bitmaps' buffer)
	uint32_t    bitmaps      = 0;  // probes whose presence bitmap is staged
	uint32_t    n_global     = 0;     // measure columns left in global memory (after the staged ones)
	bool        gsm          = false; // group sums in shared memory
	bool        half         = false; // half-vector tiles
	uint32_t    gslots       = 0;     // their slots (a power of two)
	uint32_t    gsum_off     = 0;     // their offset (words) in the CTA scratch
	std::string key;
};
// False when a staged column is not uniform FOR or one column is probed twice
// (the descriptor must already be validated).
bool       jit_probe_shape(const fls_join_groupby_desc* desc, JitProbeShape& sh);
bool       jit_compile(const fls_join_groupby_desc* desc, const JitProbeShape& sh);
// d_ws (optional, 16-byte aligned): room for the presence bitmaps, built
// once per call by a prepass; without it each CTA builds them.
fls_status jit_probe_groupby(const fls_join_groupby_desc* desc, int32_t* d_res, int32_t sparse_rows, void* d_ws,
                             uint64_t ws_bytes, cudaStream_t stream, bool& used);
// Bytes of workspace the specialised kernel of this query can use (0: none).
uint64_t jit_probe_workspace_bytes(const fls_join_groupby_desc* desc);
// Decode of a uniform FOR column: mode 0 = fused uint64 sum into d_sum, mode 1
// = to HBM (stored order) into d_out.
fls_status jit_decode(const fls_column* col, int mode, uint32_t* d_out, uint64_t* d_sum, cudaStream_t stream,
                      bool& used);

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
	StageCfg c = cfg;
	c.err      = device_error_word(stream);
	kern<<<grid, threads, smem, stream>>>(c, op);
	count_launch();
	return cuda_check(cudaGetLastError(), "staged kernel launch");
}

} // namespace fls
