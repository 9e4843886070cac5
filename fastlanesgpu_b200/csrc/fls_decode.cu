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
	DecodeSumOp op {};
	op.sum = reinterpret_cast<unsigned long long*>(d_sum);
	return launch_staged(cfg, op, grid, threads, smem, st);
}

} // extern "C"
