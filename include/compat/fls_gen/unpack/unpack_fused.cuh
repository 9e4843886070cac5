/* fls_gen/unpack/unpack_fused.cuh under the reference's path
 * (fastlanes/src/include/fls_gen/unpack/unpack_fused.cuh): the register-form
 * decoder generated::unpack::cuda::fused::unpack(in, out, bw) and the global
 * unpack_device / load_registers / unpack_global, on fls_crystal.cuh's
 * decoders (every bit width 0..32). */
#pragma once
#include "../../../fls_crystal.cuh"

namespace generated { namespace unpack { namespace cuda { namespace fused {
__device__ __forceinline__ void unpack(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint8_t bw) {
	fls::crystal::detail::unpack_rows_dyn(in, out, bw);
}
#define FLS_COMPAT_FUSED(B)                                                                                            \
	__device__ __forceinline__ void unpack_##B##bw_32ow_32crw_1uf(const uint32_t* __restrict__ a_in_p,             \
	                                                               uint32_t* __restrict__ a_out_p) {                \
		fls::crystal::detail::unpack_rows_ptr<B>(a_in_p, a_out_p);                                                   \
	}
FLS_BW_CASES_0_32(FLS_COMPAT_FUSED)
#undef FLS_COMPAT_FUSED
}}}} // namespace generated::unpack::cuda::fused

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void load_registers(int i, T* out, T* registers) {
	fls::crystal::detail::load_registers<T, BLOCK_THREADS, ITEMS_PER_THREAD>(i, out, registers);
}

// One warp per vector: grid = number of vectors, 32 threads.
static __global__ void unpack_global(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint8_t bw) {
	in += (static_cast<uint64_t>(blockIdx.x) * bw) << 5;
	out += static_cast<uint64_t>(blockIdx.x) << 10;
	uint32_t registers[32];
	generated::unpack::cuda::fused::unpack(in, registers, bw);
	load_registers<uint32_t, 32, 32>(threadIdx.x, out, registers);
}

__device__ __forceinline__ void unpack_device(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint8_t bw) {
	generated::unpack::cuda::fused::unpack(in, out, bw);
}

__device__ __forceinline__ void unpack_device(const int32_t* __restrict__ in, int32_t* __restrict__ out, uint8_t bw) {
	fls::crystal::detail::unpack_rows_dyn(reinterpret_cast<const uint32_t*>(in), out, bw);
}
