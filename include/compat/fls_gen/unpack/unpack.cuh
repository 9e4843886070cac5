/* fls_gen/unpack/unpack.cuh under the reference's path
 * (fastlanes/src/include/fls_gen/unpack/unpack.cuh): the normal-form decoder
 * generated::unpack::cuda::normal::unpack(in, out, bw) -- the warp writes the
 * vector, lane l storing row r at out[l + 32r] -- and the global
 * unpack_device / unpack_global, on fls_crystal.cuh's decoders (every bit
 * width 0..32). */
#pragma once
#include "../../../fls_crystal.cuh"

namespace generated { namespace unpack { namespace cuda { namespace normal {
__device__ __forceinline__ void unpack(const uint32_t* in, uint32_t* out, uint8_t bw) {
	fls::crystal::detail::unpack_strided_dyn(in, out, bw);
}
#define FLS_COMPAT_NORMAL(B)                                                                                           \
	__device__ __forceinline__ void unpack_##B##bw_32ow_32crw_1uf(const uint32_t* __restrict__ a_in_p,             \
	                                                               uint32_t* __restrict__ a_out_p) {                \
		fls::crystal::detail::unpack_strided_ptr<B>(a_in_p, a_out_p);                                                \
	}
FLS_BW_CASES_0_32(FLS_COMPAT_NORMAL)
#undef FLS_COMPAT_NORMAL
}}}} // namespace generated::unpack::cuda::normal

// One warp per vector: grid = number of vectors, 32 threads.
static __global__ void unpack_global(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint8_t bw) {
	in += (static_cast<uint64_t>(blockIdx.x) * bw) << 5;
	out += static_cast<uint64_t>(blockIdx.x) << 10;
	generated::unpack::cuda::normal::unpack(in, out, bw);
}

__device__ __forceinline__ void unpack_device(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint8_t bw) {
	generated::unpack::cuda::normal::unpack(in, out, bw);
}

__device__ __forceinline__ void unpack_device(const int32_t* __restrict__ in, int32_t* __restrict__ out, uint8_t bw) {
	fls::crystal::detail::unpack_strided_dyn(reinterpret_cast<const uint32_t*>(in), out, bw);
}
