// TEST INFRASTRUCTURE ONLY: reference normal unpack + rsum, run lane by lane.
#include "host_shim.h"
#define unpack_device  ref_normal_unpack_device
#define unpack_global  ref_normal_unpack_global
#include "fls_gen/unpack/unpack.cuh"
#include "fls_gen/rsum/rsum.cuh"
#include "ref_api.h"

extern "C" int ref_unpack_u32(const uint32_t* in, uint32_t* out, unsigned bw) {
	if (bw > 32) { return -1; }
	for (unsigned lane = 0; lane < 32; ++lane) {
		fls_shim_thread_idx.x = lane;
		generated::unpack::cuda::normal::unpack(in, out, static_cast<uint8_t>(bw));
	}
	return 0;
}

extern "C" void ref_rsum_u32(const uint32_t* in, uint32_t* out, const uint32_t* base) {
	for (unsigned lane = 0; lane < 32; ++lane) {
		fls_shim_thread_idx.x = lane;
		d_rsum_32(in, out, base);
	}
}
