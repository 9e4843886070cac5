// TEST INFRASTRUCTURE ONLY: reference register-form unpack, run lane by lane.
#include "host_shim.h"
#define unpack_device  ref_fused_unpack_device
#define unpack_global  ref_fused_unpack_global
#define load_registers ref_fused_load_registers
#include "fls_gen/unpack/unpack_fused.cuh"
#include "ref_api.h"

extern "C" int ref_unpack_fused_u32(const uint32_t* in, uint32_t* out, unsigned bw) {
	if (bw > 32) { return -1; }
	uint32_t regs[32];
	for (unsigned lane = 0; lane < 32; ++lane) {
		fls_shim_thread_idx.x = lane;
		generated::unpack::cuda::fused::unpack(in, regs, static_cast<uint8_t>(bw));
		for (unsigned r = 0; r < 32; ++r) { out[32 * r + lane] = regs[r]; }
	}
	return 0;
}
