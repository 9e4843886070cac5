// TEST INFRASTRUCTURE ONLY: reference specialised decoders, run lane by lane.
#include "host_shim.h"
#define unpack_device  ref_h16_unpack_device
#define unpack_global  ref_h16_unpack_global
#define load_registers ref_h16_load_registers
#include "fls_gen/unpack/hardcoded_16.cuh"
#include "ref_api.h"

extern "C" int ref_unpack8_u32(const uint32_t* in_quarter, uint32_t* out256, unsigned bw) {
	switch (bw) {
	case 0: case 4: case 8: case 12: case 16: case 20: break;
	default: return -1;
	}
	uint32_t regs[8];
	for (unsigned lane = 0; lane < 32; ++lane) {
		fls_shim_thread_idx.x = lane;
		unpack_8_at_a_time::unpack(in_quarter, regs, static_cast<uint8_t>(bw));
		for (unsigned r = 0; r < 8; ++r) { out256[32 * r + lane] = regs[r]; }
	}
	return 0;
}

extern "C" int ref_unpack_h16(const uint32_t* in, uint16_t* out, unsigned bw) {
	switch (bw) {
	case 4: case 6: case 16: case 24: break;
	default: return -1;
	}
	uint16_t regs[32];
	for (unsigned lane = 0; lane < 32; ++lane) {
		fls_shim_thread_idx.x = lane;
		hardcoded_16::unpack(in, regs, static_cast<uint8_t>(bw));
		for (unsigned r = 0; r < 32; ++r) { out[32 * r + lane] = regs[r]; }
	}
	return 0;
}
