// TEST INFRASTRUCTURE ONLY.  The reference's delta decode + sum kernel
// (fastlanes/src/delta_shared_memory.cu, included where it lies, unchanged)
// compiled against this project's drop-in device headers (include/compat
// first on the include path): per 1024-value vector the normal-form
// unpack_device into shared memory, d_rsum_32 with the vector's 32 lane
// bases, BlockLoad and BlockSum (delta_shared_memory.cu:24-61).
#define main fls_ref_delta_main
#include "delta_shared_memory.cu"
#undef main

extern "C" {

// bases: 32 words per vector; packed: 32 * bw words per vector; *sum zeroed
// by the caller.
int dropin_delta_sum(const uint32_t* bases, const uint32_t* packed, uint64_t n_vec, uint32_t bw, uint64_t n_values,
                     unsigned long long* sum) {
	QueryMtd m {};
	m.n_vec = n_vec;
	m.bw    = static_cast<uint8_t>(bw);
	m.n_tup = n_values;
	QueryKernel<32, 32><<<static_cast<unsigned>(n_vec), 32>>>(bases, packed, m, sum);
	return static_cast<int>(cudaDeviceSynchronize());
}

int dropin_delta_take_error(uint32_t* bits) { return static_cast<int>(fls::crystal::fls_crystal_take_error(bits)); }

} // extern "C"
