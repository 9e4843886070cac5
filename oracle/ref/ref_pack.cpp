// TEST INFRASTRUCTURE ONLY: C entry points for the reference's host encoders.
#include <cstdint>
#include "fls_gen/pack/pack.hpp"
#include "fls_gen/transpose/transpose.hpp"
#include "fls_gen/unrsum/unrsum.hpp"
#include "ref_api.h"

extern "C" void ref_pack_u32(const uint32_t* in, uint32_t* out, unsigned bw) {
	generated::pack::fallback::scalar::pack(in, out, static_cast<uint8_t>(bw));
}
extern "C" void ref_pack_u8(const uint8_t* in, uint8_t* out, unsigned bw) {
	generated::pack::fallback::scalar::pack(in, out, static_cast<uint8_t>(bw));
}
extern "C" void ref_pack_u16(const uint16_t* in, uint16_t* out, unsigned bw) {
	generated::pack::fallback::scalar::pack(in, out, static_cast<uint8_t>(bw));
}
extern "C" void ref_pack_u64(const uint64_t* in, uint64_t* out, unsigned bw) {
	generated::pack::fallback::scalar::pack(in, out, static_cast<uint8_t>(bw));
}
extern "C" void ref_transpose_i_u32(const uint32_t* in, uint32_t* out) {
	generated::transpose::fallback::scalar::transpose_i(in, out);
}
extern "C" void ref_transpose_o_u32(const uint32_t* in, uint32_t* out) {
	generated::transpose::fallback::scalar::transpose_o(in, out);
}
extern "C" void ref_unrsum_u32(const uint32_t* in, uint32_t* out) {
	generated::unrsum::fallback::scalar::unrsum(in, out);
}
