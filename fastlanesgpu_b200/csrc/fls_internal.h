// fls_internal.h -- declarations shared by the host encoders, the C ABI layer
// and the CUDA kernels of libfls_gpu.so.  Not part of the public ABI.
#pragma once

#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/fls_gpu.h"

namespace fls {

// ---- error reporting (thread-local message behind fls_last_error) ----
fls_status set_error(fls_status st, const std::string& msg);
void       clear_error();

// ---- host format helpers (fls_host.cpp) ----
uint32_t transposed_pos(uint32_t j);
unsigned bit_width(uint32_t v);
void     transpose_i(const uint32_t* in, uint32_t* out);
void     untranspose(const uint32_t* in, uint32_t* out);
void     unrsum(const uint32_t* in, uint32_t* out);
void     pack(const uint32_t* in, uint32_t* out, unsigned bw);
uint32_t vec_payload_words(uint32_t scheme, uint32_t bw, uint32_t aux);
bool     encode_vector(const int32_t* in, uint32_t scheme, uint32_t layout, bool round4, uint32_t* out,
                       fls_vec_meta* m);
void     scheme_sizes(const int32_t* v, uint32_t* size5);
uint8_t  best_scheme(const uint32_t* size5);
void     vector_stats(const int32_t* v, float* f16);

// FLS_ERR_INVALID_ARG unless 0 < n <= FLS_MAX_VALUES (`who` names the caller).
fls_status check_n_values(uint64_t n, const char* who);

// Largest payload of one vector in words (DICT with 1024 distinct 32-bit values).
constexpr uint32_t kMaxVecWords = 32u * 10u + 1024u;

// Device error word bits (fls_kernels.cu).
enum : uint32_t {
	kErrBadMeta    = 1u << 0, // scheme / bit width out of range
	kErrBounds     = 1u << 1, // vector payload outside the data buffer
	kErrTimeout    = 1u << 2, // a bounded wait gave up
	kErrHash       = 1u << 3, // a probe hashed outside its table
	kErrCapacity   = 1u << 4, // staged vector larger than the staging slot
};

} // namespace fls
