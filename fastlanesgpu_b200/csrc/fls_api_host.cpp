// fls_api_host.cpp -- C ABI of the host-side encoders (include/fls_gpu.h).
#include <omp.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "fls_internal.h"

namespace fls {
namespace {
thread_local std::string t_last_error;

// Copies vector v of a column into a full 1024-value buffer, padding a partial
// last vector with its last value (keeps the range and the runs unchanged).
void load_vector(const int32_t* values, uint64_t n, uint64_t v, int32_t* buf) {
	const uint64_t start = v * 1024u;
	const uint64_t cnt   = std::min<uint64_t>(1024u, n - start);
	std::memcpy(buf, values + start, sizeof(int32_t) * cnt);
	for (uint64_t j = cnt; j < 1024u; ++j) { buf[j] = buf[cnt - 1]; }
}

int resolve_threads(int n_threads) { return n_threads > 0 ? n_threads : omp_get_max_threads(); }
} // namespace

fls_status set_error(fls_status st, const std::string& msg) {
	t_last_error = msg;
	return st;
}
void clear_error() { t_last_error.clear(); }

fls_status check_n_values(uint64_t n, const char* who) {
	if (n == 0 || n > FLS_MAX_VALUES) {
		return set_error(FLS_ERR_INVALID_ARG, std::string(who) + ": the value count must be in 1..FLS_MAX_VALUES (2^40)");
	}
	return FLS_OK;
}

} // namespace fls

using namespace fls;

extern "C" {

const char* fls_last_error(void) { return t_last_error.c_str(); }

fls_status fls_pack_u32(const uint32_t* in, uint32_t* out, uint8_t bw) {
	if (!in || (!out && bw)) { return set_error(FLS_ERR_INVALID_ARG, "fls_pack_u32: null pointer"); }
	if (bw > 32) { return set_error(FLS_ERR_BAD_BW, "fls_pack_u32: bit width > 32"); }
	pack(in, out, bw);
	return FLS_OK;
}

fls_status fls_transpose_i_u32(const uint32_t* in, uint32_t* out) {
	if (!in || !out) { return set_error(FLS_ERR_INVALID_ARG, "fls_transpose_i_u32: null pointer"); }
	transpose_i(in, out);
	return FLS_OK;
}

fls_status fls_untranspose_u32(const uint32_t* in, uint32_t* out) {
	if (!in || !out) { return set_error(FLS_ERR_INVALID_ARG, "fls_untranspose_u32: null pointer"); }
	untranspose(in, out);
	return FLS_OK;
}

fls_status fls_unrsum_u32(const uint32_t* in, uint32_t* out) {
	if (!in || !out) { return set_error(FLS_ERR_INVALID_ARG, "fls_unrsum_u32: null pointer"); }
	unrsum(in, out);
	return FLS_OK;
}

fls_status fls_vector_rle(const int32_t* vec, uint8_t* idx, int32_t* dict, uint16_t* dict4, uint32_t* n_dict) {
	if (!vec || !idx || !dict || !dict4 || !n_dict) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_vector_rle: null pointer");
	}
	// rle.hpp:8-41: per 256-value mini-vector a local run index (uint8) and a
	// dictionary of run values; dict4[m] is where mini-vector m's entries start.
	uint32_t n = 0;
	for (uint32_t m = 0; m < 4; ++m) {
		dict4[m]      = static_cast<uint16_t>(n);
		uint32_t local = 0;
		for (uint32_t i = 0; i < 256; ++i) {
			const uint32_t j = 256u * m + i;
			if (i == 0) {
				dict[n++] = vec[j];
			} else if (vec[j] != vec[j - 1]) {
				dict[n++] = vec[j];
				++local;
			}
			idx[j] = static_cast<uint8_t>(local);
		}
	}
	*n_dict = n;
	return FLS_OK;
}

uint64_t fls_encode_bound_words(uint64_t n_values) {
	const uint64_t n_vec = (n_values + 1023u) / 1024u;
	return n_vec * kMaxVecWords;
}

fls_status fls_encode_uniform(const int32_t* values, uint64_t n, uint32_t scheme, uint32_t layout, uint8_t bw,
                              int32_t base, uint32_t* out, uint64_t* out_words, uint8_t* out_bw) {
	if (!values || !out || !out_words || n == 0) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_encode_uniform: null pointer or n == 0");
	}
	if (scheme != FLS_SCHEME_FOR && scheme != FLS_SCHEME_DELTA) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_encode_uniform: scheme must be FOR or DELTA");
	}
	if (layout > FLS_LAYOUT_TRANSPOSED) { return set_error(FLS_ERR_INVALID_ARG, "fls_encode_uniform: bad layout"); }
	if (bw > 32 && bw != 0xff) { return set_error(FLS_ERR_BAD_BW, "fls_encode_uniform: bit width > 32"); }
	const uint64_t n_vec = (n + 1023u) / 1024u;
	// Bit width that fits every vector (FOR: values - base; DELTA: deltas).
	unsigned need = 0;
#pragma omp parallel for reduction(max : need) schedule(static)
	for (int64_t v = 0; v < static_cast<int64_t>(n_vec); ++v) {
		int32_t  buf[1024];
		uint32_t tr[1024], d[1024];
		load_vector(values, n, static_cast<uint64_t>(v), buf);
		if (scheme == FLS_SCHEME_FOR) {
			for (uint32_t j = 0; j < 1024; ++j) {
				need = std::max(need, bit_width(static_cast<uint32_t>(buf[j]) - static_cast<uint32_t>(base)));
			}
		} else {
			transpose_i(reinterpret_cast<const uint32_t*>(buf), tr);
			unrsum(tr, d);
			for (uint32_t j = 0; j < 1024; ++j) { need = std::max(need, bit_width(d[j])); }
		}
	}
	const unsigned use = (bw == 0xff) ? need : bw;
	if (use < need) { return set_error(FLS_ERR_BAD_BW, "fls_encode_uniform: values do not fit the bit width"); }
	const uint64_t stride = (scheme == FLS_SCHEME_FOR) ? 32u * use : 32u + 32u * use;
#pragma omp parallel for schedule(static)
	for (int64_t v = 0; v < static_cast<int64_t>(n_vec); ++v) {
		int32_t   buf[1024];
		uint32_t  tmp[1024], tr[1024];
		uint32_t* dst = out + static_cast<uint64_t>(v) * stride;
		load_vector(values, n, static_cast<uint64_t>(v), buf);
		if (scheme == FLS_SCHEME_FOR) {
			for (uint32_t j = 0; j < 1024; ++j) {
				tmp[j] = static_cast<uint32_t>(buf[j]) - static_cast<uint32_t>(base);
			}
			if (layout == FLS_LAYOUT_TRANSPOSED) {
				transpose_i(tmp, tr);
				pack(tr, dst, use);
			} else {
				pack(tmp, dst, use);
			}
		} else {
			transpose_i(reinterpret_cast<const uint32_t*>(buf), tr);
			unrsum(tr, tmp);
			std::memcpy(dst, tr, sizeof(uint32_t) * 32);
			pack(tmp, dst + 32, use);
		}
	}
	*out_words = n_vec * stride;
	if (out_bw) { *out_bw = static_cast<uint8_t>(use); }
	return FLS_OK;
}

fls_status fls_encode_column(const int32_t* values, uint64_t n, const uint8_t* schemes, uint32_t scheme,
                             uint32_t layout, int round4, uint32_t* out, uint64_t* out_words, fls_vec_meta* meta,
                             uint32_t* max_vec_words, uint32_t* scheme_mask) {
	if (!values || !out || !out_words || !meta || n == 0) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_encode_column: null pointer or n == 0");
	}
	if (!schemes && scheme >= FLS_N_SCHEMES) { return set_error(FLS_ERR_INVALID_ARG, "fls_encode_column: bad scheme"); }
	if (layout > FLS_LAYOUT_TRANSPOSED) { return set_error(FLS_ERR_INVALID_ARG, "fls_encode_column: bad layout"); }
	const uint64_t n_vec = (n + 1023u) / 1024u;
	bool           bad   = false;
	// Pass 1: encode into a scratch slot to learn each vector's metadata.
#pragma omp parallel
	{
		std::vector<uint32_t> scratch(kMaxVecWords + 4);
#pragma omp for schedule(dynamic, 64) reduction(|| : bad)
		for (int64_t v = 0; v < static_cast<int64_t>(n_vec); ++v) {
			int32_t buf[1024];
			load_vector(values, n, static_cast<uint64_t>(v), buf);
			uint32_t s = schemes ? schemes[v] : scheme;
			if (s >= FLS_N_SCHEMES) {
				bad = true;
				continue;
			}
			if (!encode_vector(buf, s, layout, round4 != 0, scratch.data(), &meta[v])) {
				encode_vector(buf, FLS_SCHEME_FOR, layout, round4 != 0, scratch.data(), &meta[v]);
			}
		}
	}
	if (bad) { return set_error(FLS_ERR_INVALID_ARG, "fls_encode_column: bad per-vector scheme"); }
	uint64_t off = 0;
	uint32_t mx = 0, mask = 0;
	for (uint64_t v = 0; v < n_vec; ++v) {
		const uint32_t w = vec_payload_words(meta[v].scheme, meta[v].bw, meta[v].aux);
		meta[v].offset   = off;
		off += w;
		mx = std::max(mx, w);
		mask |= 1u << meta[v].scheme;
	}
	// Pass 2: encode in place at the final offsets.
#pragma omp parallel for schedule(dynamic, 64)
	for (int64_t v = 0; v < static_cast<int64_t>(n_vec); ++v) {
		int32_t      buf[1024];
		fls_vec_meta m;
		load_vector(values, n, static_cast<uint64_t>(v), buf);
		encode_vector(buf, meta[v].scheme, layout, round4 != 0, out + meta[v].offset, &m);
	}
	*out_words = off;
	if (max_vec_words) { *max_vec_words = mx; }
	if (scheme_mask) { *scheme_mask = mask; }
	return FLS_OK;
}

fls_status fls_encode_exhaustive(const int32_t* values, uint64_t n, uint32_t* sizes, uint8_t* best, int n_threads) {
	if (!values || n == 0 || (!sizes && !best)) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_encode_exhaustive: null pointer or n == 0");
	}
	const uint64_t n_vec = (n + 1023u) / 1024u;
#pragma omp parallel for schedule(dynamic, 64) num_threads(resolve_threads(n_threads))
	for (int64_t v = 0; v < static_cast<int64_t>(n_vec); ++v) {
		int32_t  buf[1024];
		uint32_t s5[FLS_N_SCHEMES];
		load_vector(values, n, static_cast<uint64_t>(v), buf);
		scheme_sizes(buf, s5);
		if (sizes) { std::memcpy(sizes + 5u * static_cast<uint64_t>(v), s5, sizeof(s5)); }
		if (best) { best[v] = best_scheme(s5); }
	}
	return FLS_OK;
}

fls_status fls_vector_stats(const int32_t* values, uint64_t n, float* stats16, int n_threads) {
	if (!values || !stats16 || n == 0) { return set_error(FLS_ERR_INVALID_ARG, "fls_vector_stats: null pointer"); }
	const uint64_t n_vec = (n + 1023u) / 1024u;
#pragma omp parallel for schedule(static) num_threads(resolve_threads(n_threads))
	for (int64_t v = 0; v < static_cast<int64_t>(n_vec); ++v) {
		int32_t buf[1024];
		load_vector(values, n, static_cast<uint64_t>(v), buf);
		vector_stats(buf, stats16 + 16u * static_cast<uint64_t>(v));
	}
	return FLS_OK;
}

} // extern "C"
