// fls_widths.cpp -- FastLanes bit-packing of the 8-, 16- and 64-bit lane
// widths on the host (the 32-bit form lives in fls_host.cpp).
//
// A vector is 1024 values of T bits in S = 1024 / T lanes: lane i holds the
// rows r = 0..T-1, value S*r + i, masked to bw bits and packed LSB-first into
// T-bit words, word k of lane i at out[S*k + i] (fastlanes/src/pack.cpp:5-1742
// for 8 bits, the 16-bit block after it, 7280-29520 for 64 bits, dispatched
// at 29521, 29552 and 29710).  Every width has 128-byte rows, so a packed
// vector is 128*bw bytes whatever T is.
#include <cstring>

#include "fls_internal.h"

namespace fls {
namespace {

template <class T>
constexpr unsigned kBits = 8u * sizeof(T);

template <class T>
T low_mask_t(unsigned bw) {
	return bw >= kBits<T> ? static_cast<T>(~T {0}) : static_cast<T>((T {1} << bw) - 1u);
}

template <class T>
void pack_t(const T* in, T* out, unsigned bw) {
	constexpr unsigned B = kBits<T>, S = 1024u / B;
	if (bw == 0) { return; }
	const T m = low_mask_t<T>(bw);
	for (unsigned i = 0; i < S; ++i) {
		T        acc  = 0;
		unsigned fill = 0, k = 0;
		for (unsigned r = 0; r < B; ++r) {
			const T v = static_cast<T>(in[S * r + i] & m);
			acc       = static_cast<T>(acc | static_cast<T>(v << fill));
			if (fill + bw >= B) {
				out[S * k++ + i] = acc;
				acc              = fill + bw > B ? static_cast<T>(v >> (B - fill)) : T {0};
				fill             = fill + bw - B;
			} else {
				fill += bw;
			}
		}
	}
}

template <class T>
void unpack_t(const T* in, T* out, unsigned bw) {
	constexpr unsigned B = kBits<T>, S = 1024u / B;
	const T            m = low_mask_t<T>(bw);
	for (unsigned i = 0; i < S; ++i) {
		for (unsigned r = 0; r < B; ++r) {
			T v = 0;
			if (bw) {
				const unsigned bit = r * bw, k = bit / B, s = bit % B;
				v                  = static_cast<T>(in[S * k + i] >> s);
				if (s + bw > B) { v = static_cast<T>(v | static_cast<T>(in[S * (k + 1) + i] << (B - s))); }
			}
			out[S * r + i] = static_cast<T>(v & m);
		}
	}
}

// A column of n T-bit values minus `base` (modulo 2^T) packed vector by vector;
// the last vector is padded with the column's last value.  Fails if a value
// minus base needs more than bw bits.
template <class T>
fls_status pack_column_t(const T* in, uint64_t n, unsigned bw, T base, T* out) {
	constexpr unsigned B = kBits<T>;
	const T            m = low_mask_t<T>(bw);
	const uint64_t     n_vec = (n + 1023u) / 1024u;
	T                  vec[1024];
	for (uint64_t v = 0; v < n_vec; ++v) {
		for (uint32_t j = 0; j < 1024; ++j) {
			const uint64_t idx = v * 1024u + j;
			const T        x   = static_cast<T>(in[idx < n ? idx : n - 1] - base);
			if (bw < B && (x & static_cast<T>(~m)) != 0) {
				return set_error(FLS_ERR_BAD_BW, "fls_pack_column: values do not fit the bit width");
			}
			vec[j] = x;
		}
		pack_t<T>(vec, out + v * (1024u / B) * bw, bw);
	}
	return FLS_OK;
}

bool width_ok(uint32_t bits) { return bits == 8 || bits == 16 || bits == 32 || bits == 64; }

} // namespace
} // namespace fls

using namespace fls;

extern "C" {

fls_status fls_pack_u8(const uint8_t* in, uint8_t* out, uint8_t bw) {
	if (!in || !out) { return set_error(FLS_ERR_INVALID_ARG, "fls_pack_u8: null pointer"); }
	if (bw > 8) { return set_error(FLS_ERR_BAD_BW, "fls_pack_u8: bit width > 8"); }
	pack_t<uint8_t>(in, out, bw);
	return FLS_OK;
}

fls_status fls_pack_u16(const uint16_t* in, uint16_t* out, uint8_t bw) {
	if (!in || !out) { return set_error(FLS_ERR_INVALID_ARG, "fls_pack_u16: null pointer"); }
	if (bw > 16) { return set_error(FLS_ERR_BAD_BW, "fls_pack_u16: bit width > 16"); }
	pack_t<uint16_t>(in, out, bw);
	return FLS_OK;
}

fls_status fls_pack_u64(const uint64_t* in, uint64_t* out, uint8_t bw) {
	if (!in || !out) { return set_error(FLS_ERR_INVALID_ARG, "fls_pack_u64: null pointer"); }
	if (bw > 64) { return set_error(FLS_ERR_BAD_BW, "fls_pack_u64: bit width > 64"); }
	pack_t<uint64_t>(in, out, bw);
	return FLS_OK;
}

fls_status fls_unpack_u8(const uint8_t* in, uint8_t* out, uint8_t bw) {
	if (!in || !out) { return set_error(FLS_ERR_INVALID_ARG, "fls_unpack_u8: null pointer"); }
	if (bw > 8) { return set_error(FLS_ERR_BAD_BW, "fls_unpack_u8: bit width > 8"); }
	unpack_t<uint8_t>(in, out, bw);
	return FLS_OK;
}

fls_status fls_unpack_u16(const uint16_t* in, uint16_t* out, uint8_t bw) {
	if (!in || !out) { return set_error(FLS_ERR_INVALID_ARG, "fls_unpack_u16: null pointer"); }
	if (bw > 16) { return set_error(FLS_ERR_BAD_BW, "fls_unpack_u16: bit width > 16"); }
	unpack_t<uint16_t>(in, out, bw);
	return FLS_OK;
}

fls_status fls_unpack_u64(const uint64_t* in, uint64_t* out, uint8_t bw) {
	if (!in || !out) { return set_error(FLS_ERR_INVALID_ARG, "fls_unpack_u64: null pointer"); }
	if (bw > 64) { return set_error(FLS_ERR_BAD_BW, "fls_unpack_u64: bit width > 64"); }
	unpack_t<uint64_t>(in, out, bw);
	return FLS_OK;
}

fls_status fls_pack_column(const void* in, uint64_t n, uint32_t value_bits, uint8_t bw, uint64_t base, void* out) {
	if (!in || !out || n == 0) { return set_error(FLS_ERR_INVALID_ARG, "fls_pack_column: null pointer or n == 0"); }
	if (!width_ok(value_bits)) { return set_error(FLS_ERR_INVALID_ARG, "fls_pack_column: value_bits must be 8/16/32/64"); }
	if (bw > value_bits) { return set_error(FLS_ERR_BAD_BW, "fls_pack_column: bit width larger than the values"); }
	switch (value_bits) {
	case 8:
		return pack_column_t<uint8_t>(static_cast<const uint8_t*>(in), n, bw, static_cast<uint8_t>(base),
		                              static_cast<uint8_t*>(out));
	case 16:
		return pack_column_t<uint16_t>(static_cast<const uint16_t*>(in), n, bw, static_cast<uint16_t>(base),
		                               static_cast<uint16_t*>(out));
	case 32:
		return pack_column_t<uint32_t>(static_cast<const uint32_t*>(in), n, bw, static_cast<uint32_t>(base),
		                               static_cast<uint32_t*>(out));
	default:
		return pack_column_t<uint64_t>(static_cast<const uint64_t*>(in), n, bw, base, static_cast<uint64_t*>(out));
	}
}

} // extern "C"
