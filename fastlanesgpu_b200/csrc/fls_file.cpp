// fls_file.cpp -- the encoded-column container: one column's payload words
// and per-vector metadata in a single self-describing byte string, so that
// encoded data can be written to storage and read back (checkpoint/resume of
// an encoded table) without re-encoding.
//
// The reference keeps raw int32 columns on disk (storeColumn / loadColumn,
// fastlanes/src/include/crystal_ssb_utils.h:108-127) and re-encodes them on
// every run (compress_ssb.cu:357-454, with its per-vector {bw, base, offset}
// arrays); it has no encoded-data format, so this layout is this library's:
//
//   [payload: n_words x u32][zero pad to 16 B][meta: n_vec x fls_vec_meta]
//   [footer: 96 B]
//
// all little-endian.  The footer comes last (a reader finds it from the end),
// holds the column descriptor, the metadata offset, CRC-32C checksums of the
// payload and metadata bytes and of the footer itself, a version and the
// magic "FLSCOLv1".  Opening a container checks the three checksums, every
// field and every vector's metadata against the payload before handing out a
// descriptor, so a damaged or hostile file is refused on the host instead of
// reaching a kernel (a damaged descriptor -- a FOR base, the layout, the row
// count -- would otherwise decode to other values without any fault).
#include <cstring>
#include <mutex>

#include "fls_internal.h"

namespace fls {
namespace {

constexpr char     kMagic[8]    = {'F', 'L', 'S', 'C', 'O', 'L', 'v', '1'};
constexpr uint32_t kVersion     = 2; // 1 had no footer checksum
constexpr uint64_t kFooterBytes = 96;

struct Footer {
	uint64_t n_values;
	uint64_t n_words;     // payload words stored
	uint64_t n_vec;
	uint64_t meta_offset; // bytes from the start; 0 for a uniform column
	uint32_t layout, scheme, bw;
	int32_t  base;
	uint32_t max_vec_words, scheme_mask;
	uint32_t has_meta;
	uint32_t crc_words, crc_meta;
	uint32_t crc_footer; // CRC-32C of the footer with this field zero
	uint32_t reserved[3];
	uint32_t version;
	char     magic[8];
};
static_assert(sizeof(Footer) == kFooterBytes, "footer layout");

// CRC-32C (Castagnoli polynomial, reflected 0x82F63B78), table-driven.
const uint32_t* crc_table() {
	static uint32_t       t[256];
	static std::once_flag once;
	std::call_once(once, [] {
		for (uint32_t i = 0; i < 256; ++i) {
			uint32_t c = i;
			for (int k = 0; k < 8; ++k) { c = (c & 1u) ? (c >> 1) ^ 0x82F63B78u : c >> 1; }
			t[i] = c;
		}
	});
	return t;
}

uint32_t crc32c(const void* data, uint64_t n) {
	const uint32_t* t = crc_table();
	const uint8_t*  p = static_cast<const uint8_t*>(data);
	uint32_t        c = 0xffffffffu;
	for (uint64_t i = 0; i < n; ++i) { c = t[(c ^ p[i]) & 0xffu] ^ (c >> 8); }
	return c ^ 0xffffffffu;
}

uint64_t align16(uint64_t b) { return (b + 15u) & ~uint64_t {15u}; }

uint64_t n_vectors(uint64_t n) { return (n + 1023u) / 1024u; }

// The container's size for a column with n_words payload words.
uint64_t container_bytes(const fls_column& c) {
	return align16(4u * c.n_words) + (c.meta ? 16u * n_vectors(c.n_values) : 0u) + kFooterBytes;
}

// Every vector's metadata lies inside the payload and names a valid scheme.
fls_status check_vectors(const fls_vec_meta* meta, uint64_t n_vec, uint64_t n_words, uint32_t max_vec_words,
                         uint32_t scheme_mask) {
	for (uint64_t v = 0; v < n_vec; ++v) {
		const fls_vec_meta& m = meta[v];
		if (m.scheme >= FLS_N_SCHEMES || m.bw > 32) {
			return set_error(FLS_ERR_INVALID_ARG, "container: vector " + std::to_string(v) + " has a bad scheme or bit width");
		}
		if ((m.scheme == FLS_SCHEME_RLE || m.scheme == FLS_SCHEME_DICT) && (m.aux == 0 || m.aux > 1024)) {
			return set_error(FLS_ERR_INVALID_ARG, "container: vector " + std::to_string(v) + " has a bad run/dictionary count");
		}
		const uint32_t w = vec_payload_words(m.scheme, m.bw, m.aux);
		if ((m.offset & 3u) || m.offset > n_words || w > n_words - m.offset || w > max_vec_words ||
		    !((scheme_mask >> m.scheme) & 1u)) {
			return set_error(FLS_ERR_INVALID_ARG, "container: vector " + std::to_string(v) + " lies outside the payload");
		}
	}
	return FLS_OK;
}

// The column description a container may hold, checked by the writer before
// any byte is written and by the reader before a descriptor is handed out, so
// a column that one refuses the other refuses too.  Sizes are compared by
// division: n_values is capped at FLS_MAX_VALUES, and no product of a count
// and a vector size is formed that could wrap.
fls_status check_description(uint64_t n_values, uint64_t n_words, uint32_t layout, uint32_t scheme, uint32_t bw,
                             const fls_vec_meta* meta, uint32_t max_vec_words, uint32_t scheme_mask) {
	if (n_values == 0 || n_values > FLS_MAX_VALUES || layout > FLS_LAYOUT_TRANSPOSED) {
		return set_error(FLS_ERR_INVALID_ARG, "container: inconsistent column description (row count or layout)");
	}
	const uint64_t n_vec = n_vectors(n_values);
	if (meta) {
		if (max_vec_words > kMaxVecWords) {
			return set_error(FLS_ERR_INVALID_ARG, "container: largest vector payload out of range");
		}
		return check_vectors(meta, n_vec, n_words, max_vec_words, scheme_mask);
	}
	if ((scheme != FLS_SCHEME_FOR && scheme != FLS_SCHEME_DELTA) || bw > 32 ||
	    (scheme == FLS_SCHEME_DELTA && layout != FLS_LAYOUT_TRANSPOSED)) {
		return set_error(FLS_ERR_INVALID_ARG, "container: bad uniform column (scheme, bit width or layout)");
	}
	const uint64_t per = scheme == FLS_SCHEME_FOR ? 32u * bw : 32u + 32u * bw;
	if (per != 0 && n_vec > n_words / per) {
		return set_error(FLS_ERR_INVALID_ARG, "container: uniform column larger than its payload");
	}
	return FLS_OK;
}

} // namespace
} // namespace fls

using namespace fls;

extern "C" {

uint64_t fls_column_container_bytes(const fls_column* col) { return col ? container_bytes(*col) : 0u; }

fls_status fls_column_write_container(const fls_column* col, void* out, uint64_t out_bytes, uint64_t* written) {
	if (!col || !out || !col->data) { return set_error(FLS_ERR_INVALID_ARG, "fls_column_write_container: null pointer"); }
	if (col->n_values == 0 || col->n_values > FLS_MAX_VALUES || col->n_words > (UINT64_MAX >> 4)) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_column_write_container: empty column or more than FLS_MAX_VALUES rows");
	}
	const uint64_t need = container_bytes(*col);
	if (out_bytes < need) {
		return set_error(FLS_ERR_CAPACITY, "fls_column_write_container: output smaller than fls_column_container_bytes");
	}
	fls_status s = check_description(col->n_values, col->n_words, col->layout, col->scheme, col->bw, col->meta,
	                                 col->max_vec_words, col->scheme_mask);
	if (s != FLS_OK) { return s; }
	const uint64_t n_vec = n_vectors(col->n_values);
	uint8_t*       o     = static_cast<uint8_t*>(out);
	const uint64_t pay_b = 4u * col->n_words;
	std::memcpy(o, col->data, pay_b);
	std::memset(o + pay_b, 0, align16(pay_b) - pay_b);
	Footer f {};
	f.n_values      = col->n_values;
	f.n_words       = col->n_words;
	f.n_vec         = n_vec;
	f.meta_offset   = col->meta ? align16(pay_b) : 0u;
	f.layout        = col->layout;
	f.scheme        = col->scheme;
	f.bw            = col->bw;
	f.base          = col->base;
	f.max_vec_words = col->max_vec_words;
	f.scheme_mask   = col->scheme_mask;
	f.has_meta      = col->meta ? 1u : 0u;
	f.crc_words     = crc32c(col->data, pay_b);
	f.crc_meta      = 0;
	if (col->meta) {
		std::memcpy(o + f.meta_offset, col->meta, 16u * n_vec);
		f.crc_meta = crc32c(col->meta, 16u * n_vec);
	}
	f.version = kVersion;
	std::memcpy(f.magic, kMagic, sizeof(kMagic));
	f.crc_footer = crc32c(&f, kFooterBytes);
	std::memcpy(o + need - kFooterBytes, &f, kFooterBytes);
	if (written) { *written = need; }
	return FLS_OK;
}

fls_status fls_column_open_container(const void* buf, uint64_t bytes, fls_column* col) {
	if (!buf || !col) { return set_error(FLS_ERR_INVALID_ARG, "fls_column_open_container: null pointer"); }
	if (reinterpret_cast<uintptr_t>(buf) & 15u) {
		return set_error(FLS_ERR_ALIGNMENT, "fls_column_open_container: buffer must be 16-byte aligned");
	}
	if (bytes < kFooterBytes) { return set_error(FLS_ERR_INVALID_ARG, "container: shorter than its footer"); }
	const uint8_t* b = static_cast<const uint8_t*>(buf);
	Footer         f;
	std::memcpy(&f, b + bytes - kFooterBytes, kFooterBytes);
	if (std::memcmp(f.magic, kMagic, sizeof(kMagic)) != 0) {
		return set_error(FLS_ERR_INVALID_ARG, "container: bad magic (not an encoded column)");
	}
	if (f.version != kVersion) {
		return set_error(FLS_ERR_UNSUPPORTED, "container: version " + std::to_string(f.version) + " not supported");
	}
	{
		Footer z          = f;
		z.crc_footer      = 0;
		if (crc32c(&z, kFooterBytes) != f.crc_footer) {
			return set_error(FLS_ERR_INVALID_ARG, "container: footer checksum mismatch");
		}
	}
	const uint64_t body = bytes - kFooterBytes;
	if (f.n_values == 0 || f.n_values > FLS_MAX_VALUES || f.n_vec != n_vectors(f.n_values) || f.n_words > body / 4u ||
	    f.layout > FLS_LAYOUT_TRANSPOSED || f.has_meta > 1u || f.reserved[0] || f.reserved[1] || f.reserved[2]) {
		return set_error(FLS_ERR_INVALID_ARG, "container: inconsistent column description");
	}
	const uint64_t pay_b = 4u * f.n_words;
	if (f.has_meta) {
		if (f.meta_offset != align16(pay_b) || f.n_vec > (body - f.meta_offset) / 16u ||
		    f.meta_offset + 16u * f.n_vec != body) {
			return set_error(FLS_ERR_INVALID_ARG, "container: metadata outside the container");
		}
	} else if (f.meta_offset != 0 || align16(pay_b) != body) {
		return set_error(FLS_ERR_INVALID_ARG, "container: size does not match the payload");
	}
	if (crc32c(b, pay_b) != f.crc_words) { return set_error(FLS_ERR_INVALID_ARG, "container: payload checksum mismatch"); }
	const fls_vec_meta* meta = f.has_meta ? reinterpret_cast<const fls_vec_meta*>(b + f.meta_offset) : nullptr;
	if (meta && crc32c(meta, 16u * f.n_vec) != f.crc_meta) {
		return set_error(FLS_ERR_INVALID_ARG, "container: metadata checksum mismatch");
	}
	fls_status s = check_description(f.n_values, f.n_words, f.layout, f.scheme, f.bw, meta, f.max_vec_words,
	                                 f.scheme_mask);
	if (s != FLS_OK) { return s; }
	fls_column c {};
	c.data          = reinterpret_cast<const uint32_t*>(b);
	c.meta          = meta;
	c.n_values      = f.n_values;
	c.n_words       = f.n_words;
	c.layout        = f.layout;
	c.scheme        = f.scheme;
	c.bw            = f.bw;
	c.base          = f.base;
	c.max_vec_words = f.max_vec_words;
	c.scheme_mask   = f.scheme_mask;
	*col            = c;
	return FLS_OK;
}

} // extern "C"
