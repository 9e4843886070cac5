/*
 * fls_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference's
 * FastLanes decode + Crystal query path; see fls_oracle.h for what pins it.
 * Loaded only by tests/, the smoke entry point and bench.py's CPU baseline.
 */
#include "fls_oracle.h"

#include <stdlib.h>
#include <math.h>
#include <string.h>

/* ---- layout ------------------------------------------------------------ */

static const uint32_t k_row_quad[4] = {0, 2, 1, 3};

uint32_t orc_tpos(uint32_t j) {
	/* transpose.cpp:4110-4135 (and the row order of rsum.cuh:4-107): chunk c of
	 * 32 consecutive values lands in one lane, visited in rsum row order. */
	uint32_t c    = j >> 5, s = j & 31u;
	uint32_t lane = (c >> 1) | ((c & 1u) << 4);
	uint32_t row  = 4u * (s & 7u) + k_row_quad[s >> 3];
	return 32u * row + lane;
}

void orc_transpose_i(const uint32_t* in, uint32_t* out) {
	for (uint32_t j = 0; j < 1024; ++j) { out[orc_tpos(j)] = in[j]; }
}

void orc_untranspose(const uint32_t* in, uint32_t* out) {
	for (uint32_t j = 0; j < 1024; ++j) { out[j] = in[orc_tpos(j)]; }
}

/* ---- bit-packing -------------------------------------------------------- */

unsigned orc_bit_width(uint32_t v) {
	unsigned bw = 0;
	while (v) { ++bw; v >>= 1; }
	return bw;
}

static uint32_t mask_of(unsigned bw) { return bw >= 32 ? 0xffffffffu : ((1u << bw) - 1u); }

void orc_pack(const uint32_t* in, uint32_t* out, unsigned bw) {
	/* pack.cpp:1954-1990: lane i packs rows r = 0..31 of in[32r+i] LSB-first into
	 * its own word stream; word k of lane i is out[32k+i]. */
	if (bw == 0) { return; }
	const uint32_t m = mask_of(bw);
	memset(out, 0, sizeof(uint32_t) * 32u * bw);
	for (uint32_t lane = 0; lane < 32; ++lane) {
		for (uint32_t r = 0; r < 32; ++r) {
			uint64_t v   = in[32u * r + lane] & m;
			uint32_t bit = r * bw, k = bit >> 5, sh = bit & 31u;
			out[32u * k + lane] |= (uint32_t)(v << sh);
			if (sh + bw > 32) { out[32u * (k + 1) + lane] |= (uint32_t)(v >> (32u - sh)); }
		}
	}
}

void orc_unpack(const uint32_t* in, uint32_t* out, unsigned bw) {
	/* unpack.cuh:201-279: inverse of orc_pack; a value that straddles words k and
	 * k+1 takes its high bits from the low bits of word k+1. */
	const uint32_t m = mask_of(bw);
	for (uint32_t lane = 0; lane < 32; ++lane) {
		for (uint32_t r = 0; r < 32; ++r) {
			if (bw == 0) { out[32u * r + lane] = 0; continue; }
			uint32_t bit = r * bw, k = bit >> 5, sh = bit & 31u;
			uint64_t w   = in[32u * k + lane];
			if (sh + bw > 32) { w |= (uint64_t)in[32u * (k + 1) + lane] << 32; }
			out[32u * r + lane] = (uint32_t)(w >> sh) & m;
		}
	}
}

void orc_unpack_quarter(const uint32_t* in_quarter, uint32_t* out256, unsigned bw) {
	/* hardcoded_16.cuh:436-786 decodes rows 8q..8q+7 from in = vec + q*bw*8; for
	 * bw % 4 == 0 those rows start on a word boundary of every lane stream. */
	const uint32_t m = mask_of(bw);
	for (uint32_t lane = 0; lane < 32; ++lane) {
		for (uint32_t r = 0; r < 8; ++r) {
			if (bw == 0) { out256[32u * r + lane] = 0; continue; }
			uint32_t bit = r * bw, k = bit >> 5, sh = bit & 31u;
			uint64_t w   = in_quarter[32u * k + lane];
			if (sh + bw > 32) { w |= (uint64_t)in_quarter[32u * (k + 1) + lane] << 32; }
			out256[32u * r + lane] = (uint32_t)(w >> sh) & m;
		}
	}
}

/* ---- delta over the transposed layout ----------------------------------- */

/* Row visited at step s of a lane's running sum (rsum.cuh:4-107). */
static uint32_t rsum_row(uint32_t s) { return 4u * (s & 7u) + k_row_quad[s >> 3]; }

void orc_unrsum(const uint32_t* in, uint32_t* out) {
	/* unrsum.cpp:120-256: per lane, the difference to the previous row in rsum
	 * order; row 0 gets 0 (its value is the lane's base). */
	for (uint32_t lane = 0; lane < 32; ++lane) {
		uint32_t prev = in[lane];
		out[lane]     = 0;
		for (uint32_t s = 1; s < 32; ++s) {
			uint32_t p = 32u * rsum_row(s) + lane;
			out[p]     = in[p] - prev;
			prev       = in[p];
		}
	}
}

void orc_rsum(const uint32_t* deltas, uint32_t* out, const uint32_t* base) {
	/* rsum.cuh:4-107: lane i starts at base[i] and accumulates in rsum order. */
	for (uint32_t lane = 0; lane < 32; ++lane) {
		uint32_t acc = base[lane];
		for (uint32_t s = 0; s < 32; ++s) {
			uint32_t p = 32u * rsum_row(s) + lane;
			acc += deltas[p];
			out[p] = acc;
		}
	}
}

/* ---- reference RLE ------------------------------------------------------- */

static uint32_t rle_minivec(const int32_t* v, uint8_t* idx, int32_t* dict) {
	/* rle.hpp:8-25 */
	int32_t  cur = v[0];
	uint32_t ci  = 0;
	idx[0]       = 0;
	dict[0]      = cur;
	for (uint32_t i = 1; i < 256; ++i) {
		if (v[i] != cur) {
			++ci;
			dict[ci] = v[i];
			cur      = v[i];
		}
		idx[i] = (uint8_t)ci;
	}
	return ci + 1;
}

int orc_vector_rle(const int32_t* vec, uint8_t* idx, int32_t* dict, uint16_t* dict4) {
	/* rle.hpp:28-41: four 256-value mini-vectors, dictionaries concatenated. */
	dict4[0] = 0;
	for (uint32_t m = 0; m < 4; ++m) {
		uint32_t n = rle_minivec(vec + 256u * m, idx + 256u * m, dict + dict4[m]);
		if (m < 3) {
			dict4[m + 1] = (uint16_t)(dict4[m] + n);
		} else {
			return (int)(dict4[3] + n);
		}
	}
	return 0;
}

/* ---- encoded-vector schemes ---------------------------------------------- */

static uint32_t pad4(uint32_t w) { return (w + 3u) & ~3u; }

static unsigned round_up4(unsigned bw) { return bw == 0 ? 0 : ((bw + 3u) & ~3u); }

/* Sequential LSB-first bit-packing of n values (the dictionary stream). */
static uint32_t pack_seq(const uint32_t* v, uint32_t n, unsigned bw, uint32_t* out) {
	uint32_t words = pad4((n * bw + 31u) / 32u);
	memset(out, 0, sizeof(uint32_t) * words);
	if (bw == 0) { return words; }
	for (uint32_t k = 0; k < n; ++k) {
		uint64_t x   = v[k] & mask_of(bw);
		uint32_t bit = k * bw, w = bit >> 5, sh = bit & 31u;
		out[w] |= (uint32_t)(x << sh);
		if (sh + bw > 32) { out[w + 1] |= (uint32_t)(x >> (32u - sh)); }
	}
	return words;
}

static uint32_t unpack_seq_one(const uint32_t* in, uint32_t k, unsigned bw) {
	if (bw == 0) { return 0; }
	uint32_t bit = k * bw, w = bit >> 5, sh = bit & 31u;
	uint64_t x   = in[w];
	if (sh + bw > 32) { x |= (uint64_t)in[w + 1] << 32; }
	return (uint32_t)(x >> sh) & mask_of(bw);
}

static int cmp_i32(const void* a, const void* b) {
	int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
	return (x > y) - (x < y);
}

static void min_max(const int32_t* in, uint32_t n, int32_t* mn, int32_t* mx) {
	*mn = in[0];
	*mx = in[0];
	for (uint32_t i = 1; i < n; ++i) {
		if (in[i] < *mn) { *mn = in[i]; }
		if (in[i] > *mx) { *mx = in[i]; }
	}
}

/* Global run index of every value: rle.hpp's local index plus the offset of
 * its mini-vector's dictionary. */
static uint32_t rle_global(const int32_t* in, uint32_t* gidx, int32_t* dict) {
	uint8_t  idx[1024];
	uint16_t d4[4];
	uint32_t n = (uint32_t)orc_vector_rle(in, idx, dict, d4);
	for (uint32_t j = 0; j < 1024; ++j) { gidx[j] = (uint32_t)d4[j >> 8] + idx[j]; }
	return n;
}

int orc_encode_vec(const int32_t* in, uint32_t scheme, int transposed, int round4, uint32_t* out, orc_vec* meta) {
	int32_t mn, mx;
	min_max(in, 1024, &mn, &mx);
	memset(meta, 0, sizeof(*meta));
	meta->scheme = scheme;
	uint32_t tmp[1024], tr[1024];
	switch (scheme) {
	case ORC_CONST:
		if (mn != mx) { return -1; }
		meta->base = mn;
		return 0;
	case ORC_FOR: {
		/* FOR (subtract the vector minimum, ssb_utils.h:187-205) then bit-pack
		 * at the range's bit width (optionally rounded up as find_bw does,
		 * ssb_utils.h:222-239). */
		unsigned bw = orc_bit_width((uint32_t)mx - (uint32_t)mn);
		if (round4) { bw = round_up4(bw); }
		for (uint32_t j = 0; j < 1024; ++j) { tmp[j] = (uint32_t)in[j] - (uint32_t)mn; }
		if (transposed) {
			orc_transpose_i(tmp, tr);
			memcpy(tmp, tr, sizeof(tmp));
		}
		orc_pack(tmp, out, bw);
		meta->base    = mn;
		meta->bw      = bw;
		meta->n_words = 32u * bw;
		return 0;
	}
	case ORC_DELTA: {
		/* delta_shared_memory.cu:142-157: transpose_i, unrsum, bases = first 32
		 * transposed values, pack the deltas. */
		uint32_t d[1024];
		orc_transpose_i((const uint32_t*)in, tr);
		orc_unrsum(tr, d);
		uint32_t mxd = 0;
		for (uint32_t j = 0; j < 1024; ++j) {
			if (d[j] > mxd) { mxd = d[j]; }
		}
		unsigned bw = orc_bit_width(mxd);
		memcpy(out, tr, sizeof(uint32_t) * 32);
		orc_pack(d, out + 32, bw);
		meta->bw      = bw;
		meta->n_words = 32u + 32u * bw;
		return 0;
	}
	case ORC_RLE: {
		/* Run index (rle.hpp) as a transposed delta at bit width 1 with 16-bit
		 * lane bases, followed by the FOR'd run values packed sequentially. */
		uint32_t gidx[1024], d[1024];
		int32_t  dict[1024];
		uint32_t n = rle_global(in, gidx, dict);
		orc_transpose_i(gidx, tr);
		orc_unrsum(tr, d);
		uint16_t* b16 = (uint16_t*)out;
		for (uint32_t l = 0; l < 32; ++l) { b16[l] = (uint16_t)tr[l]; }
		orc_pack(d, out + 16, 1);
		int32_t dmn, dmx;
		min_max(dict, n, &dmn, &dmx);
		unsigned bw = orc_bit_width((uint32_t)dmx - (uint32_t)dmn);
		for (uint32_t k = 0; k < n; ++k) { tmp[k] = (uint32_t)dict[k] - (uint32_t)dmn; }
		uint32_t dw   = pack_seq(tmp, n, bw, out + 48);
		meta->base    = dmn;
		meta->bw      = bw;
		meta->aux     = n;
		meta->n_words = 48u + dw;
		return 0;
	}
	case ORC_DICT: {
		/* Sorted distinct values as a FOR'd sequentially packed dictionary,
		 * codes FastLanes bit-packed at bit_width(n_dict - 1). */
		int32_t sorted[1024];
		memcpy(sorted, in, sizeof(sorted));
		qsort(sorted, 1024, sizeof(int32_t), cmp_i32);
		uint32_t n = 0;
		for (uint32_t j = 0; j < 1024; ++j) {
			if (j == 0 || sorted[j] != sorted[j - 1]) { sorted[n++] = sorted[j]; }
		}
		unsigned cbw = orc_bit_width(n - 1);
		for (uint32_t j = 0; j < 1024; ++j) {
			uint32_t lo = 0, hi = n - 1;
			while (lo < hi) {
				uint32_t mid = (lo + hi) >> 1;
				if (sorted[mid] < in[j]) {
					lo = mid + 1;
				} else {
					hi = mid;
				}
			}
			tmp[j] = lo;
		}
		if (transposed) {
			orc_transpose_i(tmp, tr);
			memcpy(tmp, tr, sizeof(tmp));
		}
		orc_pack(tmp, out, cbw);
		unsigned bw = orc_bit_width((uint32_t)sorted[n - 1] - (uint32_t)sorted[0]);
		for (uint32_t k = 0; k < n; ++k) { tmp[k] = (uint32_t)sorted[k] - (uint32_t)sorted[0]; }
		uint32_t dw   = pack_seq(tmp, n, bw, out + 32u * cbw);
		meta->base    = sorted[0];
		meta->bw      = bw;
		meta->aux     = n;
		meta->n_words = 32u * cbw + dw;
		return 0;
	}
	default: return -1;
	}
}

void orc_decode_vec(const uint32_t* in, const orc_vec* meta, int transposed, int32_t* out) {
	uint32_t v[1024], t[1024];
	switch (meta->scheme) {
	case ORC_CONST:
		for (uint32_t j = 0; j < 1024; ++j) { out[j] = meta->base; }
		return;
	case ORC_FOR:
		orc_unpack(in, v, meta->bw);
		if (transposed) {
			orc_untranspose(v, t);
			memcpy(v, t, sizeof(v));
		}
		for (uint32_t j = 0; j < 1024; ++j) { out[j] = (int32_t)(v[j] + (uint32_t)meta->base); }
		return;
	case ORC_DELTA:
		orc_unpack(in + 32, v, meta->bw);
		orc_rsum(v, t, in);
		orc_untranspose(t, (uint32_t*)out);
		return;
	case ORC_RLE: {
		uint32_t        base[32];
		const uint16_t* b16 = (const uint16_t*)in;
		for (uint32_t l = 0; l < 32; ++l) { base[l] = b16[l]; }
		orc_unpack(in + 16, v, 1);
		orc_rsum(v, t, base);
		orc_untranspose(t, v);
		for (uint32_t j = 0; j < 1024; ++j) {
			out[j] = (int32_t)(unpack_seq_one(in + 48, v[j], meta->bw) + (uint32_t)meta->base);
		}
		return;
	}
	case ORC_DICT: {
		unsigned cbw = orc_bit_width(meta->aux - 1);
		orc_unpack(in, v, cbw);
		if (transposed) {
			orc_untranspose(v, t);
			memcpy(v, t, sizeof(v));
		}
		for (uint32_t j = 0; j < 1024; ++j) {
			out[j] = (int32_t)(unpack_seq_one(in + 32u * cbw, v[j], meta->bw) + (uint32_t)meta->base);
		}
		return;
	}
	default: memset(out, 0, sizeof(int32_t) * 1024);
	}
}

void orc_scheme_sizes(const int32_t* in, uint32_t* size5) {
	uint32_t buf[4096];
	orc_vec  m;
	for (uint32_t s = 0; s < 5; ++s) {
		if (orc_encode_vec(in, s, 1, 0, buf, &m) != 0) {
			size5[s] = 0xffffffffu;
		} else {
			size5[s] = 4u * m.n_words + 16u;
		}
	}
}

/* ---- query path ---------------------------------------------------------- */

int64_t orc_filter_agg(const int32_t* date, const int32_t* disc, const int32_t* qty, const int32_t* price,
                       uint64_t n, int32_t date_lo, int32_t date_hi, int32_t disc_lo, int32_t disc_hi,
                       int32_t qty_lt) {
	/* fls_q11.cu:49-72: predicates on date, quantity and discount, then
	 * sum += price * discount over the selected rows (64-bit products). */
	int64_t sum = 0;
	for (uint64_t t = 0; t < n; ++t) {
		int f = date[t] >= date_lo && date[t] <= date_hi;
		f     = f && qty[t] < qty_lt;
		f     = f && disc[t] >= disc_lo && disc[t] <= disc_hi;
		if (f) { sum += (int64_t)price[t] * (int64_t)disc[t]; }
	}
	return sum;
}

/* HASH(X,Y,Z) ((X-Z) % Y), join.cuh:26; a negative remainder is out of the
 * table in the reference (undefined there) and a miss here. */
static int pht_hash(int32_t key, int32_t len, int32_t keys_min, int32_t* h) {
	int32_t x = (int32_t)((uint32_t)key - (uint32_t)keys_min) % len;
	if (x < 0) { return 0; }
	*h = x;
	return 1;
}

void orc_pht1_build(const int32_t* filter, int32_t filter_eq, const int32_t* keys, uint64_t n, int32_t* ht,
                    int32_t len, int32_t keys_min) {
	/* join.cuh:190-245: atomicCAS(&ht[hash], 0, key) for selected rows. */
	for (uint64_t t = 0; t < n; ++t) {
		int32_t h;
		if (filter && filter[t] != filter_eq) { continue; }
		if (!pht_hash(keys[t], len, keys_min, &h)) { continue; }
		if (ht[h] == 0) { ht[h] = keys[t]; }
	}
}

void orc_pht2_build(const int32_t* filter, int32_t filter_eq, const int32_t* keys, const int32_t* vals, uint64_t n,
                    int32_t* ht, int32_t len, int32_t keys_min) {
	/* join.cuh:255-275: atomicCAS on the key word, then store the value.  With
	 * distinct keys (a perfect hash) the outcome does not depend on order. */
	for (uint64_t t = 0; t < n; ++t) {
		int32_t h;
		if (filter && filter[t] != filter_eq) { continue; }
		if (!pht_hash(keys[t], len, keys_min, &h)) { continue; }
		if (ht[2 * h] == 0) { ht[2 * h] = keys[t]; }
		ht[2 * h + 1] = vals[t];
	}
}

void orc_probe_groupby(const int32_t* supp, const int32_t* part, const int32_t* date, const int32_t* rev, uint64_t n,
                       const int32_t* ht_s, int32_t s_len, const int32_t* ht_p, int32_t p_len, const int32_t* ht_d,
                       int32_t d_len, int32_t d_keys_min, int32_t* res) {
	/* fls_q21.cu:50-77 with the probes of join.cuh:28-188 (PHT_1: slot != 0;
	 * PHT_2: the (key,value) pair read as one u64, value = slot >> 32). */
	const int32_t n_grp = (1998 - 1992 + 1) * (5 * 5 * 40);
	for (uint64_t t = 0; t < n; ++t) {
		int32_t  h;
		uint64_t slot;
		if (!pht_hash(supp[t], s_len, 0, &h) || ht_s[h] == 0) { continue; }
		if (!pht_hash(part[t], p_len, 0, &h)) { continue; }
		memcpy(&slot, &ht_p[2 * (int64_t)h], 8);
		if (slot == 0) { continue; }
		int32_t brand = (int32_t)(slot >> 32);
		if (!pht_hash(date[t], d_len, d_keys_min, &h)) { continue; }
		memcpy(&slot, &ht_d[2 * (int64_t)h], 8);
		if (slot == 0) { continue; }
		int32_t year = (int32_t)(slot >> 32);
		int32_t g    = (brand * 7 + (year - 1992)) % n_grp;
		if (g < 0) { continue; }
		res[4 * g]     = year;
		res[4 * g + 1] = brand;
		uint64_t acc;
		memcpy(&acc, &res[4 * g + 2], 8);
		acc += (uint64_t)(int64_t)rev[t];
		memcpy(&res[4 * g + 2], &acc, 8);
	}
}

/* PHT_2 lookup: hit, and the payload (the u64 slot's high word). */
static int pht2_get(const int32_t* ht, int32_t len, int32_t keys_min, int32_t key, int32_t* val) {
	int32_t  h;
	uint64_t slot;
	if (!pht_hash(key, len, keys_min, &h)) { return 0; }
	memcpy(&slot, &ht[2 * (int64_t)h], 8);
	if (slot == 0) { return 0; }
	*val = (int32_t)(slot >> 32);
	return 1;
}

static void add_i64(int32_t* p, int64_t x) {
	uint64_t acc;
	memcpy(&acc, p, 8);
	acc += (uint64_t)x;
	memcpy(p, &acc, 8);
}

void orc_pht_build_ranges(const int32_t* filter, int32_t lo0, int32_t hi0, int32_t lo1, int32_t hi1,
                          const int32_t* keys, const int32_t* vals, uint64_t n, int32_t* ht, int32_t len,
                          int32_t keys_min) {
	/* crystal-opt src/ssb/q22.cu:118-154 (BlockPredGTE/AndLTE), q33.cu:100-109
	 * (BlockPredEQ/OrEQ) followed by join.cuh's selective builds. */
	for (uint64_t t = 0; t < n; ++t) {
		int32_t h;
		if (filter && !((filter[t] >= lo0 && filter[t] <= hi0) || (filter[t] >= lo1 && filter[t] <= hi1))) {
			continue;
		}
		if (!pht_hash(keys[t], len, keys_min, &h)) { continue; }
		if (!vals) {
			if (ht[h] == 0) { ht[h] = keys[t]; }
		} else {
			if (ht[2 * h] == 0) { ht[2 * h] = keys[t]; }
			ht[2 * h + 1] = vals[t];
		}
	}
}

void orc_join_groupby(uint64_t n, const orc_probe* probes, uint32_t n_probes, const int32_t* agg,
                      const int32_t* agg_sub, uint32_t n_keys, const int32_t* key_probe, const int32_t* key_mul,
                      const int32_t* key_slot, int32_t group_sub, int32_t n_groups, uint32_t stride,
                      uint32_t sum_slot, uint32_t sum_bits, int32_t* res) {
	/* crystal-opt src/ssb/q32.cu:70-104 and q42.cu:70-116 are this loop with
	 * their probes, key formulas and records: each probe drops the row on a
	 * miss (PHT_1: slot == 0; PHT_2: the (key, value) pair read as one u64 is
	 * 0) or keeps the PHT_2 payload; the selected row writes its key payloads
	 * into its record and adds its measure to the record's sum. */
	for (uint64_t t = 0; t < n; ++t) {
		int32_t  pay[8] = {0, 0, 0, 0, 0, 0, 0, 0};
		int      keep   = 1;
		uint32_t key    = 0u - (uint32_t)group_sub;
		for (uint32_t q = 0; q < n_probes && keep; ++q) {
			const orc_probe* p = &probes[q];
			if (p->kind == 1) {
				int32_t h;
				keep = pht_hash(p->col[t], p->len, p->keys_min, &h) && p->ht[h] != 0;
			} else {
				keep = pht2_get(p->ht, p->len, p->keys_min, p->col[t], &pay[q]);
			}
		}
		if (!keep) { continue; }
		for (uint32_t k = 0; k < n_keys; ++k) { key += (uint32_t)pay[key_probe[k]] * (uint32_t)key_mul[k]; }
		const int32_t g = (int32_t)key % n_groups;
		if (g < 0) { continue; }
		int32_t* rec = res + (int64_t)g * stride;
		for (uint32_t k = 0; k < n_keys; ++k) {
			if (key_slot[k] >= 0) { rec[key_slot[k]] = pay[key_probe[k]]; }
		}
		const int32_t m = (int32_t)((uint32_t)agg[t] - (agg_sub ? (uint32_t)agg_sub[t] : 0u));
		if (sum_bits == 32) {
			rec[sum_slot] = (int32_t)((uint32_t)rec[sum_slot] + (uint32_t)m);
		} else {
			add_i64(&rec[sum_slot], (int64_t)m);
		}
	}
}

void orc_q31_groupby(const int32_t* supp, const int32_t* cust, const int32_t* date, const int32_t* rev, uint64_t n,
                     const int32_t* ht_s, int32_t s_len, const int32_t* ht_c, int32_t c_len, const int32_t* ht_d,
                     int32_t d_len, int32_t d_keys_min, int32_t* res) {
	/* fls_q31.cu:57-93 probe_v1: supplier -> s_nation, customer -> c_nation,
	 * date -> year (all PHT_2); group (s_nation*175 + c_nation*7 + year-1992)
	 * % 4375 into records of 6 words {year, c_nation, s_nation, -, sum}. */
	const int32_t n_grp = (1998 - 1992 + 1) * 25 * 25;
	for (uint64_t t = 0; t < n; ++t) {
		int32_t s_nation, c_nation, year;
		if (!pht2_get(ht_s, s_len, 0, supp[t], &s_nation)) { continue; }
		if (!pht2_get(ht_c, c_len, 0, cust[t], &c_nation)) { continue; }
		if (!pht2_get(ht_d, d_len, d_keys_min, date[t], &year)) { continue; }
		const int32_t g = (int32_t)((uint32_t)s_nation * 175u + (uint32_t)c_nation * 7u + ((uint32_t)year - 1992u)) % n_grp;
		if (g < 0) { continue; }
		res[6 * g]     = year;
		res[6 * g + 1] = c_nation;
		res[6 * g + 2] = s_nation;
		add_i64(&res[6 * g + 4], (int64_t)rev[t]);
	}
}

void orc_q41_groupby(const int32_t* supp, const int32_t* cust, const int32_t* part, const int32_t* date,
                     const int32_t* rev, const int32_t* cost, uint64_t n, const int32_t* ht_s, int32_t s_len,
                     const int32_t* ht_c, int32_t c_len, const int32_t* ht_p, int32_t p_len, const int32_t* ht_d,
                     int32_t d_len, int32_t d_keys_min, int32_t* res) {
	/* fls_q41.cu:61-112 probe_v1: supplier (PHT_1), customer -> c_nation,
	 * part (PHT_1), date -> year; group (c_nation*7 + year-1992) % 175 into
	 * records of 4 words {year, c_nation, sum}; measure revenue - supplycost as
	 * an int32 difference. */
	const int32_t n_grp = (1998 - 1992 + 1) * 25;
	for (uint64_t t = 0; t < n; ++t) {
		int32_t h, c_nation, year;
		if (!pht_hash(supp[t], s_len, 0, &h) || ht_s[h] == 0) { continue; }
		if (!pht2_get(ht_c, c_len, 0, cust[t], &c_nation)) { continue; }
		if (!pht_hash(part[t], p_len, 0, &h) || ht_p[h] == 0) { continue; }
		if (!pht2_get(ht_d, d_len, d_keys_min, date[t], &year)) { continue; }
		const int32_t g = (int32_t)((uint32_t)c_nation * 7u + ((uint32_t)year - 1992u)) % n_grp;
		if (g < 0) { continue; }
		res[4 * g]     = year;
		res[4 * g + 1] = c_nation;
		add_i64(&res[4 * g + 2], (int64_t)(int32_t)((uint32_t)rev[t] - (uint32_t)cost[t]));
	}
}

/* ---- learned selector ------------------------------------------------------ */

double orc_mlp_loss_grad(const float* P, const float* x, const uint8_t* y, uint32_t B, double* g) {
	enum { I = 16, H = 64, O = 5, W1 = 0, B1 = W1 + H * I, W2 = B1 + H, B2 = W2 + H * H, W3 = B2 + H, B3 = W3 + O * H };
	memset(g, 0, sizeof(double) * ORC_MLP_N_PARAMS);
	double loss = 0.0;
	for (uint32_t b = 0; b < B; ++b) {
		const float* xb = x + (size_t)b * I;
		double       h1[H], h2[H], z[O], d2[H], d1[H];
		for (int j = 0; j < H; ++j) {
			double a = P[B1 + j];
			for (int i = 0; i < I; ++i) { a += (double)P[W1 + j * I + i] * xb[i]; }
			h1[j] = a > 0 ? a : 0;
		}
		for (int j = 0; j < H; ++j) {
			double a = P[B2 + j];
			for (int i = 0; i < H; ++i) { a += (double)P[W2 + j * H + i] * h1[i]; }
			h2[j] = a > 0 ? a : 0;
		}
		double m = -1e300, s = 0;
		for (int k = 0; k < O; ++k) {
			double a = P[B3 + k];
			for (int j = 0; j < H; ++j) { a += (double)P[W3 + k * H + j] * h2[j]; }
			z[k] = a;
			if (a > m) { m = a; }
		}
		for (int k = 0; k < O; ++k) {
			z[k] = exp(z[k] - m);
			s += z[k];
		}
		const int t = y[b] < O ? y[b] : 0;
		loss += -log(z[t] / s) / B;
		double dz[O];
		for (int k = 0; k < O; ++k) { dz[k] = (z[k] / s - (k == t)) / B; }
		for (int k = 0; k < O; ++k) {
			g[B3 + k] += dz[k];
			for (int j = 0; j < H; ++j) { g[W3 + k * H + j] += dz[k] * h2[j]; }
		}
		for (int j = 0; j < H; ++j) {
			double a = 0;
			for (int k = 0; k < O; ++k) { a += (double)P[W3 + k * H + j] * dz[k]; }
			d2[j] = h2[j] > 0 ? a : 0;
			g[B2 + j] += d2[j];
			for (int i = 0; i < H; ++i) { g[W2 + j * H + i] += d2[j] * h1[i]; }
		}
		for (int i = 0; i < H; ++i) {
			double a = 0;
			for (int j = 0; j < H; ++j) { a += (double)P[W2 + j * H + i] * d2[j]; }
			d1[i] = h1[i] > 0 ? a : 0;
			g[B1 + i] += d1[i];
			for (int f = 0; f < I; ++f) { g[W1 + i * I + f] += d1[i] * xb[f]; }
		}
	}
	return loss;
}

static unsigned bw_u32(uint32_t v) {
	unsigned b = 0;
	while (v) { ++b; v >>= 1; }
	return b;
}

void orc_vector_stats(const int32_t* v, float* f) {
	int32_t mn, mx;
	min_max(v, 1024, &mn, &mx);
	const uint32_t rbw = bw_u32((uint32_t)mx - (uint32_t)mn);
	uint32_t max_d = 0, runs = 0, up = 0, down = 0, eq = 0, lh = 0, lq = 0, bitmap[32] = {0}, cc = 0;
	uint64_t sabs  = 0;
	for (uint32_t c = 0; c < 32; ++c) {
		int same = 1;
		for (uint32_t s = 1; s < 32; ++s) { same = same && v[32 * c + s] == v[32 * c]; }
		cc += (uint32_t)same;
	}
	for (uint32_t j = 0; j < 1024; ++j) {
		const uint32_t u = (uint32_t)v[j] - (uint32_t)mn;
		lh += (rbw == 0 || u < (1u << (rbw / 2))) ? 1u : 0u;
		lq += (rbw <= 4 || u < (1u << (rbw - 4))) ? 1u : 0u;
		const uint32_t h = ((uint32_t)v[j] * 0x9e3779b1u) >> 22;
		bitmap[h >> 5] |= 1u << (h & 31u);
		if (j == 0) {
			++runs;
			continue;
		}
		const int64_t d = (int64_t)v[j] - (int64_t)v[j - 1];
		sabs += (uint64_t)(d < 0 ? -d : d);
		up += d > 0;
		down += d < 0;
		eq += d == 0;
		if (j & 31u) {
			const uint32_t dd = (uint32_t)v[j] - (uint32_t)v[j - 1];
			if (dd > max_d) { max_d = dd; }
		}
		runs += ((j & 255u) == 0 || d != 0) ? 1u : 0u;
	}
	uint32_t occ = 0;
	for (int w = 0; w < 32; ++w) { occ += (uint32_t)__builtin_popcount(bitmap[w]); }
	const uint64_t md   = sabs >> 10;
	const uint32_t amin = mn < 0 ? (uint32_t)(-(int64_t)mn) : (uint32_t)mn;
	f[0]  = (float)rbw / 32.0f;
	f[1]  = (float)bw_u32(max_d) / 32.0f;
	f[2]  = (float)runs / 1024.0f;
	f[3]  = (float)up / 1024.0f;
	f[4]  = (float)down / 1024.0f;
	f[5]  = (float)eq / 1024.0f;
	f[6]  = (float)occ / 1024.0f;
	f[7]  = (float)bw_u32(occ) / 16.0f;
	f[8]  = (float)bw_u32((uint32_t)(md > 0xffffffffull ? 0xffffffffull : md)) / 32.0f;
	f[9]  = (float)lh / 1024.0f;
	f[10] = (float)lq / 1024.0f;
	f[11] = (float)bw_u32(amin) / 32.0f;
	f[12] = mn == mx ? 1.0f : 0.0f;
	f[13] = (float)bw_u32(runs) / 16.0f;
	f[14] = (float)cc / 32.0f;
	f[15] = 1.0f;
}

/* ---- tile-based RLE (RFOR): tile_based/src/rlebinpack.cpp:9-146 ------- */

uint64_t orc_rfor_bound(uint64_t n) { return 4u + ((n + 511u) / 512u) * (3u + 512u); }

/* Appends one block (min, widths, count, packed fields) at stream[*o]. */
static void rfor_block(uint32_t* stream, uint64_t* o, const uint32_t* x, uint32_t count) {
	uint32_t mn = x[0];
	for (uint32_t k = 1; k < count; ++k) { mn = x[k] < mn ? x[k] : mn; }
	uint32_t bw = 0;
	for (uint32_t k = 0; k < count; ++k) {
		const unsigned b = orc_bit_width(x[k] - mn);
		bw               = b > bw ? b : bw;
	}
	stream[(*o)++] = mn;
	stream[(*o)++] = bw + (bw << 8) + (bw << 16) + (bw << 24);
	stream[(*o)++] = count;
	/* field after field, LSB first, carrying into the next word */
	uint64_t w = *o, shift = 0;
	stream[w]  = 0;
	for (uint32_t k = 0; k < count; ++k) {
		const uint32_t v = x[k] - mn;
		if (bw == 0) { continue; }
		if (shift == 32) {
			stream[++w] = 0;
			shift       = 0;
		}
		stream[w] |= v << shift;
		if (shift + bw > 32) {
			stream[++w] = v >> (32 - shift);
			shift       = shift + bw - 32;
		} else {
			shift += bw;
		}
	}
	*o = w + 1;
}

void orc_rfor_encode(const uint32_t* in, uint64_t n, uint32_t* val, uint32_t* rl, uint32_t* val_off, uint32_t* rl_off,
                     uint64_t* n_val, uint64_t* n_rl) {
	uint64_t vo = 4, ro = 4;
	val[0] = rl[0] = 512;
	val[1] = rl[1] = 4;
	val[2] = rl[2] = (uint32_t)n;
	val[3] = rl[3] = in[0];
	uint32_t v[512], l[512];
	for (uint64_t t = 0; t < n / 512; ++t) {
		const uint32_t* x = in + 512 * t;
		uint32_t        count = 0, run = 1;
		for (uint32_t i = 1; i < 512; ++i) {
			if (x[i] != x[i - 1]) {
				v[count]   = x[i - 1];
				l[count++] = run;
				run        = 1;
			} else {
				++run;
			}
		}
		v[count]   = x[511];
		l[count++] = run;
		val_off[t] = (uint32_t)vo;
		rl_off[t]  = (uint32_t)ro;
		rfor_block(val, &vo, v, count);
		rfor_block(rl, &ro, l, count);
	}
	val_off[n / 512] = (uint32_t)vo;
	rl_off[n / 512]  = (uint32_t)ro;
	*n_val           = vo;
	*n_rl            = ro;
}

static uint32_t rfor_field(const uint32_t* p, uint32_t k, uint32_t bw) {
	if (bw == 0) { return 0; }
	const uint64_t bit = (uint64_t)k * bw;
	uint64_t       two = p[bit >> 5];
	if ((bit & 31) + bw > 32) { two |= (uint64_t)p[(bit >> 5) + 1] << 32; }
	return (uint32_t)((two >> (bit & 31)) & ((1ull << bw) - 1ull));
}

int orc_rfor_decode(const uint32_t* val, const uint32_t* rl, const uint32_t* val_off, const uint32_t* rl_off,
                    uint64_t n, uint32_t* out) {
	for (uint64_t t = 0; t * 512 < n; ++t) {
		const uint32_t* vb = val + val_off[t];
		const uint32_t* rb = rl + rl_off[t];
		const uint32_t  count = vb[2], vbw = vb[1] & 255, rbw = rb[1] & 255;
		if (count == 0 || count > 512 || rb[2] != count || vbw > 32 || rbw > 32) { return -1; }
		uint32_t p = 0;
		for (uint32_t k = 0; k < count; ++k) {
			const uint32_t x   = vb[0] + rfor_field(vb + 3, k, vbw);
			const uint32_t len = rb[0] + rfor_field(rb + 3, k, rbw);
			for (uint32_t i = 0; i < len; ++i, ++p) {
				if (p >= 512) { return -1; }
				if (t * 512 + p < n) { out[t * 512 + p] = x; }
			}
		}
		if (p != 512) { return -1; }
	}
	return 0;
}

uint64_t orc_splitmix64(uint64_t* state) {
	uint64_t z = (*state += 0x9e3779b97f4a7c15ull);
	z          = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
	z          = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
	return z ^ (z >> 31);
}

/* FastLanes packing of the other lane widths (pack.cpp:5-1742 8-bit,
 * the 16-bit block after it, 7280-29520 64-bit; dispatch at 29521, 29552,
 * 29710): a vector of 1024 T-bit values has S = 1024/T lanes; lane i packs
 * rows r = 0..T-1 (value S*r + i), masked to bw bits, LSB-first into T-bit
 * words, word k of lane i at out[S*k + i]. */
#define ORC_PACK_WIDTH(T, B)                                                                                          \
	void orc_pack_##B(const T* in, T* out, unsigned bw) {                                                         \
		const unsigned S = 1024u / (B);                                                                       \
		const T        m = bw >= (B) ? (T)~(T)0 : (T)((((T)1) << bw) - 1u);                                  \
		for (unsigned i = 0; i < S; ++i) {                                                                    \
			unsigned k = 0, fill = 0;                                                                     \
			T        acc = 0;                                                                             \
			if (bw == 0) { continue; }                                                                    \
			for (unsigned r = 0; r < (B); ++r) {                                                          \
				const T v = (T)(in[S * r + i] & m);                                                   \
				acc |= (T)(v << fill);                                                                \
				if (fill + bw >= (B)) {                                                               \
					out[S * k++ + i] = acc;                                                        \
					acc  = fill + bw > (B) ? (T)(v >> ((B) - fill)) : (T)0;                        \
					fill = fill + bw - (B);                                                        \
				} else {                                                                              \
					fill += bw;                                                                    \
				}                                                                                     \
			}                                                                                             \
		}                                                                                                     \
	}                                                                                                             \
	void orc_unpack_##B(const T* in, T* out, unsigned bw) {                                                       \
		const unsigned S = 1024u / (B);                                                                       \
		const T        m = bw >= (B) ? (T)~(T)0 : (T)((((T)1) << bw) - 1u);                                  \
		for (unsigned i = 0; i < S; ++i) {                                                                    \
			for (unsigned r = 0; r < (B); ++r) {                                                          \
				const unsigned bit = r * bw, k = bit / (B), s = bit % (B);                            \
				T              v   = 0;                                                               \
				if (bw) {                                                                             \
					v = (T)(in[S * k + i] >> s);                                                   \
					if (s + bw > (B)) { v |= (T)(in[S * (k + 1) + i] << ((B) - s)); }              \
				}                                                                                     \
				out[S * r + i] = (T)(v & m);                                                          \
			}                                                                                             \
		}                                                                                                     \
	}
ORC_PACK_WIDTH(uint8_t, 8)
ORC_PACK_WIDTH(uint16_t, 16)
ORC_PACK_WIDTH(uint64_t, 64)
