// TEST INFRASTRUCTURE ONLY: the reference CPU arm for the fused query shapes.
//
// Decode uses the reference's own register-form unpack (unpack_fused.cuh,
// host-compiled lane by lane); the per-row predicate / probe / aggregate
// loops restate fastlanes/src/ssb/fls_q11.cu:49-72 (filter-aggregate) and
// fastlanes/src/ssb/fls_q21.cu:50-77 with crystal-opt/join.cuh:26,119-127
// (perfect-hash probes and the int64 group-by), with OpenMP over vectors.
#include <cstdint>
#include <cstring>
#include <omp.h>
#include "ref_api.h"

namespace {
inline void decode_vec(const uint32_t* col, unsigned bw, uint64_t v, uint32_t* out) {
	ref_unpack_fused_u32(col + v * 32ull * bw, out, bw);
}
// HASH(X,Y,Z) ((X-Z) % Y) -- crystal-opt/join.cuh:26.  Negative or out-of-range
// results are undefined behaviour in the reference; here they count as a miss.
inline bool pht_slot(int32_t key, int32_t len, int32_t keys_min, int32_t* h) {
	int32_t x = (key - keys_min) % len;
	if (x < 0 || x >= len) { return false; }
	*h = x;
	return true;
}
} // namespace

extern "C" uint64_t ref_q11_sum(const uint32_t* date_p, unsigned date_bw, const uint32_t* disc_p, unsigned disc_bw,
                                const uint32_t* qty_p, unsigned qty_bw, const uint32_t* price_p, unsigned price_bw,
                                uint64_t n_rows, int32_t date_lo, int32_t date_hi, int32_t disc_lo, int32_t disc_hi,
                                int32_t qty_lt, int n_threads) {
	const uint64_t n_vec = (n_rows + 1023) / 1024;
	long long      total = 0;
#pragma omp parallel for schedule(static) reduction(+ : total) num_threads(n_threads)
	for (uint64_t v = 0; v < n_vec; ++v) {
		uint32_t d[1024], q[1024], s[1024], p[1024];
		decode_vec(date_p, date_bw, v, d);
		decode_vec(qty_p, qty_bw, v, q);
		decode_vec(disc_p, disc_bw, v, s);
		decode_vec(price_p, price_bw, v, p);
		const uint64_t n = (v + 1 == n_vec) ? n_rows - v * 1024 : 1024;
		long long      sum = 0;
		for (uint64_t t = 0; t < n; ++t) {
			int flag = (int32_t)d[t] >= date_lo && (int32_t)d[t] <= date_hi;
			flag     = flag && (int32_t)q[t] < qty_lt;
			flag     = flag && (int32_t)s[t] >= disc_lo && (int32_t)s[t] <= disc_hi;
			if (flag) { sum += (long long)(int32_t)p[t] * (long long)(int32_t)s[t]; }
		}
		total += sum;
	}
	return (uint64_t)total;
}

extern "C" void ref_q21_groupby(const uint32_t* supp_p, unsigned supp_bw, const uint32_t* part_p, unsigned part_bw,
                                const uint32_t* date_p, unsigned date_bw, const uint32_t* rev_p, unsigned rev_bw,
                                uint64_t n_rows, const int32_t* ht_s, int32_t s_len, const int32_t* ht_p,
                                int32_t p_len, const int32_t* ht_d, int32_t d_len, int32_t d_keys_min, int32_t* res,
                                int n_threads) {
	const uint64_t n_vec = (n_rows + 1023) / 1024;
	const int      n_grp = (1998 - 1992 + 1) * (5 * 5 * 40);
#pragma omp parallel num_threads(n_threads)
	{
		long long* local = new long long[n_grp]();
		char*      seen  = new char[n_grp]();
		int32_t*   yb    = new int32_t[2 * n_grp]();
#pragma omp for schedule(static)
		for (uint64_t v = 0; v < n_vec; ++v) {
			uint32_t s[1024], p[1024], d[1024], r[1024];
			decode_vec(supp_p, supp_bw, v, s);
			decode_vec(part_p, part_bw, v, p);
			decode_vec(date_p, date_bw, v, d);
			decode_vec(rev_p, rev_bw, v, r);
			const uint64_t n = (v + 1 == n_vec) ? n_rows - v * 1024 : 1024;
			for (uint64_t t = 0; t < n; ++t) {
				int32_t h;
				if (!pht_slot((int32_t)s[t], s_len, 0, &h) || ht_s[h] == 0) { continue; }
				if (!pht_slot((int32_t)p[t], p_len, 0, &h)) { continue; }
				uint64_t slot;
				std::memcpy(&slot, &ht_p[2 * (int64_t)h], 8);
				if (slot == 0) { continue; }
				int32_t brand = (int32_t)(slot >> 32);
				if (!pht_slot((int32_t)d[t], d_len, d_keys_min, &h)) { continue; }
				std::memcpy(&slot, &ht_d[2 * (int64_t)h], 8);
				if (slot == 0) { continue; }
				int32_t year = (int32_t)(slot >> 32);
				int     g    = (brand * 7 + (year - 1992)) % n_grp;
				if (g < 0) { continue; }
				yb[2 * g]     = year;
				yb[2 * g + 1] = brand;
				seen[g]       = 1;
				local[g] += (long long)(int32_t)r[t];
			}
		}
#pragma omp critical
		{
			for (int g = 0; g < n_grp; ++g) {
				if (!seen[g]) { continue; }
				res[4 * g]     = yb[2 * g];
				res[4 * g + 1] = yb[2 * g + 1];
				uint64_t acc;
				std::memcpy(&acc, &res[4 * g + 2], 8);
				acc += (uint64_t)local[g];
				std::memcpy(&res[4 * g + 2], &acc, 8);
			}
		}
		delete[] local;
		delete[] seen;
		delete[] yb;
	}
}

extern "C" uint64_t ref_decode_sum(const uint32_t* packed, unsigned bw, uint64_t n_vec, int n_threads) {
	unsigned long long total = 0;
#pragma omp parallel for schedule(static) reduction(+ : total) num_threads(n_threads)
	for (uint64_t v = 0; v < n_vec; ++v) {
		uint32_t out[1024];
		ref_unpack_u32(packed + v * 32ull * bw, out, bw);
		unsigned long long s = 0;
		for (int t = 0; t < 1024; ++t) { s += out[t]; }
		total += s;
	}
	return total;
}

extern "C" uint64_t ref_decode(const uint32_t* packed, unsigned bw, uint64_t n_vec, uint32_t* out, int n_threads) {
#pragma omp parallel for schedule(static) num_threads(n_threads)
	for (uint64_t v = 0; v < n_vec; ++v) { ref_unpack_u32(packed + v * 32ull * bw, out + v * 1024, bw); }
	return n_vec * 1024;
}

// Packs a whole column with the reference's pack.cpp, vector by vector
// (fls_q11.cu:207-223); a partial last vector is padded with its last value.
extern "C" void ref_pack_column(const uint32_t* values, uint64_t n, unsigned bw, uint32_t* out, int n_threads) {
	const uint64_t n_vec = (n + 1023) / 1024;
#pragma omp parallel for schedule(static) num_threads(n_threads)
	for (uint64_t v = 0; v < n_vec; ++v) {
		uint32_t       buf[1024];
		const uint64_t cnt = (v + 1 == n_vec) ? n - v * 1024 : 1024;
		std::memcpy(buf, values + v * 1024, cnt * sizeof(uint32_t));
		for (uint64_t j = cnt; j < 1024; ++j) { buf[j] = buf[cnt - 1]; }
		ref_pack_u32(buf, out + v * 32ull * bw, bw);
	}
}

// The reference's decoders + the loops of fls_q31.cu:57-93 (probe_v1): PHT_2
// supplier / customer / date payloads, group (s_nation*175 + c_nation*7 +
// year-1992) % 4375, records of 6 words {year, c_nation, s_nation, -, sum}.
static bool pht2_payload(const int32_t* ht, int32_t len, int32_t keys_min, int32_t key, int32_t* val) {
	int32_t h;
	if (!pht_slot(key, len, keys_min, &h)) { return false; }
	uint64_t slot;
	std::memcpy(&slot, &ht[2 * (int64_t)h], 8);
	if (slot == 0) { return false; }
	*val = (int32_t)(slot >> 32);
	return true;
}

static void merge_groups(int32_t* res, const int32_t* words, const long long* sums, const char* seen, int n_grp,
                         int stride, int n_words, int sum_slot) {
	for (int g = 0; g < n_grp; ++g) {
		if (!seen[g]) { continue; }
		for (int w = 0; w < n_words; ++w) { res[stride * g + w] = words[n_words * g + w]; }
		uint64_t acc;
		std::memcpy(&acc, &res[stride * g + sum_slot], 8);
		acc += (uint64_t)sums[g];
		std::memcpy(&res[stride * g + sum_slot], &acc, 8);
	}
}

extern "C" void ref_q31_groupby(const uint32_t* supp_p, unsigned supp_bw, const uint32_t* cust_p, unsigned cust_bw,
                                const uint32_t* date_p, unsigned date_bw, const uint32_t* rev_p, unsigned rev_bw,
                                uint64_t n_rows, const int32_t* ht_s, int32_t s_len, const int32_t* ht_c,
                                int32_t c_len, const int32_t* ht_d, int32_t d_len, int32_t d_keys_min, int32_t* res,
                                int n_threads) {
	const uint64_t n_vec = (n_rows + 1023) / 1024;
	const int      n_grp = (1998 - 1992 + 1) * 25 * 25;
#pragma omp parallel num_threads(n_threads)
	{
		long long* local = new long long[n_grp]();
		char*      seen  = new char[n_grp]();
		int32_t*   words = new int32_t[3 * n_grp]();
#pragma omp for schedule(static)
		for (uint64_t v = 0; v < n_vec; ++v) {
			uint32_t s[1024], c[1024], d[1024], r[1024];
			decode_vec(supp_p, supp_bw, v, s);
			decode_vec(cust_p, cust_bw, v, c);
			decode_vec(date_p, date_bw, v, d);
			decode_vec(rev_p, rev_bw, v, r);
			const uint64_t n = (v + 1 == n_vec) ? n_rows - v * 1024 : 1024;
			for (uint64_t t = 0; t < n; ++t) {
				int32_t s_nation, c_nation, year;
				if (!pht2_payload(ht_s, s_len, 0, (int32_t)s[t], &s_nation)) { continue; }
				if (!pht2_payload(ht_c, c_len, 0, (int32_t)c[t], &c_nation)) { continue; }
				if (!pht2_payload(ht_d, d_len, d_keys_min, (int32_t)d[t], &year)) { continue; }
				const int g = (s_nation * 25 * 7 + c_nation * 7 + (year - 1992)) % n_grp;
				if (g < 0) { continue; }
				words[3 * g]     = year;
				words[3 * g + 1] = c_nation;
				words[3 * g + 2] = s_nation;
				seen[g]          = 1;
				local[g] += (long long)(int32_t)r[t];
			}
		}
#pragma omp critical
		merge_groups(res, words, local, seen, n_grp, 6, 3, 4);
		delete[] local;
		delete[] seen;
		delete[] words;
	}
}

// The reference's decoders + the loops of fls_q41.cu:61-112 (probe_v1):
// supplier and part PHT_1, customer -> c_nation and date -> year PHT_2, group
// (c_nation*7 + year-1992) % 175, measure revenue - supplycost (int32).
extern "C" void ref_q41_groupby(const uint32_t* supp_p, unsigned supp_bw, const uint32_t* cust_p, unsigned cust_bw,
                                const uint32_t* part_p, unsigned part_bw, const uint32_t* date_p, unsigned date_bw,
                                const uint32_t* rev_p, unsigned rev_bw, const uint32_t* cost_p, unsigned cost_bw,
                                uint64_t n_rows, const int32_t* ht_s, int32_t s_len, const int32_t* ht_c,
                                int32_t c_len, const int32_t* ht_p, int32_t p_len, const int32_t* ht_d, int32_t d_len,
                                int32_t d_keys_min, int32_t* res, int n_threads) {
	const uint64_t n_vec = (n_rows + 1023) / 1024;
	const int      n_grp = (1998 - 1992 + 1) * 25;
#pragma omp parallel num_threads(n_threads)
	{
		long long* local = new long long[n_grp]();
		char*      seen  = new char[n_grp]();
		int32_t*   words = new int32_t[2 * n_grp]();
#pragma omp for schedule(static)
		for (uint64_t v = 0; v < n_vec; ++v) {
			uint32_t s[1024], c[1024], p[1024], d[1024], r[1024], k[1024];
			decode_vec(supp_p, supp_bw, v, s);
			decode_vec(cust_p, cust_bw, v, c);
			decode_vec(part_p, part_bw, v, p);
			decode_vec(date_p, date_bw, v, d);
			decode_vec(rev_p, rev_bw, v, r);
			decode_vec(cost_p, cost_bw, v, k);
			const uint64_t n = (v + 1 == n_vec) ? n_rows - v * 1024 : 1024;
			for (uint64_t t = 0; t < n; ++t) {
				int32_t h, c_nation, year;
				if (!pht_slot((int32_t)s[t], s_len, 0, &h) || ht_s[h] == 0) { continue; }
				if (!pht2_payload(ht_c, c_len, 0, (int32_t)c[t], &c_nation)) { continue; }
				if (!pht_slot((int32_t)p[t], p_len, 0, &h) || ht_p[h] == 0) { continue; }
				if (!pht2_payload(ht_d, d_len, d_keys_min, (int32_t)d[t], &year)) { continue; }
				const int g = (c_nation * 7 + (year - 1992)) % n_grp;
				if (g < 0) { continue; }
				words[2 * g]     = year;
				words[2 * g + 1] = c_nation;
				seen[g]          = 1;
				local[g] += (long long)(int32_t)(r[t] - k[t]);
			}
		}
#pragma omp critical
		merge_groups(res, words, local, seen, n_grp, 4, 2, 2);
		delete[] local;
		delete[] seen;
		delete[] words;
	}
}
