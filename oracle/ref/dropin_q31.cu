// TEST INFRASTRUCTURE ONLY.  The reference's own Q3.1 kernels
// (fastlanes/src/ssb/fls_q31.cu, included where it lies, unchanged) compiled
// against this project's drop-in device headers (include/compat first on the
// include path).  probe_v1 decodes each column with the normal-form
// unpack_device (unpack.cuh) into shared memory and reads it back with
// BlockLoad; probe_v2 probes with BlockProbeAndPHT_2_R_S into shared tiles;
// probe_v3 / probe_v4 use unpack_8_at_a_time with BlockLoad / BlockPredLoad.
// The launchers run them as the file's runQuery does (fls_q31.cu:372-470).
#define main fls_ref_q31_main
#include "ssb/fls_q31.cu"
#undef main

extern "C" {

// ht_s: 2 * s_len, ht_c: 2 * c_len, ht_d: 2 * d_val_len from key 19920101;
// zeroed by the caller.
int dropin_q31_build(int* s_region, int* s_suppkey, int* s_nation, int s_len, int* c_region, int* c_custkey,
                     int* c_nation, int c_len, int* d_datekey, int* d_year, int d_len, int* ht_s, int* ht_c, int* ht_d,
                     int d_val_len) {
	constexpr int BT = 32, IPT = 8, TILE = BT * IPT;
	build_hashtable_s<BT, IPT><<<(s_len + TILE - 1) / TILE, BT>>>(s_region, s_suppkey, s_nation, s_len, ht_s, s_len);
	build_hashtable_c<BT, IPT><<<(c_len + TILE - 1) / TILE, BT>>>(c_region, c_custkey, c_nation, c_len, ht_c, c_len);
	build_hashtable_d<BT, IPT><<<(d_len + TILE - 1) / TILE, BT>>>(d_datekey, d_year, d_len, ht_d, d_val_len, 19920101);
	return static_cast<int>(cudaDeviceSynchronize());
}

// res: 6 * 4375 ints, zeroed by the caller.  Revenue is packed for versions 1
// and 2, plain int32 for 3 and 4.
int dropin_q31_probe(int version, int* lo_orderdate, int* lo_custkey, int* lo_suppkey, int* lo_revenue, int lo_len,
                     int* ht_s, int s_len, int* ht_c, int c_len, int* ht_d, int d_len, int* res) {
	constexpr int BT = 32;
	if (version == 1 || version == 2) {
		constexpr int IPT = 32;
		auto          k   = version == 1 ? probe_v1<BT, IPT> : probe_v2<BT, IPT>;
		k<<<(lo_len + BT * IPT - 1) / (BT * IPT), BT>>>(lo_orderdate, lo_custkey, lo_suppkey, lo_revenue, lo_len,
		                                                ht_s, s_len, ht_c, c_len, ht_d, d_len, res);
	} else {
		constexpr int IPT = 8;
		auto          k   = version == 3 ? probe_v3<BT, IPT> : probe_v4<BT, IPT>;
		k<<<(lo_len + BT * IPT - 1) / (BT * IPT), BT>>>(lo_orderdate, lo_custkey, lo_suppkey, lo_revenue, lo_len,
		                                                ht_s, s_len, ht_c, c_len, ht_d, d_len, res);
	}
	return static_cast<int>(cudaDeviceSynchronize());
}

// Bit widths the file packs with (query_mtd.ssb): orderdate, custkey, suppkey, revenue.
void dropin_q31_widths(int* out4) {
	out4[0] = query_mtd.ssb.lo_orderdate_bw;
	out4[1] = query_mtd.ssb.lo_chosen_custkey_bw;
	out4[2] = query_mtd.ssb.lo_chosen_suppkey_bw;
	out4[3] = query_mtd.ssb.lo_revenue_bw;
}

int dropin_q31_take_error(uint32_t* bits) { return static_cast<int>(fls::crystal::fls_crystal_take_error(bits)); }

} // extern "C"
