// TEST INFRASTRUCTURE ONLY.  The reference's own Q2.1 kernels
// (fastlanes/src/ssb/fls_q21.cu, included where it lies, unchanged) compiled
// against this project's drop-in device headers: include/compat comes first
// on the include path, so crystal/crystal.cuh, fls_gen/unpack/hardcoded_16.cuh
// and fls_gen/unpack/unpack_fused.cuh resolve to include/fls_crystal.cuh.
// The launchers below run the reference's hash-table builds
// (build_hashtable_s/p/d: BlockLoad, BlockPredEQ, BlockBuildSelectivePHT_1/_2)
// and probes (probe_v1: unpack_device into 32 registers; probe_v2:
// unpack_8_at_a_time::unpack_device + BlockLoad; probe_v3: the same with
// BlockPredLoad) as the file's runQuery does (fls_q21.cu:265-330).
#define main fls_ref_q21_main
#include "ssb/fls_q21.cu"
#undef main

extern "C" {

// Hash tables of Q2.1: ht_s (s_len slots), ht_p (2 * p_len), ht_d
// (2 * d_val_len from key 19920101), zeroed by the caller.
int dropin_q21_build(int* s_region, int* s_suppkey, int s_len, int* p_category, int* p_partkey, int* p_brand1,
                     int p_len, int* d_datekey, int* d_year, int d_len, int* ht_s, int* ht_p, int* ht_d,
                     int d_val_len) {
	constexpr int BT = 32, IPT = 8, TILE = BT * IPT;
	build_hashtable_s<BT, IPT><<<(s_len + TILE - 1) / TILE, BT>>>(s_region, s_suppkey, s_len, ht_s, s_len);
	build_hashtable_p<BT, IPT><<<(p_len + TILE - 1) / TILE, BT>>>(p_category, p_partkey, p_brand1, p_len, ht_p, p_len);
	build_hashtable_d<BT, IPT><<<(d_len + TILE - 1) / TILE, BT>>>(d_datekey, d_year, d_len, ht_d, d_val_len, 19920101);
	return static_cast<int>(cudaDeviceSynchronize());
}

// One probe version over packed columns at the file's bit widths
// (query_mtd.ssb: orderdate 16 after subtracting 19920101, partkey 20,
// suppkey 16, revenue 24 -- packed for v1, raw int32 for v2/v3); res holds
// 4 * 7000 ints, zeroed by the caller.
int dropin_q21_probe(int version, int* lo_orderdate, int* lo_partkey, int* lo_suppkey, int* lo_revenue, int lo_len,
                     int* ht_s, int s_len, int* ht_p, int p_len, int* ht_d, int d_len, int* res) {
	if (version == 1) {
		constexpr int BT = 32, IPT = 32;
		probe_v1<BT, IPT><<<(lo_len + BT * IPT - 1) / (BT * IPT), BT>>>(
		    lo_orderdate, lo_partkey, lo_suppkey, lo_revenue, lo_len, ht_s, s_len, ht_p, p_len, ht_d, d_len, res);
	} else {
		constexpr int BT = 32, IPT = 8;
		auto          k = version == 2 ? probe_v2<BT, IPT> : probe_v3<BT, IPT>;
		k<<<(lo_len + BT * IPT - 1) / (BT * IPT), BT>>>(lo_orderdate, lo_partkey, lo_suppkey, lo_revenue, lo_len,
		                                                ht_s, s_len, ht_p, p_len, ht_d, d_len, res);
	}
	return static_cast<int>(cudaDeviceSynchronize());
}

// Bit widths the file packs its columns with (query_mtd.ssb).
void dropin_q21_widths(int* out4) {
	out4[0] = query_mtd.ssb.lo_orderdate_bw;
	out4[1] = query_mtd.ssb.lo_partkey_bw;
	out4[2] = query_mtd.ssb.lo_chosen_suppkey_bw;
	out4[3] = query_mtd.ssb.lo_revenue_bw;
}

// Decoder error bits of this translation unit (cleared).
int dropin_q21_take_error(uint32_t* bits) { return static_cast<int>(fls::crystal::fls_crystal_take_error(bits)); }

} // extern "C"
