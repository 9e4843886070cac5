// TEST INFRASTRUCTURE ONLY.  The reference's own Q4.1 kernels over
// per-vector bit widths (fastlanes/src/ssb/compress_ssb.cu, included where it
// lies, unchanged) compiled against this project's drop-in device headers
// (include/compat first on the include path).  Its probe reads lo_custkey and
// lo_orderdate with a bit width, base and word offset per 1024-value vector
// (quarter q of vector v at offset[v] + q*bw*8) through
// unpack_8_at_a_time::unpack_device, the other keys at fixed widths; its
// builds use BlockPredEQ, BlockPredOrEQ and BlockBuildSelectivePHT_1/_2.
// The launchers run them as the file's runQuery does (compress_ssb.cu:217-330).
#define main fls_ref_q41_main
#include "ssb/compress_ssb.cu"
#undef main

extern "C" {

// ht_s, ht_p: s_len / p_len slots; ht_c: 2 * c_len; ht_d: 2 * d_val_len from
// key 19920101; all zeroed by the caller.
int dropin_q41_build(int* s_region, int* s_suppkey, int s_len, int* p_mfgr, int* p_partkey, int p_len,
                     int* c_region, int* c_custkey, int* c_nation, int c_len, int* d_datekey, int* d_year, int d_len,
                     int* ht_s, int* ht_p, int* ht_c, int* ht_d, int d_val_len) {
	constexpr int BT = 32, IPT = 8, TILE = BT * IPT;
	build_hashtable_s<BT, IPT><<<(s_len + TILE - 1) / TILE, BT>>>(s_region, s_suppkey, s_len, ht_s, s_len);
	build_hashtable_p<BT, IPT><<<(p_len + TILE - 1) / TILE, BT>>>(p_mfgr, p_partkey, p_len, ht_p, p_len);
	build_hashtable_c<BT, IPT><<<(c_len + TILE - 1) / TILE, BT>>>(c_region, c_custkey, c_nation, c_len, ht_c, c_len);
	build_hashtable_d<BT, IPT><<<(d_len + TILE - 1) / TILE, BT>>>(d_datekey, d_year, d_len, ht_d, d_val_len, 19920101);
	return static_cast<int>(cudaDeviceSynchronize());
}

// res: 4 * 175 ints, zeroed by the caller.
int dropin_q41_probe(int* lo_orderdate, int* od_bw, int* od_base, int* od_offset, int* lo_partkey, int* lo_custkey,
                     int* ck_bw, int* ck_base, int* ck_offset, int* lo_suppkey, int* lo_revenue, int* lo_supplycost,
                     int lo_len, int* ht_p, int p_len, int* ht_s, int s_len, int* ht_c, int c_len, int* ht_d, int d_len,
                     int* res) {
	constexpr int BT = 32, IPT = 8;
	probe<BT, IPT><<<(lo_len + BT * IPT - 1) / (BT * IPT), BT>>>(
	    lo_orderdate, od_bw, od_base, od_offset, lo_partkey, lo_custkey, ck_bw, ck_base, ck_offset, lo_suppkey,
	    lo_revenue, lo_supplycost, lo_len, ht_p, p_len, ht_s, s_len, ht_c, c_len, ht_d, d_len, res);
	return static_cast<int>(cudaDeviceSynchronize());
}

// Fixed bit widths the file reads (query_mtd.ssb): suppkey, partkey, supplycost.
void dropin_q41_widths(int* out3) {
	out3[0] = query_mtd.ssb.lo_chosen_suppkey_bw;
	out3[1] = query_mtd.ssb.lo_partkey_bw;
	out3[2] = query_mtd.ssb.lo_chosen_supplycost_bw;
}

int dropin_q41_take_error(uint32_t* bits) { return static_cast<int>(fls::crystal::fls_crystal_take_error(bits)); }

} // extern "C"
