/*
 * ref_api.h -- TEST INFRASTRUCTURE ONLY.  C entry points into the reference's
 * own FastLanes code, compiled from its sources (see oracle/Makefile) into
 * oracle/_ref/libflsref.so.  Used by tests/ to pin the oracle, and by bench.py
 * as the reference CPU arm.  Nothing in the product links this library.
 */
#pragma once
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* fastlanes/src/pack.cpp:29607  generated::pack::fallback::scalar::pack(u32) */
void ref_pack_u32(const uint32_t* in, uint32_t* out, unsigned bw);
/* fastlanes/src/transpose.cpp:4110 / :5136  transpose_i / transpose_o (u32) */
void ref_transpose_i_u32(const uint32_t* in, uint32_t* out);
void ref_transpose_o_u32(const uint32_t* in, uint32_t* out);
/* fastlanes/src/unrsum.cpp:120  unrsum (u32) */
void ref_unrsum_u32(const uint32_t* in, uint32_t* out);

/* unpack.cuh:3330 normal::unpack, all 32 lanes: out[32*r + lane]; -1 on bad bw */
int ref_unpack_u32(const uint32_t* in, uint32_t* out, unsigned bw);
/* unpack_fused.cuh:3455 fused::unpack, lane registers scattered to out[32*r+lane] */
int ref_unpack_fused_u32(const uint32_t* in, uint32_t* out, unsigned bw);
/* rsum.cuh:4 d_rsum_32, all 32 lanes */
void ref_rsum_u32(const uint32_t* in, uint32_t* out, const uint32_t* base);
/* hardcoded_16.cuh:730 unpack_8_at_a_time::unpack on one quarter q of a vector:
 * in = vector + q*bw*8 words; out[32*r + lane] for r in 0..7.  Only bw in
 * {0,4,8,12,16,20} (the reference traps on others and its bw-24 routine writes
 * out of bounds); returns -1 for any other bw. */
int ref_unpack8_u32(const uint32_t* in_quarter, uint32_t* out256, unsigned bw);
/* hardcoded_16.cuh:390 hardcoded_16::unpack (bw 4,6,16,24) to uint16 lanes */
int ref_unpack_h16(const uint32_t* in, uint16_t* out, unsigned bw);

/* rle.hpp:29 VECTOR_RLE on one 1024-value vector (its debug printing is
 * discarded).  Returns the total number of dictionary entries. */
int ref_vector_rle(const int32_t* vec, uint8_t* idx, int32_t* dict, uint16_t* dict4);

/* tile_based/src/rlebinpack.cpp:9-146 rleBinPack (RFOR): n a multiple of 512;
 * value / run_length zero-initialised by the caller (the encoder adds into
 * them), of at least 4 + (n/512)*515 words; offsets of n/512 + 1 words.
 * sizes2 receives the words written to each stream. */
void ref_rfor_encode(const uint32_t* in, uint32_t n, uint32_t* value, uint32_t* run_length, uint32_t* val_offsets,
                     uint32_t* rl_offsets, uint32_t* sizes2);

/* generated/cuda/normal_t32_uf1/cuda_normal_t32_1024_uf1_unpack_helper.hpp:
 * the reference's golden arrays rand_arr_{bw}_b{bw}_w32_arr[1024], bw 0..32 */
const uint32_t* ref_helper_arr(unsigned bw);

/* Reference CPU arm for the fused queries: the reference's unpack (fused
 * form) per vector + the scalar query loops of fls_q11.cu:49-72 and
 * fls_q21.cu:50-77, OpenMP over vectors.  See ref_query.cpp. */
uint64_t ref_q11_sum(const uint32_t* date_p, unsigned date_bw, const uint32_t* disc_p, unsigned disc_bw,
                     const uint32_t* qty_p, unsigned qty_bw, const uint32_t* price_p, unsigned price_bw,
                     uint64_t n_rows, int32_t date_lo, int32_t date_hi, int32_t disc_lo, int32_t disc_hi,
                     int32_t qty_lt, int n_threads);
void ref_q21_groupby(const uint32_t* supp_p, unsigned supp_bw, const uint32_t* part_p, unsigned part_bw,
                     const uint32_t* date_p, unsigned date_bw, const uint32_t* rev_p, unsigned rev_bw,
                     uint64_t n_rows, const int32_t* ht_s, int32_t s_len, const int32_t* ht_p, int32_t p_len,
                     const int32_t* ht_d, int32_t d_len, int32_t d_keys_min, int32_t* res, int n_threads);
void ref_pack_column(const uint32_t* values, uint64_t n, unsigned bw, uint32_t* out, int n_threads);
uint64_t ref_decode_sum(const uint32_t* packed, unsigned bw, uint64_t n_vec, int n_threads);
uint64_t ref_decode(const uint32_t* packed, unsigned bw, uint64_t n_vec, uint32_t* out, int n_threads);

#ifdef __cplusplus
}
#endif
