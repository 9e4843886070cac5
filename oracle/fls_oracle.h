/*
 * fls_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's FastLanes decode + Crystal query path, used
 * as the parity checker for the CUDA library.  Only tests/, the smoke entry point
 * and bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Parity is pinned against the reference itself: tests compare every function
 * here with the reference's own code compiled from its sources
 * (oracle/_ref/libflsref.so: pack.cpp, transpose.cpp, unrsum.cpp, unpack.cuh,
 * unpack_fused.cuh, hardcoded_16.cuh, rsum.cuh, rle.hpp) and with its golden
 * arrays (generated/cuda/normal_t32_uf1/..._unpack_helper.hpp), and the
 * committed fixtures under tests/golden/ were produced by that library.
 *
 * All functions work on one 1024-value vector unless stated otherwise.
 */
#ifndef FLS_ORACLE_H
#define FLS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- layout ------------------------------------------------------------ */
/* Position of original index j (0..1023) in the FastLanes transposed order
 * (transpose.cpp:4110): lane (c>>1)|((c&1)<<4) holds chunk c = j/32 and
 * s = j%32 sits at row 4*(s&7) + {0,2,1,3}[s>>3]; position = 32*row + lane. */
uint32_t orc_tpos(uint32_t j);
void     orc_transpose_i(const uint32_t* in, uint32_t* out);   /* out[tpos(j)] = in[j] */
void     orc_untranspose(const uint32_t* in, uint32_t* out);   /* out[j] = in[tpos(j)] */

/* ---- bit-packing (pack.cpp:1954-1990, unpack.cuh:201-279) --------------- */
unsigned orc_bit_width(uint32_t max_value);
void     orc_pack(const uint32_t* in, uint32_t* out, unsigned bw);   /* out: 32*bw words */
void     orc_unpack(const uint32_t* in, uint32_t* out, unsigned bw); /* out: 1024 values */
/* rows [8q, 8q+8) of every lane from a quarter pointer in = vec + q*bw*8
 * (hardcoded_16.cuh:436-786; valid for bw % 4 == 0) */
void     orc_unpack_quarter(const uint32_t* in_quarter, uint32_t* out256, unsigned bw);

/* ---- delta over the transposed layout (unrsum.cpp:120, rsum.cuh:4) ------ */
void orc_unrsum(const uint32_t* in_transposed, uint32_t* out_deltas);
void orc_rsum(const uint32_t* deltas, uint32_t* out_transposed, const uint32_t* base32);

/* ---- reference RLE (rle.hpp:8-44) ---------------------------------------- */
/* Returns the number of dictionary entries; idx[j] is the per-256 local run
 * index, dict4[m] the dictionary offset of mini-vector m. */
int orc_vector_rle(const int32_t* vec, uint8_t* idx, int32_t* dict, uint16_t* dict4);

/* ---- per-vector schemes of the encoded-column format --------------------- */
enum {
	ORC_FOR = 0,   /* FOR + FastLanes bit-packing                          */
	ORC_DELTA = 1, /* transposed delta: 32 base words + packed deltas       */
	ORC_RLE = 2,   /* run index as bw-1 transposed delta + packed dict      */
	ORC_CONST = 3, /* one value, no payload                                 */
	ORC_DICT = 4   /* FastLanes bit-packed codes + packed sorted dictionary */
};

/* Encoded vector: payload words and the fields of its metadata entry.  The
 * payload word counts are always multiples of 4 (16-byte aligned vectors). */
typedef struct orc_vec {
	uint32_t scheme, bw, aux, n_words;
	int32_t  base;
} orc_vec;

/* Encode one vector with a given scheme (transposed selects the transposed
 * layout for FOR/DICT codes; DELTA and RLE are always transposed).  Returns 0
 * on success, -1 if the scheme cannot represent the vector (CONST). */
int orc_encode_vec(const int32_t* in, uint32_t scheme, int transposed, int round4, uint32_t* out, orc_vec* meta);
/* Decode one vector to ORIGINAL order. */
void orc_decode_vec(const uint32_t* in, const orc_vec* meta, int transposed, int32_t* out);
/* Exact encoded size in bytes (payload + 16 B metadata) of every scheme;
 * size[s] = UINT32_MAX when the scheme cannot represent the vector. */
void orc_scheme_sizes(const int32_t* in, uint32_t* size5);

/* ---- query path (fls_q11.cu:49-72, fls_q21.cu:50-77, join.cuh) ----------- */
/* Filter-aggregate over decoded int32 columns: sum of price*disc over rows with
 * date in [date_lo,date_hi], qty < qty_lt, disc in [disc_lo,disc_hi]. */
int64_t orc_filter_agg(const int32_t* date, const int32_t* disc, const int32_t* qty, const int32_t* price,
                       uint64_t n, int32_t date_lo, int32_t date_hi, int32_t disc_lo, int32_t disc_hi,
                       int32_t qty_lt);
/* Selective perfect-hash builds (join.cuh:190-334): PHT_1 stores the key,
 * PHT_2 stores (key, value) pairs; slot = (key - keys_min) % len. */
void orc_pht1_build(const int32_t* filter, int32_t filter_eq, const int32_t* keys, uint64_t n, int32_t* ht,
                    int32_t len, int32_t keys_min);
void orc_pht2_build(const int32_t* filter, int32_t filter_eq, const int32_t* keys, const int32_t* vals, uint64_t n,
                    int32_t* ht, int32_t len, int32_t keys_min);
/* Probe + group-by of fls_q21.cu probe_v1: res is int32[4*7000]; group g gets
 * res[4g]=year, res[4g+1]=brand and a uint64 revenue sum at res[4g+2]. */
void orc_q31_groupby(const int32_t* supp, const int32_t* cust, const int32_t* date, const int32_t* rev, uint64_t n,
                     const int32_t* ht_s, int32_t s_len, const int32_t* ht_c, int32_t c_len, const int32_t* ht_d,
                     int32_t d_len, int32_t d_keys_min, int32_t* res);
void orc_q41_groupby(const int32_t* supp, const int32_t* cust, const int32_t* part, const int32_t* date,
                     const int32_t* rev, const int32_t* cost, uint64_t n, const int32_t* ht_s, int32_t s_len,
                     const int32_t* ht_c, int32_t c_len, const int32_t* ht_p, int32_t p_len, const int32_t* ht_d,
                     int32_t d_len, int32_t d_keys_min, int32_t* res);
void orc_probe_groupby(const int32_t* supp, const int32_t* part, const int32_t* date, const int32_t* rev, uint64_t n,
                       const int32_t* ht_s, int32_t s_len, const int32_t* ht_p, int32_t p_len, const int32_t* ht_d,
                       int32_t d_len, int32_t d_keys_min, int32_t* res);

/* FastLanes bit-packing of 8-, 16- and 64-bit lanes (pack.cpp:29521,
 * 29552, 29710) and its inverse: 1024 values, 1024/T lanes, bw <= T. */
void orc_pack_8(const uint8_t* in, uint8_t* out, unsigned bw);
void orc_unpack_8(const uint8_t* in, uint8_t* out, unsigned bw);
void orc_pack_16(const uint16_t* in, uint16_t* out, unsigned bw);
void orc_unpack_16(const uint16_t* in, uint16_t* out, unsigned bw);
void orc_pack_64(const uint64_t* in, uint64_t* out, unsigned bw);
void orc_unpack_64(const uint64_t* in, uint64_t* out, unsigned bw);

/* Dimension predicates of the crystal-opt SSB builds (pred.cuh BlockPredEQ,
 * GTE/AndLTE, OrEQ): rows whose filter value lies in [lo0, hi0] or
 * [lo1, hi1] (filter NULL: every row); vals NULL builds a PHT_1. */
void orc_pht_build_ranges(const int32_t* filter, int32_t lo0, int32_t hi0, int32_t lo1, int32_t hi1,
                          const int32_t* keys, const int32_t* vals, uint64_t n, int32_t* ht, int32_t len,
                          int32_t keys_min);

/* The join + group-by loop every SSB join query of crystal-opt src/ssb
 * (q21-q43.cu) and fastlanes src/ssb (fls_q21/q31/q41.cu) instantiates,
 * over decoded columns: probes in order, group = (sum of PHT_2 payloads x
 * multipliers - group_sub) % n_groups in wrapping 32-bit arithmetic, key words
 * and a sum per record (sum_bits 64: int64 at words sum_slot..+1; 32: wrapping
 * int32 at word sum_slot), measure agg or agg - agg_sub. */
typedef struct orc_probe {
	const int32_t* col;
	const int32_t* ht;
	int32_t        len, keys_min, kind; /* kind 1: PHT_1, 2: PHT_2 */
} orc_probe;
void orc_join_groupby(uint64_t n, const orc_probe* probes, uint32_t n_probes, const int32_t* agg,
                      const int32_t* agg_sub, uint32_t n_keys, const int32_t* key_probe, const int32_t* key_mul,
                      const int32_t* key_slot, int32_t group_sub, int32_t n_groups, uint32_t stride,
                      uint32_t sum_slot, uint32_t sum_bits, int32_t* res);

/* ---- learned selector MLP, double precision (the gradient checker) ------- */
/* Parameter layout W1[64][16], b1[64], W2[64][64], b2[64], W3[5][64], b3[5];
 * ReLU hidden layers, mean softmax cross-entropy over the batch.  Writes the
 * loss and d(loss)/d(param) for every parameter (5573 doubles). */
#define ORC_MLP_N_PARAMS 5573
double orc_mlp_loss_grad(const float* params, const float* x, const uint8_t* y, uint32_t batch, double* grads);
/* 16 selector statistics of one vector (the same definitions as the library). */
void orc_vector_stats(const int32_t* v, float* f16);

/* ---- tile-based RLE (RFOR) ------------------------------------------------
 * tile_based/src/rlebinpack.cpp:9-146 (encoder; n a multiple of 512, the
 * caller pads with the last value as rlebinpack.cpp:217-219 does): both
 * streams start {512, 4, n, in[0]}; per tile the runs (value, length) with
 * min, bit width of (x - min) (ceil(log2(x+1)), :75-83), a block {min,
 * bw * 0x01010101, count, fields packed LSB first} whose packed part takes
 * max(1, ceil(count*bw/32)) words (:101-128); offsets[t] = block start,
 * offsets[tiles] = end (:141-142).  Streams must hold orc_rfor_bound(n) words;
 * returns the words written to each through n_val / n_rl.  Widths of 32 are
 * packed as the format defines (the reference shifts by 32 there).
 * orc_rfor_decode: the decoder's semantics (rlebinpack_kernel.cuh:20-145):
 * position p of a tile holds the value of the run whose cumulative length
 * first exceeds p.  Returns -1 on an inconsistent block. */
uint64_t orc_rfor_bound(uint64_t n);
void orc_rfor_encode(const uint32_t* in, uint64_t n, uint32_t* val, uint32_t* rl, uint32_t* val_off, uint32_t* rl_off,
                     uint64_t* n_val, uint64_t* n_rl);
int orc_rfor_decode(const uint32_t* val, const uint32_t* rl, const uint32_t* val_off, const uint32_t* rl_off,
                    uint64_t n, uint32_t* out);

/* ---- synthetic inputs (SplitMix64; shared with the Python tests) --------- */
uint64_t orc_splitmix64(uint64_t* state);

#ifdef __cplusplus
}
#endif
#endif
