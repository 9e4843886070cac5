/*
 * fls_gpu.h -- C ABI of the B200 (sm_100a) FastLanes decode + fused query library.
 *
 * Drop-in boundary for the hot path of FastLanesGPU: FastLanes vector decode
 * (1024-value interleaved bit-packing, FOR, delta over the transposed layout,
 * RLE) fused into Crystal-style tile query kernels.  The reference exposes this
 * path only as header templates and host functions; every entry point below
 * names the reference interface it replaces (paths relative to the reference
 * project root).
 *
 * Conventions
 *  - The caller owns every buffer.  Pointers documented as "device" must be
 *    device memory of the current device; "host" pointers are host memory.
 *  - Device calls are asynchronous and stream-ordered on `stream`
 *    (0 = legacy default stream).  They never allocate device memory.
 *  - Every call returns an fls_status.  Nothing calls exit(), traps the GPU or
 *    throws across the ABI.  Kernels validate per-vector metadata and record
 *    violations in a device error word instead of reading out of bounds;
 *    fls_check_device_error() synchronises `stream` and reports it.
 *  - Packed data buffers must be 16-byte aligned; every vector starts on a
 *    16-byte boundary (vector word offsets are multiples of 4).
 */
#ifndef FLS_GPU_H
#define FLS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* fls_stream_t; /* == cudaStream_t */

typedef enum fls_status {
	FLS_OK                = 0,
	FLS_ERR_INVALID_ARG   = 1, /* null pointer, bad enum, inconsistent sizes  */
	FLS_ERR_BAD_BW        = 2, /* bit width > 32 (or > 10 for dictionary codes) */
	FLS_ERR_ALIGNMENT     = 3, /* packed buffer or vector not 16-byte aligned  */
	FLS_ERR_CUDA          = 4, /* a CUDA runtime call failed (see message)      */
	FLS_ERR_DEVICE        = 5, /* a kernel reported bad metadata / bad input    */
	FLS_ERR_TIMEOUT       = 6, /* a bounded device wait gave up                 */
	FLS_ERR_UNSUPPORTED   = 7, /* combination not supported (e.g. layouts mix)  */
	FLS_ERR_CAPACITY      = 8, /* output / workspace too small                  */
	FLS_ERR_NO_DEVICE     = 9  /* no CUDA device, or not an sm_100 device       */
} fls_status;

/* Per-vector encodings.  FOR with bw 0 is a constant vector too; CONST is the
 * explicit zero-payload form. */
typedef enum fls_scheme {
	FLS_SCHEME_FOR   = 0, /* FOR base + FastLanes bit-packing (pack.cpp)             */
	FLS_SCHEME_DELTA = 1, /* 32 lane bases + packed deltas (transpose+unrsum+pack)   */
	FLS_SCHEME_RLE   = 2, /* run index as bw-1 transposed delta + packed run values  */
	FLS_SCHEME_CONST = 3, /* single value, no payload                                */
	FLS_SCHEME_DICT  = 4, /* bit-packed codes + packed sorted dictionary             */
	FLS_N_SCHEMES    = 5
} fls_scheme;

/* Row order of a column's 1024-value vectors.  NORMAL: lane i, row r holds
 * value 32r+i (pack.cpp).  TRANSPOSED: FastLanes transposed order
 * (transpose.cpp:4110); DELTA and RLE vectors are always transposed.  All
 * columns of one query must share a layout so that rows line up. */
typedef enum fls_layout { FLS_LAYOUT_NORMAL = 0, FLS_LAYOUT_TRANSPOSED = 1 } fls_layout;

/* Order of fls_decode_u32 output for transposed columns. */
typedef enum fls_order { FLS_ORDER_STORED = 0, FLS_ORDER_ORIGINAL = 1 } fls_order;

/* Per-vector metadata (16 bytes), the generalisation of the reference's
 * per-vector {bw, base, offset} arrays (fastlanes/src/ssb/compress_ssb.cu:372-454). */
typedef struct fls_vec_meta {
	uint64_t offset; /* word offset of the vector's payload (multiple of 4) */
	int32_t  base;   /* FOR base / minimum of the dictionary              */
	uint8_t  scheme; /* fls_scheme                                        */
	uint8_t  bw;     /* bit width of the packed values / deltas / dict    */
	uint16_t aux;    /* RLE: number of runs; DICT: dictionary size        */
} fls_vec_meta;

/* Largest column the library accepts: 2^40 values (2^30 vectors).  Larger
 * counts are refused with FLS_ERR_INVALID_ARG before any size arithmetic, so
 * that vector counts and payload sizes derived from n_values cannot wrap. */
#define FLS_MAX_VALUES (1ull << 40)

/* An encoded column resident in device memory.  With meta == NULL the column
 * is "uniform" like the reference's (one scheme/bw/base for all vectors,
 * vector v at word 32*bw*v for FOR, (32+32*bw)*v for DELTA). */
typedef struct fls_column {
	const uint32_t*     data;          /* device, 16-byte aligned packed words   */
	const fls_vec_meta* meta;          /* device, n_vec entries, or NULL         */
	uint64_t            n_values;      /* rows (the last vector may be partial)  */
	uint64_t            n_words;       /* size of data in words (bounds checks)  */
	uint32_t            layout;        /* fls_layout                             */
	uint32_t            scheme;        /* uniform columns: FOR or DELTA          */
	uint32_t            bw;            /* uniform columns                        */
	int32_t             base;          /* uniform columns (FOR)                  */
	uint32_t            max_vec_words; /* largest vector payload, in words       */
	uint32_t            scheme_mask;   /* bit s set if scheme s occurs           */
} fls_column;

/* ---------------------------------------------------------------- errors */

/* Human-readable text of the last error raised on this host thread. */
const char* fls_last_error(void);
/* Reads and clears the error word of `stream`: one atomic exchange on the
 * device, in stream order, takes the bits (a bit raised after it stays for the
 * next check), then the stream is synchronised.  Returns FLS_OK,
 * FLS_ERR_DEVICE or FLS_ERR_TIMEOUT.  The reference reports device-side
 * problems by exit() or trap (fastlanes/src/include/gpu_utils.h:41-58,
 * fls_gen/unpack/hardcoded_16.cuh:755). */
fls_status fls_check_device_error(fls_stream_t stream);
/* Gives `stream` an error word of its own (no reference counterpart): d_words
 * is a caller-owned pair of device uint32 words, zeroed by the caller and
 * 8-byte aligned.  Kernels this library launches on `stream` (on the current
 * device) record errors in d_words[0], and fls_check_device_error(stream)
 * reports exactly those; d_words[1] receives the bits each check takes out.
 * Streams without a word share the device's default word, so a check on one
 * of them may report another unbound stream's error.  Binding again replaces
 * the word; d_words == NULL removes the binding.  The binding is looked up
 * when a call enqueues its kernels: keep the words alive while work that was
 * enqueued with them may run. */
fls_status fls_bind_error_word(fls_stream_t stream, uint32_t* d_words);

/* Self-test of failure detection (no reference counterpart): one warp runs
 * the bounded mbarrier wait of the staged pipelines on a barrier that nothing
 * arrives on, gives up after `polls` (1..1024, about 20 us each at most) tries
 * and raises the timeout bit, so the next fls_check_device_error returns
 * FLS_ERR_TIMEOUT; the context stays usable.  Nothing faults or hangs. */
fls_status fls_selftest_bounded_wait(uint32_t polls, fls_stream_t stream);

/* ------------------------------------------------- host encoders (CPU) */

/* fastlanes/src/pack.cpp:29607 generated::pack::fallback::scalar::pack(u32):
 * packs one 1024-value vector into 32*bw words. */
fls_status fls_pack_u32(const uint32_t* in, uint32_t* out, uint8_t bw);
/* fastlanes/src/transpose.cpp:4110 transpose_i (u32). */
fls_status fls_transpose_i_u32(const uint32_t* in, uint32_t* out);
/* Inverse of transpose_i.  (The reference's transpose_o, transpose.cpp:5136,
 * applies the same permutation as transpose_i and is not its inverse.) */
fls_status fls_untranspose_u32(const uint32_t* in, uint32_t* out);
/* fastlanes/src/unrsum.cpp:120 unrsum (u32). */
fls_status fls_unrsum_u32(const uint32_t* in, uint32_t* out);
/* fastlanes/src/include/fls_gen/rle/rle.hpp:29 VECTOR_RLE; returns the total
 * dictionary size in *n_dict. */
fls_status fls_vector_rle(const int32_t* vec, uint8_t* idx, int32_t* dict, uint16_t* dict4, uint32_t* n_dict);

/* Worst-case payload words of a column of n values (any scheme mix). */
uint64_t fls_encode_bound_words(uint64_t n_values);

/* Encodes a uniform (reference-style) column: FOR with one base and bit width
 * for all vectors (fls_q11.cu:187-223), or DELTA with one delta bit width
 * (delta_shared_memory.cu:142-157).  bw = 0xff picks the smallest bit width
 * that fits; base is the FOR base (ignored for DELTA).  Values past n are
 * padded with the last value.  out: host, fls_encode_bound_words(n) words. */
fls_status fls_encode_uniform(const int32_t* values, uint64_t n, uint32_t scheme, uint32_t layout, uint8_t bw,
                              int32_t base, uint32_t* out, uint64_t* out_words, uint8_t* out_bw);

/* Encodes a column vector by vector with the given per-vector schemes
 * (schemes == NULL: every vector uses `scheme`).  Writes payload words and one
 * fls_vec_meta per vector (offsets relative to `out`).  round4 rounds FOR bit
 * widths up to a multiple of 4 (ssb_utils.h:222-239 find_bw).  A scheme that
 * cannot represent a vector (CONST on a non-constant vector) falls back to FOR. */
fls_status fls_encode_column(const int32_t* values, uint64_t n, const uint8_t* schemes, uint32_t scheme,
                             uint32_t layout, int round4, uint32_t* out, uint64_t* out_words, fls_vec_meta* meta,
                             uint32_t* max_vec_words, uint32_t* scheme_mask);

/* The same encoder on the GPU, for a column already in device memory:
 * identical words and metadata to fls_encode_column.  d_schemes (device, one
 * per vector) may be NULL to use `scheme` for every vector; an out-of-range
 * per-vector scheme is encoded as FOR and flagged in the device error word.
 * d_out holds at least fls_encode_bound_words(n) words; d_meta n_vec entries
 * (both 16-byte aligned); d_info (device uint64[3]) receives the payload words
 * written, the largest vector's words and the scheme mask.  d_workspace holds
 * fls_encode_gpu_workspace_bytes(n) bytes.  Stream-ordered; no reference
 * counterpart (the reference encodes on the host, pack.cpp:29607). */
uint64_t   fls_encode_gpu_workspace_bytes(uint64_t n);
fls_status fls_encode_column_gpu(const int32_t* d_values, uint64_t n, const uint8_t* d_schemes, uint32_t scheme,
                                 uint32_t layout, int round4, uint32_t* d_out, uint64_t out_capacity_words,
                                 fls_vec_meta* d_meta, uint64_t* d_info, void* d_workspace, uint64_t workspace_bytes,
                                 fls_stream_t stream);

/* FastLanes packing of the other lane widths: 1024 values of T bits in
 * 1024/T lanes, row r of lane i = value (1024/T)*r + i, masked to bw bits,
 * LSB-first, word k of lane i at out[(1024/T)*k + i]; every width has
 * 128-byte rows (128*bw bytes per vector).  fastlanes/src/pack.cpp:29521 (u8),
 * 29552 (u16), 29710 (u64); the inverses are those declared in
 * fls_gen/unpack/unpack.hpp:7-10 (the reference has no host body for them). */
fls_status fls_pack_u8(const uint8_t* in, uint8_t* out, uint8_t bw);
fls_status fls_pack_u16(const uint16_t* in, uint16_t* out, uint8_t bw);
fls_status fls_pack_u64(const uint64_t* in, uint64_t* out, uint8_t bw);
fls_status fls_unpack_u8(const uint8_t* in, uint8_t* out, uint8_t bw);
fls_status fls_unpack_u16(const uint16_t* in, uint16_t* out, uint8_t bw);
fls_status fls_unpack_u64(const uint64_t* in, uint64_t* out, uint8_t bw);
/* A column of n values of value_bits (8, 16, 32, 64) bits, minus `base`
 * (modulo 2^value_bits), packed vector after vector at bw bits (the last vector
 * padded with the last value): ceil(n/1024) * 128*bw bytes.  FLS_ERR_BAD_BW if
 * a value does not fit.  Host memory. */
fls_status fls_pack_column(const void* in, uint64_t n, uint32_t value_bits, uint8_t bw, uint64_t base, void* out);
/* GPU decode of such a column (d_in, 16-byte aligned): d_out (optional,
 * ceil(n/1024)*1024 values of the column's width) receives every vector with
 * the base added modulo 2^T, *d_sum (optional, device) the uint64 sum of the n
 * values (modulo 2^64).  The reference decodes 32-bit lanes only on the GPU
 * (fls_gen/unpack/unpack.cuh); 32-bit columns use fls_decode_u32. */
fls_status fls_decode_u8(const uint8_t* d_in, uint64_t n, uint8_t bw, uint8_t base, uint8_t* d_out, uint64_t* d_sum,
                         fls_stream_t stream);
fls_status fls_decode_u16(const uint16_t* d_in, uint64_t n, uint8_t bw, uint16_t base, uint16_t* d_out,
                          uint64_t* d_sum, fls_stream_t stream);
fls_status fls_decode_u64(const uint64_t* d_in, uint64_t n, uint8_t bw, uint64_t base, uint64_t* d_out,
                          uint64_t* d_sum, fls_stream_t stream);

/* Encoded-column container: the payload words and per-vector metadata of a
 * column with HOST pointers (data, meta) in one byte string --
 * [payload][zero pad to 16 B][metadata][96-byte footer: descriptor, CRC-32C
 * of payload, metadata and footer, version 2, magic "FLSCOLv1"] -- so encoded columns
 * can be stored and read back without re-encoding.  The reference keeps raw
 * int32 columns on disk (crystal_ssb_utils.h:108-127 storeColumn /
 * loadColumn) and re-encodes them each run (compress_ssb.cu:357-454).
 * fls_column_open_container checks the footer, the three checksums and every
 * vector's metadata against the payload (FLS_ERR_INVALID_ARG if damaged,
 * FLS_ERR_UNSUPPORTED for another version) and fills `col` with pointers into
 * `buf` (16-byte aligned); copy data and meta to the device to query it. */
uint64_t   fls_column_container_bytes(const fls_column* col);
fls_status fls_column_write_container(const fls_column* col, void* out, uint64_t out_bytes, uint64_t* written);
fls_status fls_column_open_container(const void* buf, uint64_t bytes, fls_column* col);

/* ------------------------------------------------------------ RFOR
 * The reference's tile-based run-length format ("RFOR", tile_based/src/
 * rlebinpack.cpp:9-146, decoded by LoadRBinPack in tile_based/src/include/
 * rlebinpack_kernel.cuh:20-145): values in tiles of 512; per tile the runs'
 * values and lengths, each FOR-packed in its own stream.  Both streams start
 * with a 4-word header {512, 4, rows encoded, first value}; tile t's block in
 * a stream starts at word offsets[t]: {minimum, bit width in each of the 4
 * bytes, run count, then the count fields (x - minimum) packed LSB first, field
 * i at bit i*bw, max(1, ceil(count*bw/32)) words}.  offsets has one entry per
 * tile plus the end.  The rows are padded to whole tiles with the last value
 * (as the reference pads, rlebinpack.cpp:219).  The reference's encoder
 * packs 32-bit fields with a shift by 32 (undefined in C++); this encoder
 * packs them as the format defines.
 *
 * fls_rfor_bound_words: words one stream may take for n rows.
 * fls_rfor_encode (host): into caller buffers of that bound (values, run
 * lengths) and of (n+511)/512 + 1 words (each offsets array).
 * fls_rfor_decode_u32 / fls_rfor_decode_sum_u32 (device): one warp per tile;
 * a tile whose block is inconsistent (counts, widths, offsets, run lengths
 * not summing to the tile) is skipped and flagged (fls_check_device_error). */
typedef struct fls_rfor_column {
	const uint32_t* values;      /* device: value stream        */
	const uint32_t* run_lengths; /* device: run-length stream   */
	const uint32_t* val_offsets; /* device: tiles + 1 words     */
	const uint32_t* rl_offsets;  /* device: tiles + 1 words     */
	uint64_t        n_values;    /* rows (the last tile may be partial) */
	uint64_t        n_val_words; /* size of the value stream (bounds checks) */
	uint64_t        n_rl_words;  /* size of the run-length stream */
} fls_rfor_column;
#define FLS_RFOR_TILE 512
uint64_t   fls_rfor_bound_words(uint64_t n);
fls_status fls_rfor_encode(const uint32_t* values, uint64_t n, uint32_t* val_stream, uint32_t* rl_stream,
                           uint32_t* val_offsets, uint32_t* rl_offsets, uint64_t* n_val_words, uint64_t* n_rl_words);
fls_status fls_rfor_decode_u32(const fls_rfor_column* col, uint32_t* d_out, fls_stream_t stream);
fls_status fls_rfor_decode_sum_u32(const fls_rfor_column* col, uint64_t* d_sum, fls_stream_t stream);

/* Exhaustive per-vector encoder (the selector's labels and regret): exact encoded size in
 * bytes (payload + 16 B metadata) of every scheme for every vector
 * (sizes: n_vec*5, UINT32_MAX = not representable) and the argmin scheme, ties
 * broken by the measured decode-cost order CONST < FOR < DELTA < RLE < DICT. */
fls_status fls_encode_exhaustive(const int32_t* values, uint64_t n, uint32_t* sizes, uint8_t* best, int n_threads);

/* The 16 per-vector statistics the learned selector reads (n_vec*16 floats). */
fls_status fls_vector_stats(const int32_t* values, uint64_t n, float* stats16, int n_threads);

/* ------------------------------------------------------ decode (device) */

/* fastlanes/src/include/fls_gen/unpack/unpack.cuh:3436 unpack_global and
 * fastlanes/src/delta_global_memory.cu:24 (delta to global memory): decodes
 * every vector of `col` into d_out (n_vec*1024 values, device).  Transposed
 * columns are written in stored (transposed) order, as the reference does, or
 * in original order. */
fls_status fls_decode_u32(const fls_column* col, uint32_t* d_out, uint32_t order, fls_stream_t stream);

/* fastlanes/src/bitpack_shared_memory.cu:21 / bitpack_register.cu:21 /
 * delta_shared_memory.cu:24 QueryKernel: decode fused with a sum; *d_sum
 * (device) receives the uint64 sum of all n_values decoded values. */
fls_status fls_decode_sum_u32(const fls_column* col, uint64_t* d_sum, fls_stream_t stream);

/* ------------------------------------------------------ queries (device) */

#define FLS_MAX_QUERY_COLS 8
#define FLS_MAX_FILTERS    4
#define FLS_MAX_PROBES     4

typedef struct fls_filter {
	uint32_t col; /* index into cols                        */
	int32_t  lo;  /* keep rows with lo <= value <= hi (int32) */
	int32_t  hi;
} fls_filter;

/* fastlanes/src/ssb/fls_q11.cu:29-81 QueryKernel_v1: filters (BlockPred*,
 * crystal-opt/pred.cuh) ANDed together, then sum(a) or sum(a*b) in int64
 * over the selected rows (BlockSum, crystal-opt/reduce.cuh:26). */
typedef struct fls_filter_agg_desc {
	const fls_column* cols; /* host array of n_cols column descriptors */
	uint32_t          n_cols;
	fls_filter        filters[FLS_MAX_FILTERS];
	uint32_t          n_filters;
	int32_t           agg_a; /* column summed; -1 = count rows            */
	int32_t           agg_b; /* if >= 0: sum of a*b                       */
} fls_filter_agg_desc;

/* *d_result (device int64) receives the aggregate. */
fls_status fls_query_filter_agg(const fls_filter_agg_desc* desc, int64_t* d_result, fls_stream_t stream);

/* crystal-opt/join.cuh:190-334 BlockBuildSelectivePHT_1/_2 as driven by
 * fls_q21.cu:197-263 build_hashtable_{s,p,d}: rows with
 * (d_filter == NULL || d_filter[i] == filter_eq) insert key (PHT_1, d_vals ==
 * NULL: ht[h] = key) or (key, value) (PHT_2: ht[2h] = key, ht[2h+1] = value) at
 * h = (key - keys_min) % ht_len.  d_ht (device, ht_len or 2*ht_len int32) must
 * be zeroed by the caller (fls_q21.cu:293-297). */
fls_status fls_pht_build(const int32_t* d_filter, int32_t filter_eq, const int32_t* d_keys, const int32_t* d_vals,
                         uint64_t n, int32_t* d_ht, int32_t ht_len, int32_t keys_min, fls_stream_t stream);
/* The same build with the dimension predicates of the other SSB queries
 * (crystal-opt/pred.cuh BlockPredEQ/GTE/AndLTE/OrEQ as used by the builds of
 * crystal-opt src/ssb/q22.cu:147-154, q33.cu:102-109, q42.cu:162-171): rows
 * with lo0 <= d_filter[i] <= hi0 or lo1 <= d_filter[i] <= hi1 (an empty range,
 * lo > hi, selects nothing; d_filter == NULL selects every row). */
fls_status fls_pht_build_ranges(const int32_t* d_filter, int32_t lo0, int32_t hi0, int32_t lo1, int32_t hi1,
                                const int32_t* d_keys, const int32_t* d_vals, uint64_t n, int32_t* d_ht,
                                int32_t ht_len, int32_t keys_min, fls_stream_t stream);

typedef struct fls_probe {
	uint32_t       col;      /* probed foreign-key column                        */
	const int32_t* ht;       /* device hash table                                */
	int32_t        ht_len;   /* slots                                            */
	int32_t        keys_min; /* HASH(X,Y,Z) = (X-Z)%Y, crystal-opt/join.cuh:26     */
	int32_t        kind;     /* 1 = PHT_1 (semi-join), 2 = PHT_2 (returns value)  */
} fls_probe;

/* fastlanes/src/ssb/fls_q21.cu:21-78 probe_v1: probes in order (each AND-ed
 * into the selection), then group g = (val[key_a]*group_mul + val[key_b] -
 * group_sub) % n_groups with val[] the PHT_2 payloads, and the reference's
 * result layout: d_res[4g] = val[key_b], d_res[4g+1] = val[key_a], and an
 * int64 sum of column agg at d_res[4g+2..3].  d_res (device, 4*n_groups int32)
 * is zeroed by this call. */
typedef struct fls_join_agg_desc {
	const fls_column* cols;
	uint32_t          n_cols;
	fls_probe         probes[FLS_MAX_PROBES];
	uint32_t          n_probes;
	uint32_t          agg_col;
	int32_t           key_a, key_b; /* indices into probes (kind 2)  */
	int32_t           group_mul, group_sub, n_groups;
} fls_join_agg_desc;

fls_status fls_query_probe_groupby(const fls_join_agg_desc* desc, int32_t* d_res, fls_stream_t stream);

/* The general form of the join + group-by kernels (fls_q21.cu probe_v1,
 * fls_q31.cu:28-93 probe_v1, fls_q41.cu:27-112 probe_v1): probes in order,
 * then group g = (sum over keys of payload[key_probe[k]] * key_mul[k] -
 * group_sub) % n_groups (wrapping 32-bit arithmetic) over 1..3 PHT_2 payloads,
 * and a record of res_stride int32 words per group: payload k at word
 * key_slot[k] (-1: not written) and the int64 sum of the measure at word
 * sum_slot.  The measure is cols[agg_col], or cols[agg_col] - cols[agg_sub_col]
 * as an int32 difference (fls_q41.cu:101) when agg_sub_col >= 0.  Examples:
 * Q2.1 keys (brand x7, year x1), sub 1992, stride 4, slots (1, 0), sum 2;
 * Q3.1 keys (s_nation x175, c_nation x7, year x1), 4375 groups, stride 6,
 * slots (2, 1, 0), sum 4; Q4.1 keys (c_nation x7, year x1), 175 groups,
 * stride 4, slots (1, 0), sum 2, measure revenue - supplycost.  sum_bits 32
 * keeps a wrapping int32 sum in word sum_slot instead (crystal-opt
 * src/ssb/q32.cu:95-101, q33, q34: stride 4, sum word 3).  d_res (device,
 * n_groups * res_stride int32, 8-byte aligned) is zeroed by the call. */
#define FLS_MAX_GROUP_KEYS 3
typedef struct fls_join_groupby_desc {
	const fls_column* cols;
	uint32_t          n_cols;
	fls_probe         probes[FLS_MAX_PROBES];
	uint32_t          n_probes;
	uint32_t          agg_col;
	int32_t           agg_sub_col;
	uint32_t          n_keys;
	int32_t           key_probe[FLS_MAX_GROUP_KEYS];
	int32_t           key_mul[FLS_MAX_GROUP_KEYS];
	int32_t           key_slot[FLS_MAX_GROUP_KEYS];
	int32_t           group_sub, n_groups;
	uint32_t          res_stride, sum_slot;
	uint32_t          sum_bits; /* 64 (or 0): int64 at words sum_slot, +1; 32: int32 at word sum_slot */
} fls_join_groupby_desc;

fls_status fls_query_join_groupby(const fls_join_groupby_desc* desc, int32_t* d_res, fls_stream_t stream);

/* Optional device workspace of the join + group-by calls.  The specialised
 * kernels keep the presence bitmaps of large hash tables in shared memory;
 * with a workspace of fls_join_workspace_bytes(desc) bytes (16-byte aligned)
 * one small kernel builds them once per call and every CTA copies them,
 * without one each CTA builds them from the tables (reading every table it
 * stages whole).  0 when the query stages no bitmap.  Results are identical
 * either way; the library allocates nothing.  A non-null workspace smaller
 * than required returns FLS_ERR_CAPACITY. */
uint64_t   fls_join_workspace_bytes(const fls_join_groupby_desc* desc);
uint64_t   fls_probe_workspace_bytes(const fls_join_agg_desc* desc);
fls_status fls_query_join_groupby_ws(const fls_join_groupby_desc* desc, int32_t* d_res, void* d_workspace,
                                     uint64_t workspace_bytes, fls_stream_t stream);
fls_status fls_query_probe_groupby_ws(const fls_join_agg_desc* desc, int32_t* d_res, void* d_workspace,
                                      uint64_t workspace_bytes, fls_stream_t stream);

/* ------------------------------------ batched persistent execution (device) */

/* One filter-aggregate query of a batch: rows with lo <= cols[col] <= hi,
 * sum of cols[agg_col] (same length and layout) and the row count. */
typedef struct fls_batch_query {
	uint32_t col;
	int32_t  lo, hi;
	uint32_t agg_col;
	uint64_t n_values; /* filled in by fls_batch_create */
} fls_batch_query;

/* Host-side plan of a batch: the queries cut into work items of chunk_vectors
 * vectors.  No reference counterpart (the reference launches one grid per
 * query, fls_q11.cu:150-160). */
typedef struct fls_batch fls_batch;
fls_status fls_batch_create(const fls_column* cols, uint32_t n_cols, const fls_batch_query* queries,
                            uint32_t n_queries, uint32_t chunk_vectors, fls_batch** out);
uint64_t   fls_batch_workspace_bytes(const fls_batch* batch);
uint32_t   fls_batch_items(const fls_batch* batch);
/* Copies the plan into a caller-provided device workspace (synchronises
 * `stream`); the batch keeps using that workspace. */
fls_status fls_batch_upload(fls_batch* batch, void* d_workspace, uint64_t workspace_bytes, fls_stream_t stream);
/* Runs every query in one persistent launch: d_results (device int64[2*n_queries])
 * receives {sum, count} per query.  Only memsets and one kernel launch are
 * enqueued, so the call can be captured into a CUDA graph. */
fls_status fls_batch_run(const fls_batch* batch, int64_t* d_results, fls_stream_t stream);
void       fls_batch_destroy(fls_batch* batch);

/* ----------------------------------- learned encoding selection (device) */

/* A 16-64-64-5 FP32 MLP reads 16 per-vector statistics and scores the five
 * schemes; the exhaustive encoder (fls_encode_exhaustive) labels its training
 * vectors and remains the fallback for low-confidence picks.  Any pick is
 * lossless: the encoder recomputes bit widths exactly.  No reference
 * counterpart (the reference picks encodings by hand, ssb_utils.h:37-83).
 * Parameters: W1[64][16], b1[64], W2[64][64], b2[64], W3[5][64], b3[5]. */
#define FLS_MLP_IN       16
#define FLS_MLP_HIDDEN   64
#define FLS_MLP_OUT      5
#define FLS_MLP_N_PARAMS (64 * 16 + 64 + 64 * 64 + 64 + 5 * 64 + 5)

/* The statistics of fls_vector_stats, computed on the device from device
 * values (n_vec*16 floats, bit-identical to the host version). */
fls_status fls_vector_stats_gpu(const int32_t* d_values, uint64_t n, float* d_stats, fls_stream_t stream);
/* He-uniform initialisation from a seed. */
fls_status fls_mlp_init(float* d_params, uint64_t seed, fls_stream_t stream);
/* Device workspace needed by fls_mlp_gradients for a batch. */
uint64_t fls_mlp_workspace_bytes(uint32_t batch);
/* Mean softmax cross-entropy of a batch and its gradient w.r.t. every
 * parameter (d_grads: FLS_MLP_N_PARAMS floats; d_loss optional). */
fls_status fls_mlp_gradients(const float* d_params, const float* d_x, const uint8_t* d_labels, uint32_t batch,
                             void* d_workspace, uint64_t workspace_bytes, float* d_grads, float* d_loss,
                             fls_stream_t stream);
/* fls_mlp_gradients without a workspace argument: no counterpart in the
 * reference.  It is for callers that cannot allocate device memory -- for
 * example a host engine whose device memory all comes from its own fixed pool,
 * or an ingest loop that must not pay cudaMalloc's implicit device-wide
 * synchronisation.  The activation scratch is a static device array of this
 * library, FLS_MLP_STATIC_MAX_BATCH x 261 floats (about 2.1 MB), which every
 * device that loads the library holds until the process exits.  The caller
 * still passes the parameters, inputs, labels and the gradient / loss outputs.
 *   - batch > FLS_MLP_STATIC_MAX_BATCH returns FLS_ERR_CAPACITY (nothing runs).
 *   - The first call on a device looks up the array's device address (with
 *     that device current); make that first call before any stream capture.
 *     The address is kept for the life of the process: resetting the device
 *     (cudaDeviceReset, or a reset of its primary context) after that first
 *     call is not supported, since the array may then live elsewhere.
 *   - It calls no cudaMalloc / cudaFree.  All calls share the one array: each
 *     call writes every scratch element it later reads, so nothing carries
 *     over between calls, but calls that overlap on the GPU (other streams,
 *     other host threads) race on it and must be serialised by the caller. */
#define FLS_MLP_STATIC_MAX_BATCH 2048
fls_status fls_mlp_gradients_static(const float* d_params, const float* d_x, const uint8_t* d_labels, uint32_t batch,
                                    float* d_grads, float* d_loss, fls_stream_t stream);
/* One Adam update (t = 1-based step; d_m, d_v: moment buffers). */
fls_status fls_mlp_adam_step(float* d_params, const float* d_grads, float* d_m, float* d_v, float lr, float beta1,
                             float beta2, float eps, uint32_t t, fls_stream_t stream);
/* Inference: optional softmax probabilities (n*5), argmax scheme and its
 * probability (the confidence used for the exhaustive fallback). */
fls_status fls_mlp_infer(const float* d_params, const float* d_x, uint64_t n, float* d_probs, uint8_t* d_best,
                         float* d_conf, fls_stream_t stream);

/* The learned encoder in one call, entirely on the device (no reference
 * counterpart): the statistics of fls_vector_stats_gpu, the network's picks
 * (fls_mlp_infer with d_params), and for each vector whose confidence is below
 * `threshold` the exhaustive choice computed on the device -- the exact sizes
 * of fls_encode_exhaustive under the selector's label rule, argmin of
 * size x (1 + kappa (decode cost - 1)), costs FOR 1, DELTA 1.5, RLE 2,
 * CONST 1, DICT 4.5, ties to the cheaper decode -- then the column encoded by
 * fls_encode_column_gpu with those per-vector schemes (no FOR rounding).
 * d_info (device uint64[4]): fls_encode_column_gpu's three values and the
 * number of vectors that fell back to the exhaustive choice.  d_schemes
 * (optional, device, one per vector) receives the choices.  d_workspace:
 * fls_encode_learned_workspace_bytes(n) bytes, 256-byte aligned. */
uint64_t   fls_encode_learned_workspace_bytes(uint64_t n);
fls_status fls_encode_learned_gpu(const int32_t* d_values, uint64_t n, const float* d_params, float threshold,
                                  double kappa, uint32_t layout, uint32_t* d_out, uint64_t out_capacity_words,
                                  fls_vec_meta* d_meta, uint64_t* d_info, uint8_t* d_schemes, void* d_workspace,
                                  uint64_t workspace_bytes, fls_stream_t stream);

/* ------------------------------------- reference-shaped kernels (device) */

/* fastlanes/src/ssb/fls_q11.cu:29-81 QueryKernel_v1, written against the
 * drop-in primitive API (include/fls_crystal.cuh) and launched like the
 * reference: one 32-thread CTA per 1024-value vector.  Columns are uniform
 * bit-packed int32 columns (device, n_vec*32*bw words each).  Selection:
 * date > date_gt AND date < date_lt AND qty < qty_lt AND disc >= disc_ge AND
 * disc <= disc_le; *d_revenue = sum(price * disc) over selected rows. */
fls_status fls_crystal_q11(const int32_t* date, uint32_t date_bw, const int32_t* disc, uint32_t disc_bw,
                           const int32_t* qty, uint32_t qty_bw, const int32_t* price, uint32_t price_bw,
                           uint64_t n_rows, int32_t date_gt, int32_t date_lt, int32_t qty_lt, int32_t disc_ge,
                           int32_t disc_le, uint64_t* d_revenue, fls_stream_t stream);

/* fastlanes/src/ssb/fls_q21.cu:21-78 probe_v1 on the drop-in primitive API:
 * supplier PHT_1, part PHT_2 (brand), date PHT_2 (year), group
 * (brand*7 + year-1992) % 7000 into d_res (device int32[4*7000], zeroed here). */
fls_status fls_crystal_q21_probe(const int32_t* suppkey, uint32_t supp_bw, const int32_t* partkey, uint32_t part_bw,
                                 const int32_t* orderdate, uint32_t date_bw, const int32_t* revenue, uint32_t rev_bw,
                                 uint64_t n_rows, const int32_t* ht_s, int32_t s_len, const int32_t* ht_p,
                                 int32_t p_len, const int32_t* ht_d, int32_t d_len, int32_t d_keys_min, int32_t* d_res,
                                 fls_stream_t stream);

/* --------------------------------------------------------- tuning */

/* Launch shape of the staged decode/query kernels: warps per CTA (<= 16),
 * pipeline stages per warp, CTAs per SM and the target bytes of one staged
 * tile of consecutive vectors (0 = library default for each).  Used by the
 * autotuner; applies to subsequent calls from all threads.  Until warps are
 * set here, the specialised join + group-by kernels (FLS_TUNE_JIT) use up to
 * 20 warps per CTA where shared memory allows, every other kernel 16. */
fls_status fls_set_launch_config(uint32_t warps_per_cta, uint32_t stages, uint32_t ctas_per_sm, uint32_t tile_bytes);
fls_status fls_get_launch_config(uint32_t* warps_per_cta, uint32_t* stages, uint32_t* ctas_per_sm,
                                 uint32_t* tile_bytes);

/* Other tuning parameters of the operators. */
typedef enum fls_tune_param {
	/* Operators evaluate whole vectors while some lane of a warp still has more
	 * than this many selected rows in its 32; at or below it they switch to a
	 * loop over the selected rows that reads only their fields.  Default 4;
	 * 0 restores the default. */
	FLS_TUNE_SPARSE_ROWS = 0,
	/* 1 (default): fls_query_filter_agg, fls_query_probe_groupby,
	 * fls_decode_sum_u32 and fls_decode_u32 (stored order) on uniform FOR
	 * columns run a kernel compiled at first use (NVRTC) for the exact shape
	 * (bit widths, filter or probe count and kinds, aggregate, warps per CTA),
	 * cached per shape in the process; any compile or load failure falls back
	 * to the general kernel.  0: always the general kernel.  Results are
	 * identical either way. */
	FLS_TUNE_JIT = 1,
	/* 1 (default): the specialised join + group-by kernels sum each CTA's rows
	 * in a direct-mapped cache of group-sum slots in shared memory (the group
	 * count rounded up to a power of two, at most 2048 slots; a group whose
	 * slot another group holds adds to its record directly) and add the
	 * slots to the group records once per CTA, instead of one global int64
	 * atomic per selected row (few live groups make those atomics contend).
	 * 0: one global atomic per row.  Results are identical either way. */
	FLS_TUNE_GROUP_SMEM = 2,
	/* 1 (default): the specialised join + group-by kernels leave the measure
	 * columns (aggregated and subtracted) in global memory and read their
	 * fields for the selected rows only; 0: they stage them whole with the
	 * probe columns.  Results are identical either way. */
	FLS_TUNE_LATE_MEASURE = 3,
	/* Shared-memory budget, in KB, of the specialised join kernels' hash
	 * tables (PHT_1 as bitmaps, PHT_2 verbatim or as presence bitmaps, placed
	 * in probe order while they fit; the others are probed in global memory).
	 * A larger budget keeps more tables on chip and leaves less room for the
	 * staged vectors, so fewer warps per CTA.  Default 72; 0 restores it; at
	 * most 144.  fls_join_workspace_bytes depends on it.  Results are
	 * identical either way. */
	FLS_TUNE_TABLE_KB = 4,
	/* 1: the specialised join kernels stage half vectors (rows 0..15 or
	 * 16..31 of every lane, half of each column's words) instead of whole
	 * ones, so that a stage takes half the shared memory and about twice the
	 * warps fit beside the hash tables; 0 (default): whole vectors.  Results
	 * are identical either way. */
	FLS_TUNE_HALF_VECTORS = 5
} fls_tune_param;
fls_status fls_set_tuning(uint32_t param, int64_t value);
fls_status fls_get_tuning(uint32_t param, int64_t* value);

/* Counters of the specialised-kernel cache (all threads of the process). */
typedef struct fls_jit_stats {
	uint64_t compiled; /* shapes compiled and loaded */
	uint64_t launches; /* launches of specialised kernels */
	uint64_t failures; /* shapes whose compile or load failed (general kernel used) */
	uint64_t cached;   /* shapes currently cached */
} fls_jit_stats;
fls_status fls_get_jit_stats(fls_jit_stats* out);
/* Compile log of the most recent failed specialisation ("" if none). */
const char* fls_jit_last_log(void);
/* Compiles (NVRTC, no device needed) the specialised kernel that
 * fls_query_filter_agg would run for this query, so that the first query does
 * not pay for it (e.g. before capturing a CUDA graph).  FLS_ERR_UNSUPPORTED if
 * the query does not qualify or the compile failed (fls_last_error has the
 * log). */
fls_status fls_jit_precompile(const fls_filter_agg_desc* desc);
/* The same for the kernel fls_query_probe_groupby / fls_query_join_groupby
 * would run. */
fls_status fls_jit_precompile_probe(const fls_join_agg_desc* desc);
fls_status fls_jit_precompile_join(const fls_join_groupby_desc* desc);

/* Number of kernels this library has launched in this process (all threads). */
uint64_t fls_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* FLS_GPU_H */
