/*
 * fls_crystal.cuh -- device-side primitive API for kernel authors (header-only,
 * sm_100a).
 *
 * Same names, template parameters, argument order and semantics as the
 * reference's tile primitives and FastLanes decoders, re-implemented, so a
 * kernel written against the reference compiles against this header after
 * `using namespace fls::crystal;`:
 *
 *   InitFlags, BlockLoad, BlockPredLoad          crystal-opt/pred.cuh:7, load.cuh:56,89
 *   BlockPred{GT,LT,GTE,LTE,EQ}, BlockPredAnd*,   crystal-opt/pred.cuh:164-239
 *   BlockPredOrEQ
 *   BlockSum                                      crystal-opt/reduce.cuh:26-75
 *   BlockBuildSelectivePHT_1/_2                   crystal-opt/join.cuh:190-334
 *   BlockProbeAndPHT_1/_2, BlockProbeAndPHT_2_R_S crystal-opt/join.cuh:28-188,
 *                                                 fastlanes/join.cuh:3-82
 *   unpack_device (register form)                 fls_gen/unpack/unpack_fused.cuh:3455
 *   unpack_device_ptr (normal form)               fls_gen/unpack/unpack.cuh:3444
 *   unpack_8_at_a_time::, hardcoded::,            fls_gen/unpack/hardcoded_16.cuh:16-1206
 *   hardcoded_16:: unpack / unpack_device /
 *   load_registers / unpack_<bw>bw_32ow_32crw_1uf
 *   d_rsum_32                                     fls_gen/rsum/rsum.cuh:4
 *
 * include/compat/ holds headers under the reference's own paths
 * (crystal/crystal.cuh, crystal-opt/crystal.cuh, fastlanes/join.cuh,
 * fls_gen/unpack/{unpack,unpack_fused,hardcoded_16}.cuh, fls_gen/rsum/rsum.cuh)
 * that forward to this one: with include/compat first on the include path,
 * the reference's kernel sources compile as they are.
 *
 * Conventions kept from the reference: a tile is BLOCK_THREADS x
 * ITEMS_PER_THREAD items, item ITEM of thread t is row t + BLOCK_THREADS*ITEM
 * (striped); flags are int arrays; num_items guards the last tile;
 * HASH(X,Y,Z) = (X-Z) % Y; an empty PHT slot is 0.  Differences: unpack of any
 * bit width 0..32 (no trap on unsupported widths: the output is zero and bit 0
 * of the translation unit's decoder error word is set; 8-at-a-time decodes
 * every width whose quarter starts on a word boundary, bw % 4 == 0),
 * and BlockSum returns the block total to every thread.  The decoders compile
 * each bit width to constant shifts and masks (fls_device.cuh).
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../fastlanesgpu_b200/csrc/fls_device.cuh"

namespace fls {
namespace crystal {

#define FLS_HASH(X, Y, Z) (((X) - (Z)) % (Y))

// ------------------------------------------------------------ flags / loads

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void InitFlags(int (&selection_flags)[ITEMS_PER_THREAD]) {
#pragma unroll
	for (int i = 0; i < ITEMS_PER_THREAD; ++i) { selection_flags[i] = 1; }
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockLoad(const T* inp, T (&items)[ITEMS_PER_THREAD], int num_items) {
	const int t = threadIdx.x;
#pragma unroll
	for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
		const int row = t + BLOCK_THREADS * i;
		if (row < num_items) { items[i] = inp[row]; }
	}
}

// With the flag type as a template parameter (crystal-opt/load.cuh) or
// deduced (crystal/load.cuh's <T, BLOCK_THREADS, ITEMS_PER_THREAD>).
template <typename T, typename ST, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredLoad(const T* inp, T (&items)[ITEMS_PER_THREAD], int num_items,
                                              ST (&selection_flags)[ITEMS_PER_THREAD]) {
	const int t = threadIdx.x;
#pragma unroll
	for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
		const int row = t + BLOCK_THREADS * i;
		if (selection_flags[i] && row < num_items) { items[i] = inp[row]; }
	}
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD, typename ST>
__device__ __forceinline__ void BlockPredLoad(const T* inp, T (&items)[ITEMS_PER_THREAD], int num_items,
                                              ST (&selection_flags)[ITEMS_PER_THREAD]) {
	BlockPredLoad<T, ST, BLOCK_THREADS, ITEMS_PER_THREAD>(inp, items, num_items, selection_flags);
}

// ------------------------------------------------------------- predicates

namespace detail {
enum class Op { LT, GT, LTE, GTE, EQ };
template <Op O, typename T>
__device__ __forceinline__ bool cmp(const T& a, const T& b) {
	if constexpr (O == Op::LT) { return a < b; }
	if constexpr (O == Op::GT) { return a > b; }
	if constexpr (O == Op::LTE) { return a <= b; }
	if constexpr (O == Op::GTE) { return a >= b; }
	return a == b;
}
// mode 0: set, 1: and, 2: or -- rows past num_items keep their flag.
template <int MODE, Op O, typename T, typename ST, int BT, int IPT>
__device__ __forceinline__ void pred(const T (&items)[IPT], T compare, ST (&flags)[IPT], int num_items) {
	const int t = threadIdx.x;
#pragma unroll
	for (int i = 0; i < IPT; ++i) {
		if (t + BT * i < num_items) {
			const bool c = cmp<O>(items[i], compare);
			if constexpr (MODE == 0) { flags[i] = c; }
			if constexpr (MODE == 1) { flags[i] = flags[i] && c; }
			if constexpr (MODE == 2) { flags[i] = flags[i] || c; }
		}
	}
}
} // namespace detail

// Each predicate exists with both template parameter lists the reference
// uses: <T, BLOCK_THREADS, ITEMS_PER_THREAD> (crystal/pred.cuh, and most of
// crystal-opt/pred.cuh) and <T, ST, BLOCK_THREADS, ITEMS_PER_THREAD> with the
// flag type ST (crystal-opt/pred.cuh's BlockPredGT, BlockPredAndLT/LTE/GTE);
// explicit template arguments select the one that fits.
#define FLS_CRYSTAL_PRED(NAME, MODE, OP)                                                                               \
	template <typename T, typename ST, int BLOCK_THREADS, int ITEMS_PER_THREAD>                                      \
	__device__ __forceinline__ void NAME(T(&items)[ITEMS_PER_THREAD], T compare, ST(&selection_flags)[ITEMS_PER_THREAD], \
	                                    int num_items) {                                                             \
		detail::pred<MODE, detail::Op::OP, T, ST, BLOCK_THREADS, ITEMS_PER_THREAD>(items, compare, selection_flags,    \
		                                                                          num_items);                        \
	}                                                                                                                \
	template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD, typename ST>                                      \
	__device__ __forceinline__ void NAME(T(&items)[ITEMS_PER_THREAD], T compare, ST(&selection_flags)[ITEMS_PER_THREAD], \
	                                    int num_items) {                                                             \
		detail::pred<MODE, detail::Op::OP, T, ST, BLOCK_THREADS, ITEMS_PER_THREAD>(items, compare, selection_flags,    \
		                                                                          num_items);                        \
	}
FLS_CRYSTAL_PRED(BlockPredGT, 0, GT)
FLS_CRYSTAL_PRED(BlockPredLT, 0, LT)
FLS_CRYSTAL_PRED(BlockPredGTE, 0, GTE)
FLS_CRYSTAL_PRED(BlockPredLTE, 0, LTE)
FLS_CRYSTAL_PRED(BlockPredEQ, 0, EQ)
FLS_CRYSTAL_PRED(BlockPredAndGT, 1, GT)
FLS_CRYSTAL_PRED(BlockPredAndLT, 1, LT)
FLS_CRYSTAL_PRED(BlockPredAndGTE, 1, GTE)
FLS_CRYSTAL_PRED(BlockPredAndLTE, 1, LTE)
FLS_CRYSTAL_PRED(BlockPredAndEQ, 1, EQ)
FLS_CRYSTAL_PRED(BlockPredOrEQ, 2, EQ)
#undef FLS_CRYSTAL_PRED

// ------------------------------------------------------------- reductions

// Block-wide sum.  `shared` needs BLOCK_THREADS/32 elements.  Every thread
// receives the total (the reference guarantees it only to thread 0).
template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ T BlockSum(T item, T* shared) {
	constexpr int kWarps = (BLOCK_THREADS + 31) / 32;
	T             v      = item;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) { v += __shfl_xor_sync(0xffffffffu, v, o); }
	if constexpr (kWarps == 1) {
		return v;
	} else {
		__syncthreads();
		if ((threadIdx.x & 31) == 0) { shared[threadIdx.x >> 5] = v; }
		__syncthreads();
		T total = 0;
#pragma unroll
		for (int w = 0; w < kWarps; ++w) { total += shared[w]; }
		return total;
	}
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ T BlockSum(T (&items)[ITEMS_PER_THREAD], T* shared) {
	T s = 0;
#pragma unroll
	for (int i = 0; i < ITEMS_PER_THREAD; ++i) { s += items[i]; }
	return BlockSum<T, BLOCK_THREADS, ITEMS_PER_THREAD>(s, shared);
}

// ------------------------------------------------------- perfect hashing

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_1(K (&keys)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min, int num_items) {
	const int t = threadIdx.x;
#pragma unroll
	for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
		if (t + BLOCK_THREADS * i < num_items && selection_flags[i]) {
			const int h = FLS_HASH(keys[i], ht_len, keys_min);
			if (h >= 0) { atomicCAS(&ht[h], K(0), keys[i]); }
		}
	}
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_1(K (&keys)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         int num_items) {
	BlockBuildSelectivePHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, selection_flags, ht, ht_len, K(0), num_items);
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min, int num_items) {
	const int t = threadIdx.x;
#pragma unroll
	for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
		if (t + BLOCK_THREADS * i < num_items && selection_flags[i]) {
			const int h = FLS_HASH(keys[i], ht_len, keys_min);
			if (h >= 0) {
				atomicCAS(&ht[h << 1], K(0), keys[i]);
				ht[(h << 1) + 1] = res[i];
			}
		}
	}
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         int num_items) {
	BlockBuildSelectivePHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, res, selection_flags, ht, ht_len, K(0),
	                                                                num_items);
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_1(K (&items)[ITEMS_PER_THREAD], int (&selection_flags)[ITEMS_PER_THREAD],
                                                   const K* ht, int ht_len, K keys_min, int num_items) {
	const int t = threadIdx.x;
#pragma unroll
	for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
		if (t + BLOCK_THREADS * i < num_items && selection_flags[i]) {
			const int h        = FLS_HASH(items[i], ht_len, keys_min);
			selection_flags[i] = (h >= 0 && ht[h] != K(0)) ? 1 : 0;
		}
	}
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_1(K (&items)[ITEMS_PER_THREAD], int (&selection_flags)[ITEMS_PER_THREAD],
                                                   const K* ht, int ht_len, int num_items) {
	BlockProbeAndPHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(items, selection_flags, ht, ht_len, K(0), num_items);
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                   int (&selection_flags)[ITEMS_PER_THREAD], const K* ht, int ht_len,
                                                   K keys_min, int num_items) {
	const int t = threadIdx.x;
#pragma unroll
	for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
		if (t + BLOCK_THREADS * i < num_items && selection_flags[i]) {
			const int h = FLS_HASH(keys[i], ht_len, keys_min);
			uint64_t  slot = 0;
			if (h >= 0) { slot = *reinterpret_cast<const uint64_t*>(&ht[h << 1]); }
			if (slot != 0) {
				res[i] = static_cast<V>(slot >> 32);
			} else {
				selection_flags[i] = 0;
			}
		}
	}
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                   int (&selection_flags)[ITEMS_PER_THREAD], const K* ht, int ht_len,
                                                   int num_items) {
	BlockProbeAndPHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, res, selection_flags, ht, ht_len, K(0), num_items);
}

// Probe writing the payload into a tile array (shared memory) at the item's
// striped position (fastlanes/join.cuh:3-82).
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_2_R_S(K (&keys)[ITEMS_PER_THREAD],
                                                       V (&res)[BLOCK_THREADS * ITEMS_PER_THREAD],
                                                       int (&selection_flags)[ITEMS_PER_THREAD], const K* ht,
                                                       int ht_len, K keys_min, int num_items) {
	const int t = threadIdx.x;
#pragma unroll
	for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
		if (t + BLOCK_THREADS * i < num_items && selection_flags[i]) {
			const int h    = FLS_HASH(keys[i], ht_len, keys_min);
			uint64_t  slot = 0;
			if (h >= 0) { slot = *reinterpret_cast<const uint64_t*>(&ht[h << 1]); }
			if (slot != 0) {
				res[BLOCK_THREADS * i + t] = static_cast<V>(slot >> 32);
			} else {
				selection_flags[i] = 0;
			}
		}
	}
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_2_R_S(K (&keys)[ITEMS_PER_THREAD],
                                                       V (&res)[BLOCK_THREADS * ITEMS_PER_THREAD],
                                                       int (&selection_flags)[ITEMS_PER_THREAD], const K* ht,
                                                       int ht_len, int num_items) {
	BlockProbeAndPHT_2_R_S<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, res, selection_flags, ht, ht_len, K(0),
	                                                              num_items);
}

// ---------------------------------------------------------------- decoders

// Error word of the decoders in this translation unit: bit 0 is set when a
// decoder is asked for a bit width it cannot decode there (the reference's
// 8-at-a-time decoder traps instead, hardcoded_16.cuh:753-755); the output is
// then zero.  Read and cleared on the host with fls_crystal_take_error().
static __device__ uint32_t fls_crystal_error_word;

namespace detail {
__device__ __forceinline__ void unsupported_width() { atomicOr(&fls_crystal_error_word, 1u); }

template <int BW, typename T>
__device__ __forceinline__ void unpack_regs_bw(const uint32_t* in, uint32_t lane, T (&out)[32]) {
	fls::dev::LaneWords<BW> lw;
#pragma unroll
	for (int k = 0; k < BW; ++k) { lw.w[k] = in[32 * k + lane]; }
#pragma unroll
	for (int r = 0; r < 32; ++r) { out[r] = static_cast<T>(fls::dev::extract<BW>(lw, r)); }
}

// Register form through a pointer: out[r] = row r of the calling lane.
template <int BW, typename T>
__device__ __forceinline__ void unpack_rows_ptr(const uint32_t* in, T* out) {
	T regs[32];
	unpack_regs_bw<BW>(in, threadIdx.x & 31u, regs);
#pragma unroll
	for (int r = 0; r < 32; ++r) { out[r] = regs[r]; }
}

// Normal form: the warp writes the vector, lane l storing row r at out[l + 32r].
template <int BW, typename T>
__device__ __forceinline__ void unpack_strided_ptr(const uint32_t* in, T* out) {
	T              regs[32];
	const uint32_t lane = threadIdx.x & 31u;
	unpack_regs_bw<BW>(in, lane, regs);
#pragma unroll
	for (int r = 0; r < 32; ++r) { out[lane + 32 * r] = regs[r]; }
}

template <typename T>
__device__ __forceinline__ void unpack_rows_dyn(const uint32_t* in, T* out, uint8_t bw) {
	switch (bw) {
#define FLS_CRYSTAL_ROWS(B)                                                                                            \
	case B: unpack_rows_ptr<B>(in, out); break;
		FLS_BW_CASES_0_32(FLS_CRYSTAL_ROWS)
#undef FLS_CRYSTAL_ROWS
	default:
		for (int r = 0; r < 32; ++r) { out[r] = T(0); }
		unsupported_width();
	}
}

template <typename T>
__device__ __forceinline__ void unpack_strided_dyn(const uint32_t* in, T* out, uint8_t bw) {
	switch (bw) {
#define FLS_CRYSTAL_STRIDED(B)                                                                                         \
	case B: unpack_strided_ptr<B>(in, out); break;
		FLS_BW_CASES_0_32(FLS_CRYSTAL_STRIDED)
#undef FLS_CRYSTAL_STRIDED
	default:
		for (int r = 0; r < 32; ++r) { out[(threadIdx.x & 31u) + 32 * r] = T(0); }
		unsupported_width();
	}
}

// Rows 8q..8q+7 of the calling lane from a quarter pointer in = vector +
// q*bw*8 words: quarter q begins at bit 8q*bw of each lane's stream, i.e. on
// word q*bw/4, so for bw % 4 == 0 the pointer is exactly that word.
template <int BW, typename T>
__device__ __forceinline__ void unpack_quarter_bw(const uint32_t* in, T* out) {
	static_assert(BW % 4 == 0 && BW <= 32, "quarter decode needs a bit width that is a multiple of 4");
	const uint32_t lane = threadIdx.x & 31u;
	if constexpr (BW == 0) {
#pragma unroll
		for (int r = 0; r < 8; ++r) { out[r] = T(0); }
	} else {
		uint32_t w[BW / 4 + 1];
#pragma unroll
		for (int k = 0; k < BW / 4; ++k) { w[k] = in[32 * k + lane]; }
		w[BW / 4] = 0u;
		constexpr uint32_t m = BW >= 32 ? 0xffffffffu : ((1u << BW) - 1u);
#pragma unroll
		for (int r = 0; r < 8; ++r) {
			const int bit = r * BW, k = bit >> 5, sh = bit & 31;
			out[r] = static_cast<T>(__funnelshift_r(w[k], w[k + 1], sh) & m);
		}
	}
}

template <typename T>
__device__ __forceinline__ void unpack_quarter_dyn(const uint32_t* in, T* out, uint8_t bw) {
	switch (bw) {
#define FLS_CRYSTAL_Q(B)                                                                                               \
	case B: unpack_quarter_bw<B>(in, out); break;
		FLS_CRYSTAL_Q(0) FLS_CRYSTAL_Q(4) FLS_CRYSTAL_Q(8) FLS_CRYSTAL_Q(12) FLS_CRYSTAL_Q(16) FLS_CRYSTAL_Q(20)
		FLS_CRYSTAL_Q(24) FLS_CRYSTAL_Q(28) FLS_CRYSTAL_Q(32)
#undef FLS_CRYSTAL_Q
	default:
		for (int r = 0; r < 8; ++r) { out[r] = T(0); }
		unsupported_width();
	}
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void load_registers(int i, T* out, T* registers) {
#pragma unroll
	for (int j = 0; j < ITEMS_PER_THREAD; j++) { out[j * BLOCK_THREADS + i] = registers[j]; }
}
} // namespace detail

// Register form (unpack_fused.cuh:3455): lane l of the warp gets rows r = 0..31
// of the 1024-value vector at `in` (32*bw words), i.e. values 32*r + l, in out[r].
template <typename T>
__device__ __forceinline__ void unpack_device(const T* in, T (&out)[32], uint8_t bw) {
	detail::unpack_rows_dyn(reinterpret_cast<const uint32_t*>(in), out, bw);
}

// Normal form (unpack.cuh:3444): the warp writes the whole vector, lane l
// storing out[l + 32*r].
template <typename T>
__device__ __forceinline__ void unpack_device_ptr(const T* in, T* out, uint8_t bw) {
	detail::unpack_strided_dyn(reinterpret_cast<const uint32_t*>(in), out, bw);
}

// Rows 8q..8q+7 of the lane from a quarter pointer (the 8-at-a-time decoder
// below); false (and zeros) for a bit width that is not a multiple of 4.
template <typename T>
__device__ __forceinline__ bool unpack_quarter(const T* in_quarter, T (&out)[8], uint8_t bw) {
	if (bw > 32 || (bw & 3u)) {
		for (int r = 0; r < 8; ++r) { out[r] = T(0); }
		return false;
	}
	detail::unpack_quarter_dyn(reinterpret_cast<const uint32_t*>(in_quarter), out, bw);
	return true;
}

// The reference's specialised decoders under their namespaces and names
// (fls_gen/unpack/hardcoded_16.cuh), so that kernels calling
// `unpack_8_at_a_time::unpack_device(ptr, items, bw)` compile unchanged.
// Each namespace offers unpack(in, out, bw), unpack_device (uint32 and int32
// input), load_registers<T, BLOCK_THREADS, ITEMS_PER_THREAD>(i, out, regs)
// and the per-width routines unpack_<bw>bw_32ow_32crw_1uf(in, out).
//   unpack_8_at_a_time (:436-786): rows 8q..8q+7 from the quarter pointer,
//     every bit width that is a multiple of 4 up to 32 (the reference: 0-24,
//     its 24 writing past the output; others trap);
//   hardcoded (:788-1206): the 32 rows of the lane into uint32 registers,
//     every width 0..32 (the reference: 4, 6, 16, 24);
//   hardcoded_16 (:16-434): the same into uint16 registers (values truncated
//     to 16 bits, as the reference stores them).
#define FLS_CRYSTAL_COMMON(OUT)                                                                                        \
	template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>                                                   \
	__device__ __forceinline__ void load_registers(int i, T* out, T* registers) {                                    \
		detail::load_registers<T, BLOCK_THREADS, ITEMS_PER_THREAD>(i, out, registers);                               \
	}                                                                                                                \
	__device__ __forceinline__ void unpack_device(const uint32_t* __restrict__ in, OUT* __restrict__ out, uint8_t bw) { \
		unpack(in, out, bw);                                                                                         \
	}

namespace unpack_8_at_a_time {
__device__ __forceinline__ void unpack(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint8_t bw) {
	detail::unpack_quarter_dyn(in, out, bw);
}
FLS_CRYSTAL_COMMON(uint32_t)
__device__ __forceinline__ void unpack_device(const int32_t* __restrict__ in, int32_t* __restrict__ out, uint8_t bw) {
	detail::unpack_quarter_dyn(reinterpret_cast<const uint32_t*>(in), out, bw);
}
#define FLS_CRYSTAL_Q_NAMED(B)                                                                                         \
	__device__ __forceinline__ void unpack_##B##bw_32ow_32crw_1uf(const uint32_t* __restrict__ a_in_p,             \
	                                                               uint32_t* __restrict__ a_out_p) {                \
		detail::unpack_quarter_bw<B>(a_in_p, a_out_p);                                                               \
	}
FLS_CRYSTAL_Q_NAMED(0) FLS_CRYSTAL_Q_NAMED(4) FLS_CRYSTAL_Q_NAMED(8) FLS_CRYSTAL_Q_NAMED(12) FLS_CRYSTAL_Q_NAMED(16)
FLS_CRYSTAL_Q_NAMED(20) FLS_CRYSTAL_Q_NAMED(24) FLS_CRYSTAL_Q_NAMED(28) FLS_CRYSTAL_Q_NAMED(32)
#undef FLS_CRYSTAL_Q_NAMED
} // namespace unpack_8_at_a_time

#define FLS_CRYSTAL_ROWS_NAMED(B)                                                                                      \
	__device__ __forceinline__ void unpack_##B##bw_32ow_32crw_1uf(const uint32_t* __restrict__ a_in_p,             \
	                                                               OutT* __restrict__ a_out_p) {                    \
		detail::unpack_rows_ptr<B>(a_in_p, a_out_p);                                                                 \
	}

namespace hardcoded {
using OutT = uint32_t;
__device__ __forceinline__ void unpack(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint8_t bw) {
	detail::unpack_rows_dyn(in, out, bw);
}
FLS_CRYSTAL_COMMON(uint32_t)
__device__ __forceinline__ void unpack_device(const int32_t* __restrict__ in, int32_t* __restrict__ out, uint8_t bw) {
	detail::unpack_rows_dyn(reinterpret_cast<const uint32_t*>(in), out, bw);
}
FLS_BW_CASES_0_32(FLS_CRYSTAL_ROWS_NAMED)
} // namespace hardcoded

namespace hardcoded_16 {
using OutT = uint16_t;
__device__ __forceinline__ void unpack(const uint32_t* __restrict__ in, uint16_t* __restrict__ out, uint8_t bw) {
	detail::unpack_rows_dyn(in, out, bw);
}
FLS_CRYSTAL_COMMON(uint16_t)
__device__ __forceinline__ void unpack_device(const int32_t* __restrict__ in, uint16_t* __restrict__ out, uint8_t bw) {
	detail::unpack_rows_dyn(reinterpret_cast<const uint32_t*>(in), out, bw);
}
FLS_BW_CASES_0_32(FLS_CRYSTAL_ROWS_NAMED)
} // namespace hardcoded_16
#undef FLS_CRYSTAL_ROWS_NAMED
#undef FLS_CRYSTAL_COMMON

// Running sum over the transposed layout (rsum.cuh:4-107): lane l starts at
// base[l] and accumulates rows in rsum order; in/out are 1024-value vectors in
// stored (transposed) order, lane-strided.
__device__ __forceinline__ void d_rsum_32(const uint32_t* in, uint32_t* out, const uint32_t* base) {
	const uint32_t lane = threadIdx.x & 31u;
	uint32_t       acc  = base[lane];
#pragma unroll
	for (uint32_t s = 0; s < 32; ++s) {
		const uint32_t p = 32u * fls::dev::rsum_row(s) + lane;
		acc += in[p];
		out[p] = acc;
	}
}

// Host: the decoders' error bits of this translation unit since the last
// call, cleared (bit 0: a bit width the called decoder cannot decode).
static inline __host__ cudaError_t fls_crystal_take_error(uint32_t* bits) {
	const uint32_t zero = 0;
	cudaError_t    e    = cudaMemcpyFromSymbol(bits, fls_crystal_error_word, sizeof(uint32_t));
	if (e == cudaSuccess) { e = cudaMemcpyToSymbol(fls_crystal_error_word, &zero, sizeof(uint32_t)); }
	return e;
}

} // namespace crystal
} // namespace fls
