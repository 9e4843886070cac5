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
 *   unpack_8_at_a_time                            fls_gen/unpack/hardcoded_16.cuh:779
 *   d_rsum_32                                     fls_gen/rsum/rsum.cuh:4
 *
 * Conventions kept from the reference: a tile is BLOCK_THREADS x
 * ITEMS_PER_THREAD items, item ITEM of thread t is row t + BLOCK_THREADS*ITEM
 * (striped); flags are int arrays; num_items guards the last tile;
 * HASH(X,Y,Z) = (X-Z) % Y; an empty PHT slot is 0.  Differences: unpack of any
 * bit width 0..32 (no trap on unsupported widths; 8-at-a-time supports every
 * width whose quarter starts on a word boundary and returns false otherwise),
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

#define FLS_CRYSTAL_PRED(NAME, MODE, OP)                                                                               \
	template <typename T, typename ST, int BLOCK_THREADS, int ITEMS_PER_THREAD>                                      \
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

// ---------------------------------------------------------------- decoders

namespace detail {
template <int BW, typename T>
__device__ __forceinline__ void unpack_regs_bw(const uint32_t* in, uint32_t lane, T (&out)[32]) {
	fls::dev::LaneWords<BW> lw;
#pragma unroll
	for (int k = 0; k < BW; ++k) { lw.w[k] = in[32 * k + lane]; }
#pragma unroll
	for (int r = 0; r < 32; ++r) { out[r] = static_cast<T>(fls::dev::extract<BW>(lw, r)); }
}
} // namespace detail

// Register form (unpack_fused.cuh): lane l of the warp gets rows r = 0..31 of
// the 1024-value vector at `in` (32*bw words), i.e. values 32*r + l, in out[r].
template <typename T>
__device__ __forceinline__ void unpack_device(const T* in, T (&out)[32], uint8_t bw) {
	const uint32_t* w    = reinterpret_cast<const uint32_t*>(in);
	const uint32_t  lane = threadIdx.x & 31u;
	switch (bw) {
#define FLS_CRYSTAL_UNPACK(B)                                                                                          \
	case B: detail::unpack_regs_bw<B>(w, lane, out); break;
		FLS_BW_CASES_0_32(FLS_CRYSTAL_UNPACK)
#undef FLS_CRYSTAL_UNPACK
	default: break;
	}
}

// Normal form (unpack.cuh): the warp writes the whole vector, lane l storing
// out[l + 32*r].
template <typename T>
__device__ __forceinline__ void unpack_device_ptr(const T* in, T* out, uint8_t bw) {
	T              regs[32];
	const uint32_t lane = threadIdx.x & 31u;
	unpack_device(in, regs, bw);
#pragma unroll
	for (int r = 0; r < 32; ++r) { out[lane + 32 * r] = regs[r]; }
}

// Rows 8q..8q+7 of the lane from a quarter pointer in = vector + q*bw*8
// (hardcoded_16.cuh:436-786).  Valid when the quarter starts on a word
// boundary of every lane stream (bw % 4 == 0); returns false otherwise.
template <typename T>
__device__ __forceinline__ bool unpack_8_at_a_time(const T* in_quarter, T (&out)[8], uint8_t bw) {
	if (bw > 32 || (bw & 3u)) { return false; }
	const uint32_t* w    = reinterpret_cast<const uint32_t*>(in_quarter);
	const uint32_t  lane = threadIdx.x & 31u;
	const uint32_t  m    = bw >= 32 ? 0xffffffffu : ((1u << bw) - 1u);
#pragma unroll
	for (uint32_t r = 0; r < 8; ++r) {
		if (bw == 0) {
			out[r] = T(0);
			continue;
		}
		const uint32_t bit = r * bw, k = bit >> 5, sh = bit & 31u;
		const uint32_t hi  = (sh + bw > 32u) ? w[32u * (k + 1u) + lane] : 0u;
		out[r]             = static_cast<T>(__funnelshift_r(w[32u * k + lane], hi, sh) & m);
	}
	return true;
}

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

} // namespace crystal
} // namespace fls
