// fls_encode.cu -- the FastLanes column encoder on the GPU.
//
// Produces exactly the words and metadata of the host encoder
// (fls_encode_column, fls_host.cpp encode_vector) for a column already in
// device memory, with a per-vector scheme that may itself come from the GPU
// (the learned selector's picks), so a column can be selected and encoded
// without leaving the device.  Three steps, all stream-ordered:
//
//  1. plan: one warp per vector stages its 1024 values in shared memory and
//     computes the chosen scheme's bit width, aux and payload words;
//  2. scan: payload words -> 64-bit word offsets (written into the metadata),
//     the column's total words, largest vector and scheme mask;
//  3. write: one warp per vector writes the payload at its offset.
//
// Layout facts restated from the reference: the lane/word order of
// fastlanes/src/pack.cpp:1954-1990, the transposed order of
// fastlanes/src/transpose.cpp:4110 with the rsum visiting order of
// fls_gen/rsum/rsum.cuh:4-107, unrsum.cpp:120-256, and rle.hpp:8-44's run
// dictionary restarting every 256 values.
#include <cuda_runtime.h>

#include <algorithm>

#include "fls_pipeline.cuh"

namespace fls {
namespace {

constexpr uint32_t kEncWarps    = 8;                 // warps per CTA
constexpr uint32_t kValWords    = 33u * 32u;         // the vector, 33-padded rows
constexpr uint32_t kEncWarpWords = kValWords + 2048u; // + sort buffer + dictionary buffer
constexpr uint32_t kScanBlock   = 1024;              // vectors per scan block

struct EncParams {
	const int32_t* values;
	uint64_t       n;
	uint64_t       n_vec;
	const uint8_t* schemes; // per vector, or null: `scheme` for all
	uint32_t       scheme;
	uint32_t       layout;
	uint32_t       round4;
	uint32_t       pad_;
	uint32_t*      out;
	fls_vec_meta*  meta;
	uint32_t*      words;   // payload words per vector
	uint64_t*      bsum;    // per scan block
	uint64_t*      info;    // [0] total words, [1] max vector words, [2] scheme mask
	uint32_t*      err;
};

__device__ __forceinline__ uint32_t bits_of(uint32_t v) { return v ? 32u - __clz(v) : 0u; }
__device__ __forceinline__ uint32_t round_words4(uint32_t w) { return (w + 3u) & ~3u; }
__device__ __forceinline__ uint32_t low_mask(uint32_t bw) { return bw >= 32 ? 0xffffffffu : ((1u << bw) - 1u); }

// Value j of the staged vector (33-padded: row and chunk reads are
// bank-conflict-free).
__device__ __forceinline__ int32_t val_at(const int32_t* v, uint32_t j) { return v[j + (j >> 5)]; }

__device__ __forceinline__ uint32_t payload_words(uint32_t scheme, uint32_t bw, uint32_t aux) {
	switch (scheme) {
	case FLS_SCHEME_FOR: return 32u * bw;
	case FLS_SCHEME_DELTA: return 32u + 32u * bw;
	case FLS_SCHEME_RLE: return 48u + round_words4((aux * bw + 31u) / 32u);
	case FLS_SCHEME_CONST: return 0u;
	default: return 32u * bits_of(aux - 1u) + round_words4((aux * bw + 31u) / 32u); // DICT
	}
}

// Loads vector v (the last one padded with the column's last value, as the
// host encoder pads) into shared memory; returns this lane's min and max.
__device__ __forceinline__ void stage_vector(const EncParams& P, uint64_t v, int32_t* sv, uint32_t lane, int32_t& mn,
                                             int32_t& mx) {
	const int32_t last = __ldg(P.values + (P.n - 1));
	mn                 = INT32_MAX;
	mx                 = INT32_MIN;
	const uint64_t v0  = v * 1024u;
	if (v0 + 1024u <= P.n && (reinterpret_cast<uintptr_t>(P.values) & 15u) == 0) { // warp-uniform
		// a whole vector from a 16-byte aligned column: eight 16-byte loads
		// per lane (values 128 k + 4 lane .. + 3), all in flight at once
		int4 q[8];
#pragma unroll
		for (uint32_t k = 0; k < 8; ++k) { q[k] = __ldg(reinterpret_cast<const int4*>(P.values + v0) + 32u * k + lane); }
		asm volatile("" ::: "memory"); // every load issued before the first store below
#pragma unroll
		for (uint32_t k = 0; k < 8; ++k) {
			const uint32_t j = 128u * k + 4u * lane; // conflict-free: (j + j / 32) mod 32 differs across lanes
			const int32_t  e[4] = {q[k].x, q[k].y, q[k].z, q[k].w};
#pragma unroll
			for (uint32_t t = 0; t < 4; ++t) {
				sv[(j + t) + ((j + t) >> 5)] = e[t];
				mn                           = min(mn, e[t]);
				mx                           = max(mx, e[t]);
			}
		}
	} else {
#pragma unroll 4
		for (uint32_t r = 0; r < 32; ++r) {
			const uint64_t idx = v0 + 32u * r + lane;
			const int32_t  x   = idx < P.n ? __ldg(P.values + idx) : last;
			sv[33u * r + lane] = x;
			mn                 = min(mn, x);
			mx                 = max(mx, x);
		}
	}
	__syncwarp();
	mn = __reduce_min_sync(0xffffffffu, mn);
	mx = __reduce_max_sync(0xffffffffu, mx);
}

// Ascending bitonic sort of 1024 int32 in shared memory by one warp.
__device__ void sort1024(int32_t* a, uint32_t lane) {
	for (uint32_t k = 2; k <= 1024; k <<= 1) {
		for (uint32_t j = k >> 1; j > 0; j >>= 1) {
			for (uint32_t q = lane; q < 512; q += 32) {
				const uint32_t i = ((q & ~(j - 1u)) << 1) | (q & (j - 1u)), p = i | j;
				const int32_t  x = a[i], y = a[p];
				const bool     up = (i & k) == 0;
				if (up ? x > y : x < y) {
					a[i] = y;
					a[p] = x;
				}
			}
			__syncwarp();
		}
	}
}

// Copies the staged vector (original order) into `a` and sorts it; returns
// the number of distinct values and leaves them, ascending, in `u`.
__device__ uint32_t distinct_sorted(const int32_t* sv, int32_t* a, int32_t* u, uint32_t lane) {
	for (uint32_t j = lane; j < 1024; j += 32) { a[j] = val_at(sv, j); }
	__syncwarp();
	sort1024(a, lane);
	// row t of the sorted values (positions 32t..32t+31, one per lane): the
	// first of each value is kept, at the count of kept values before it
	uint32_t       total = 0;
	const uint32_t below = (1u << lane) - 1u;
	for (uint32_t t = 0; t < 32; ++t) {
		const uint32_t k    = 32u * t + lane;
		const int32_t  x    = a[k];
		const bool     keep = k == 0 || x != a[k ? k - 1u : 0u];
		const uint32_t b    = __ballot_sync(0xffffffffu, keep);
		if (keep) { u[total + static_cast<uint32_t>(__popc(b & below))] = x; }
		total += static_cast<uint32_t>(__popc(b));
	}
	__syncwarp();
	return total;
}

// Run starts of rle.hpp (every 256 values, or a change of value): lane L
// counts the starts of chunk L (values 32L..32L+31).
__device__ __forceinline__ uint32_t chunk_starts(const int32_t* sv, uint32_t lane) {
	uint32_t f = 0;
#pragma unroll 4
	for (uint32_t s = 0; s < 32; ++s) {
		const uint32_t j = 32u * lane + s;
		f |= ((j & 255u) == 0 || val_at(sv, j) != val_at(sv, j ? j - 1u : 0u) ? 1u : 0u) << s;
	}
	return f;
}

// Element of the lane's row r in the column's layout.
__device__ __forceinline__ uint32_t layout_index(uint32_t layout, uint32_t lane, uint32_t r) {
	return layout == FLS_LAYOUT_NORMAL ? 32u * r + lane : 32u * dev::chunk_of_lane(lane) + dev::step_of_row(r);
}

// FastLanes packing of the lane's 32 rows (x[r]) into words out[32k + lane].
__device__ __forceinline__ void pack_lane(const uint32_t (&x)[32], uint32_t bw, uint32_t* out, uint32_t lane) {
	if (bw == 0) { return; }
	const uint32_t m    = low_mask(bw);
	uint64_t       acc  = 0;
	uint32_t       fill = 0, k = 0;
#pragma unroll
	for (uint32_t r = 0; r < 32; ++r) {
		acc |= static_cast<uint64_t>(x[r] & m) << fill;
		fill += bw;
		if (fill >= 32) {
			out[32u * k++ + lane] = static_cast<uint32_t>(acc);
			acc >>= 32;
			fill -= 32;
		}
	}
}

// Sequential LSB-first packing of u[0..n) - base at bw bits, zero-padded to a
// multiple of 4 words (the host's pack_sequential).
__device__ void pack_sequential(const int32_t* u, uint32_t n, uint32_t bw, uint32_t base, uint32_t* out,
                                uint32_t lane) {
	const uint32_t words = round_words4((n * bw + 31u) / 32u);
	const uint32_t m     = low_mask(bw);
	for (uint32_t w = lane; w < words; w += 32) {
		uint32_t word = 0;
		if (bw) {
			const uint32_t bit0 = 32u * w;
			for (uint32_t k = bit0 / bw; k < n && k * bw < bit0 + 32u; ++k) {
				const uint32_t val = (static_cast<uint32_t>(u[k]) - base) & m;
				const uint32_t lo  = k * bw;
				word |= lo >= bit0 ? val << (lo - bit0) : val >> (bit0 - lo);
			}
		}
		out[w] = word;
	}
}

struct Plan {
	uint32_t scheme, bw, aux;
	int32_t  base;
};

// Scheme parameters of the staged vector (CONST on a non-constant vector
// becomes FOR, as on the host).
__device__ Plan plan_vector(const EncParams& P, uint64_t v, int32_t* sv, int32_t* a, int32_t* u, uint32_t lane,
                            int32_t mn, int32_t mx) {
	uint32_t s = P.schemes ? P.schemes[v] : P.scheme;
	if (s >= FLS_N_SCHEMES) {
		if (lane == 0) { atomicOr(P.err, kErrBadMeta); }
		s = FLS_SCHEME_FOR;
	}
	if (s == FLS_SCHEME_CONST && mn != mx) { s = FLS_SCHEME_FOR; }
	const uint32_t range = static_cast<uint32_t>(mx) - static_cast<uint32_t>(mn);
	Plan           p {s, 0u, 0u, 0};
	switch (s) {
	case FLS_SCHEME_CONST: p.base = mn; break;
	case FLS_SCHEME_FOR:
		p.bw = bits_of(range);
		if (P.round4 && p.bw) { p.bw = (p.bw + 3u) & ~3u; }
		p.base = mn;
		break;
	case FLS_SCHEME_DELTA: {
		const uint32_t c = dev::chunk_of_lane(lane);
		uint32_t       mxd = 0;
		int32_t        prev = val_at(sv, 32u * c);
		for (uint32_t t = 1; t < 32; ++t) {
			const int32_t cur = val_at(sv, 32u * c + t);
			mxd               = max(mxd, static_cast<uint32_t>(cur) - static_cast<uint32_t>(prev));
			prev              = cur;
		}
		p.bw = bits_of(__reduce_max_sync(0xffffffffu, mxd));
		break;
	}
	case FLS_SCHEME_RLE:
		p.aux  = __reduce_add_sync(0xffffffffu, __popc(chunk_starts(sv, lane)));
		p.bw   = bits_of(range);
		p.base = mn;
		break;
	default: // DICT
		p.aux  = distinct_sorted(sv, a, u, lane);
		p.bw   = bits_of(range);
		p.base = mn;
		break;
	}
	return p;
}

__global__ void __launch_bounds__(kEncWarps * 32) enc_plan_kernel(const __grid_constant__ EncParams P) {
	extern __shared__ __align__(16) int32_t esmem[];
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	int32_t*       sv   = esmem + warp * kEncWarpWords;
	int32_t *      a = sv + kValWords, *u = a + 1024;
	for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * kEncWarps + warp; v < P.n_vec;
	     v += static_cast<uint64_t>(gridDim.x) * kEncWarps) {
		int32_t mn, mx;
		stage_vector(P, v, sv, lane, mn, mx);
		const Plan     p = plan_vector(P, v, sv, a, u, lane, mn, mx);
		const uint32_t w = payload_words(p.scheme, p.bw, p.aux);
		if (lane == 0) {
			fls_vec_meta m;
			m.offset  = 0;
			m.base    = p.base;
			m.scheme  = static_cast<uint8_t>(p.scheme);
			m.bw      = static_cast<uint8_t>(p.bw);
			m.aux     = static_cast<uint16_t>(p.aux);
			P.meta[v] = m;
			P.words[v] = w;
			atomicMax(reinterpret_cast<unsigned long long*>(P.info + 1), static_cast<unsigned long long>(w));
			atomicOr(reinterpret_cast<unsigned long long*>(P.info + 2), 1ull << p.scheme);
		}
		__syncwarp();
	}
}

// ------------------------------------------------ learned selection

struct SelParams {
	const int32_t*      values;
	uint64_t            n, n_vec;
	const uint8_t*      mlp_best; // the network's pick per vector
	const float*        conf;     // and its probability
	float               threshold;
	uint32_t            pad_;
	double              kappa;
	uint8_t*            schemes;  // the chosen scheme per vector
	unsigned long long* n_fallback;
};

// The exhaustive choice for vectors the network is unsure of (confidence
// below threshold), else the network's pick.  The exact encoded sizes of
// every scheme (payload + 16 B metadata) are the host exhaustive encoder's
// (fls_host.cpp scheme_sizes), the choice the label rule of the learned
// selector: argmin of size x (1 + kappa (decode cost - 1)) with the decode
// costs FOR 1, DELTA 1.5, RLE 2, CONST 1, DICT 4.5, ties to the cheaper
// decode (FOR, CONST, DELTA, RLE, DICT), in IEEE double with each product and
// sum rounded separately (no fused multiply-add), as numpy computes it.
__global__ void __launch_bounds__(kEncWarps * 32) enc_select_kernel(const __grid_constant__ SelParams S) {
	extern __shared__ __align__(16) int32_t esmem[];
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	int32_t*       sv   = esmem + warp * kEncWarpWords;
	int32_t *      a = sv + kValWords, *u = a + 1024;
	EncParams      P {};
	P.values = S.values;
	P.n      = S.n;
	for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * kEncWarps + warp; v < S.n_vec;
	     v += static_cast<uint64_t>(gridDim.x) * kEncWarps) {
		if (!(S.conf[v] < S.threshold)) {
			if (lane == 0) { S.schemes[v] = S.mlp_best[v]; }
			continue;
		}
		int32_t mn, mx;
		stage_vector(P, v, sv, lane, mn, mx);
		const uint32_t rbw = bits_of(static_cast<uint32_t>(mx) - static_cast<uint32_t>(mn));
		uint32_t       mxd = 0;
		{
			const uint32_t c    = dev::chunk_of_lane(lane);
			int32_t        prev = val_at(sv, 32u * c);
			for (uint32_t t = 1; t < 32; ++t) {
				const int32_t cur = val_at(sv, 32u * c + t);
				mxd               = max(mxd, static_cast<uint32_t>(cur) - static_cast<uint32_t>(prev));
				prev              = cur;
			}
		}
		const uint32_t dbw    = bits_of(__reduce_max_sync(0xffffffffu, mxd));
		const uint32_t n_runs = __reduce_add_sync(0xffffffffu, __popc(chunk_starts(sv, lane)));
		const uint32_t n_dist = distinct_sorted(sv, a, u, lane);
		if (lane == 0) {
			uint32_t size[FLS_N_SCHEMES];
			size[FLS_SCHEME_FOR]   = 16u + 4u * payload_words(FLS_SCHEME_FOR, rbw, 0u);
			size[FLS_SCHEME_DELTA] = 16u + 4u * payload_words(FLS_SCHEME_DELTA, dbw, 0u);
			size[FLS_SCHEME_RLE]   = 16u + 4u * payload_words(FLS_SCHEME_RLE, rbw, n_runs);
			size[FLS_SCHEME_CONST] = mn == mx ? 16u : 0xffffffffu;
			size[FLS_SCHEME_DICT]  = 16u + 4u * payload_words(FLS_SCHEME_DICT, rbw, n_dist);
			const uint32_t order[FLS_N_SCHEMES] = {FLS_SCHEME_FOR, FLS_SCHEME_CONST, FLS_SCHEME_DELTA, FLS_SCHEME_RLE,
			                                       FLS_SCHEME_DICT};
			const double cost[FLS_N_SCHEMES] = {1.0, 1.5, 2.0, 1.0, 4.5}; // by scheme id
			uint32_t     best = order[0];
			double       best_score = 0.0;
			for (uint32_t i = 0; i < FLS_N_SCHEMES; ++i) {
				const uint32_t sc = order[i];
				if (size[sc] == 0xffffffffu) { continue; }
				const double f     = __dadd_rn(1.0, __dmul_rn(S.kappa, cost[sc] - 1.0));
				const double score = __dmul_rn(static_cast<double>(size[sc]), f);
				if (i == 0 || score < best_score) {
					best       = sc;
					best_score = score;
				}
			}
			S.schemes[v] = static_cast<uint8_t>(best);
			atomicAdd(S.n_fallback, 1ull);
		}
		__syncwarp();
	}
}

// Exclusive scan of the payload words of one block of kScanBlock vectors
// (blockDim = 256, 4 vectors per thread).  Returns the block total; with
// `write` the offsets (plus `carry`) go into the metadata.
__device__ uint64_t block_scan(const EncParams& P, uint64_t b, bool write, uint64_t carry) {
	__shared__ uint64_t wsum[8];
	const uint32_t      t = threadIdx.x, lane = t & 31u, warp = t >> 5;
	uint64_t            x[4], local = 0;
#pragma unroll
	for (uint32_t i = 0; i < 4; ++i) {
		const uint64_t v = b * kScanBlock + 4u * t + i;
		x[i]             = v < P.n_vec ? P.words[v] : 0u;
		local += x[i];
	}
	uint64_t incl = local;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= static_cast<uint32_t>(o)) { incl += y; }
	}
	if (lane == 31) { wsum[warp] = incl; }
	__syncthreads();
	uint64_t before = 0, total = 0;
	for (uint32_t w = 0; w < 8; ++w) {
		before += w < warp ? wsum[w] : 0u;
		total += wsum[w];
	}
	if (write) {
		uint64_t off = carry + before + incl - local;
#pragma unroll
		for (uint32_t i = 0; i < 4; ++i) {
			const uint64_t v = b * kScanBlock + 4u * t + i;
			if (v < P.n_vec) { P.meta[v].offset = off; }
			off += x[i];
		}
	}
	__syncthreads();
	return total;
}

__global__ void __launch_bounds__(256) enc_scan_sums_kernel(const __grid_constant__ EncParams P) {
	const uint64_t total = block_scan(P, blockIdx.x, false, 0);
	if (threadIdx.x == 0) { P.bsum[blockIdx.x] = total; }
}

// One thread: exclusive prefix of the block sums (there are n_vec / 1024 of
// them) and the column's total.
__global__ void enc_scan_blocks_kernel(const __grid_constant__ EncParams P, uint64_t n_blocks) {
	if (threadIdx.x != 0 || blockIdx.x != 0) { return; }
	uint64_t run = 0;
	for (uint64_t b = 0; b < n_blocks; ++b) {
		const uint64_t s = P.bsum[b];
		P.bsum[b]        = run;
		run += s;
	}
	P.info[0] = run;
}

// A column of one scan block: offsets and total in one launch.
__global__ void __launch_bounds__(256) enc_scan_single_kernel(const __grid_constant__ EncParams P) {
	const uint64_t total = block_scan(P, 0, true, 0);
	if (threadIdx.x == 0) { P.info[0] = total; }
}

__global__ void __launch_bounds__(256) enc_scan_offsets_kernel(const __grid_constant__ EncParams P) {
	block_scan(P, blockIdx.x, true, P.bsum[blockIdx.x]);
}

__global__ void __launch_bounds__(kEncWarps * 32) enc_write_kernel(const __grid_constant__ EncParams P) {
	extern __shared__ __align__(16) int32_t esmem[];
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	int32_t*       sv   = esmem + warp * kEncWarpWords;
	int32_t *      a = sv + kValWords, *u = a + 1024;
	for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * kEncWarps + warp; v < P.n_vec;
	     v += static_cast<uint64_t>(gridDim.x) * kEncWarps) {
		int32_t mn, mx;
		stage_vector(P, v, sv, lane, mn, mx);
		const fls_vec_meta m   = P.meta[v];
		uint32_t*          out = P.out + m.offset;
		const uint32_t     base = static_cast<uint32_t>(m.base);
		uint32_t           x[32];
		switch (m.scheme) {
		case FLS_SCHEME_FOR:
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) {
				x[r] = static_cast<uint32_t>(val_at(sv, layout_index(P.layout, lane, r))) - base;
			}
			pack_lane(x, m.bw, out, lane);
			break;
		case FLS_SCHEME_DELTA: {
			const uint32_t c = dev::chunk_of_lane(lane);
			out[lane]        = static_cast<uint32_t>(val_at(sv, 32u * c));
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) {
				const uint32_t t = dev::step_of_row(r);
				x[r] = t == 0 ? 0u
				              : static_cast<uint32_t>(val_at(sv, 32u * c + t)) -
				                    static_cast<uint32_t>(val_at(sv, 32u * c + t - 1u));
			}
			pack_lane(x, m.bw, out + 32, lane);
			break;
		}
		case FLS_SCHEME_RLE: {
			// Run index of every value: starts before its chunk + starts in it.
			const uint32_t f   = chunk_starts(sv, lane);
			const uint32_t cnt = __popc(f);
			uint32_t       pre = cnt;
#pragma unroll
			for (int o = 1; o < 32; o <<= 1) {
				const uint32_t y = __shfl_up_sync(0xffffffffu, pre, o);
				if (lane >= static_cast<uint32_t>(o)) { pre += y; }
			}
			pre -= cnt;
			// run dictionary: the value at each start, in order
			uint32_t ff = f, k = pre;
			while (ff) {
				const uint32_t t = __ffs(ff) - 1u;
				ff &= ff - 1u;
				u[k++] = val_at(sv, 32u * lane + t);
			}
			// transposed lane L holds chunk c(L): base = run index of its first
			// value, then 1-bit deltas (a start) in rsum row order
			const uint32_t c  = dev::chunk_of_lane(lane);
			const uint32_t fc = __shfl_sync(0xffffffffu, f, c);
			const uint32_t pc = __shfl_sync(0xffffffffu, pre, c);
			reinterpret_cast<uint16_t*>(out)[lane] = static_cast<uint16_t>(pc + (fc & 1u) - 1u);
			uint32_t bits = 0;
#pragma unroll
			for (uint32_t r = 0; r < 32; ++r) {
				const uint32_t t = dev::step_of_row(r);
				bits |= (t != 0 ? (fc >> t) & 1u : 0u) << r;
			}
			out[16 + lane] = bits;
			__syncwarp();
			pack_sequential(u, m.aux, m.bw, base, out + 48, lane);
			break;
		}
		case FLS_SCHEME_DICT: {
			const uint32_t n   = distinct_sorted(sv, a, u, lane);
			const uint32_t cbw = bits_of(n - 1u);
#pragma unroll 4
			for (uint32_t r = 0; r < 32; ++r) {
				const int32_t val = val_at(sv, layout_index(P.layout, lane, r));
				uint32_t      lo = 0, hi = n; // lower_bound
				while (lo < hi) {
					const uint32_t mid = (lo + hi) >> 1;
					if (u[mid] < val) {
						lo = mid + 1u;
					} else {
						hi = mid;
					}
				}
				x[r] = lo;
			}
			pack_lane(x, cbw, out, lane);
			pack_sequential(u, n, m.bw, base, out + 32u * cbw, lane);
			break;
		}
		default: break; // CONST: no payload
		}
		__syncwarp();
	}
}

} // namespace
} // namespace fls

using namespace fls;

extern "C" {

uint64_t fls_encode_gpu_workspace_bytes(uint64_t n) {
	const uint64_t n_vec = (n + 1023u) / 1024u, n_blocks = (n_vec + kScanBlock - 1) / kScanBlock;
	return ((4u * n_vec + 255u) & ~uint64_t {255u}) + 8u * n_blocks + 256u;
}

fls_status fls_encode_column_gpu(const int32_t* d_values, uint64_t n, const uint8_t* d_schemes, uint32_t scheme,
                                 uint32_t layout, int round4, uint32_t* d_out, uint64_t out_capacity_words,
                                 fls_vec_meta* d_meta, uint64_t* d_info, void* d_workspace, uint64_t workspace_bytes,
                                 fls_stream_t stream) {
	if (!d_values || !d_out || !d_meta || !d_info || !d_workspace || n == 0) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_encode_column_gpu: null pointer or n == 0");
	}
	if (fls_status s = check_n_values(n, "fls_encode_column_gpu"); s != FLS_OK) { return s; }
	if (!d_schemes && scheme >= FLS_N_SCHEMES) { return set_error(FLS_ERR_INVALID_ARG, "fls_encode_column_gpu: bad scheme"); }
	if (layout > FLS_LAYOUT_TRANSPOSED) { return set_error(FLS_ERR_INVALID_ARG, "fls_encode_column_gpu: bad layout"); }
	if ((reinterpret_cast<uintptr_t>(d_out) | reinterpret_cast<uintptr_t>(d_meta)) & 15u) {
		return set_error(FLS_ERR_ALIGNMENT, "fls_encode_column_gpu: output and metadata must be 16-byte aligned");
	}
	const uint64_t n_vec = (n + 1023u) / 1024u, n_blocks = (n_vec + kScanBlock - 1) / kScanBlock;
	if (out_capacity_words < n_vec * kMaxVecWords) {
		return set_error(FLS_ERR_CAPACITY, "fls_encode_column_gpu: output smaller than fls_encode_bound_words(n)");
	}
	if (workspace_bytes < fls_encode_gpu_workspace_bytes(n)) {
		return set_error(FLS_ERR_CAPACITY, "fls_encode_column_gpu: workspace smaller than fls_encode_gpu_workspace_bytes(n)");
	}
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	EncParams    P {};
	P.values  = d_values;
	P.n       = n;
	P.n_vec   = n_vec;
	P.schemes = d_schemes;
	P.scheme  = scheme;
	P.layout  = layout;
	P.round4  = round4 ? 1u : 0u;
	P.out     = d_out;
	P.meta    = d_meta;
	P.words   = static_cast<uint32_t*>(d_workspace);
	P.bsum    = reinterpret_cast<uint64_t*>(static_cast<char*>(d_workspace) + ((4u * n_vec + 255u) & ~uint64_t {255u}));
	P.info    = d_info;
	P.err     = device_error_word(st);
	const size_t smem = 4u * kEncWarps * kEncWarpWords;
	{
		static std::mutex mu;
		static uint64_t   configured = 0;
		int               dev        = 0;
		cudaGetDevice(&dev);
		std::lock_guard<std::mutex> lk(mu);
		if (dev >= 64 || !(configured & (1ull << dev))) {
			if ((s = cuda_check(cudaFuncSetAttribute(enc_plan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			                                         static_cast<int>(smem)),
			                    "cudaFuncSetAttribute")) != FLS_OK ||
			    (s = cuda_check(cudaFuncSetAttribute(enc_write_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			                                         static_cast<int>(smem)),
			                    "cudaFuncSetAttribute")) != FLS_OK) {
				return s;
			}
			if (dev < 64) { configured |= 1ull << dev; }
		}
	}
	if ((s = cuda_check(cudaMemsetAsync(d_info, 0, 3 * sizeof(uint64_t), st), "cudaMemsetAsync")) != FLS_OK) { return s; }
	const uint32_t grid = static_cast<uint32_t>(
	    std::min<uint64_t>((n_vec + kEncWarps - 1) / kEncWarps, static_cast<uint64_t>(di.sms) * 8u));
	enc_plan_kernel<<<grid, kEncWarps * 32, smem, st>>>(P);
	if (n_blocks == 1) {
		enc_scan_single_kernel<<<1, 256, 0, st>>>(P);
	} else {
		enc_scan_sums_kernel<<<static_cast<uint32_t>(n_blocks), 256, 0, st>>>(P);
		enc_scan_blocks_kernel<<<1, 32, 0, st>>>(P, n_blocks);
		enc_scan_offsets_kernel<<<static_cast<uint32_t>(n_blocks), 256, 0, st>>>(P);
	}
	enc_write_kernel<<<grid, kEncWarps * 32, smem, st>>>(P);
	count_launch(n_blocks == 1 ? 3 : 5);
	return cuda_check(cudaGetLastError(), "encode kernels launch");
}

uint64_t fls_encode_learned_workspace_bytes(uint64_t n) {
	const uint64_t n_vec = (n + 1023u) / 1024u;
	auto           a256  = [](uint64_t b) { return (b + 255u) & ~uint64_t {255u}; };
	return a256(64u * n_vec) + a256(4u * n_vec) + 2u * a256(n_vec) + fls_encode_gpu_workspace_bytes(n);
}

fls_status fls_encode_learned_gpu(const int32_t* d_values, uint64_t n, const float* d_params, float threshold,
                                  double kappa, uint32_t layout, uint32_t* d_out, uint64_t out_capacity_words,
                                  fls_vec_meta* d_meta, uint64_t* d_info, uint8_t* d_schemes, void* d_workspace,
                                  uint64_t workspace_bytes, fls_stream_t stream) {
	if (!d_values || !d_params || !d_info || !d_workspace || n == 0) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_encode_learned_gpu: null pointer or n == 0");
	}
	if (fls_status s = check_n_values(n, "fls_encode_learned_gpu"); s != FLS_OK) { return s; }
	if (!(kappa >= 0.0)) { return set_error(FLS_ERR_INVALID_ARG, "fls_encode_learned_gpu: kappa must be >= 0"); }
	if (workspace_bytes < fls_encode_learned_workspace_bytes(n) || (reinterpret_cast<uintptr_t>(d_workspace) & 255u)) {
		return set_error(FLS_ERR_CAPACITY,
		                 "fls_encode_learned_gpu: workspace smaller than fls_encode_learned_workspace_bytes(n) "
		                 "or not 256-byte aligned");
	}
	const uint64_t n_vec = (n + 1023u) / 1024u;
	auto           a256  = [](uint64_t b) { return (b + 255u) & ~uint64_t {255u}; };
	char*          w     = static_cast<char*>(d_workspace);
	float*         stats = reinterpret_cast<float*>(w);
	float*         conf  = reinterpret_cast<float*>(w + a256(64u * n_vec));
	uint8_t*       best  = reinterpret_cast<uint8_t*>(w + a256(64u * n_vec) + a256(4u * n_vec));
	uint8_t*       own   = best + a256(n_vec);
	void*          enc   = own + a256(n_vec);
	uint8_t*       pick  = d_schemes ? d_schemes : own;
	cudaStream_t   st    = reinterpret_cast<cudaStream_t>(stream);
	DeviceInfo     di;
	fls_status     s = device_info(di);
	if (s != FLS_OK) { return s; }
	if ((s = fls_vector_stats_gpu(d_values, n, stats, stream)) != FLS_OK) { return s; }
	if ((s = fls_mlp_infer(d_params, stats, n_vec, nullptr, best, conf, stream)) != FLS_OK) { return s; }
	const size_t smem = 4u * kEncWarps * kEncWarpWords;
	{
		static std::mutex mu;
		static uint64_t   configured = 0;
		int               dev        = 0;
		cudaGetDevice(&dev);
		std::lock_guard<std::mutex> lk(mu);
		if (dev >= 64 || !(configured & (1ull << dev))) {
			if ((s = cuda_check(cudaFuncSetAttribute(enc_select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			                                         static_cast<int>(smem)),
			                    "cudaFuncSetAttribute")) != FLS_OK) {
				return s;
			}
			if (dev < 64) { configured |= 1ull << dev; }
		}
	}
	if ((s = cuda_check(cudaMemsetAsync(d_info + 3, 0, sizeof(uint64_t), st), "cudaMemsetAsync")) != FLS_OK) {
		return s;
	}
	SelParams S {};
	S.values     = d_values;
	S.n          = n;
	S.n_vec      = n_vec;
	S.mlp_best   = best;
	S.conf       = conf;
	S.threshold  = threshold;
	S.kappa      = kappa;
	S.schemes    = pick;
	S.n_fallback = reinterpret_cast<unsigned long long*>(d_info + 3);
	const uint32_t grid = static_cast<uint32_t>(
	    std::min<uint64_t>((n_vec + kEncWarps - 1) / kEncWarps, static_cast<uint64_t>(di.sms) * 8u));
	enc_select_kernel<<<grid, kEncWarps * 32, smem, st>>>(S);
	count_launch(1);
	if ((s = cuda_check(cudaGetLastError(), "enc_select_kernel launch")) != FLS_OK) { return s; }
	return fls_encode_column_gpu(d_values, n, pick, 0u, layout, 0, d_out, out_capacity_words, d_meta, d_info, enc,
	                             fls_encode_gpu_workspace_bytes(n), stream);
}

} // extern "C"
