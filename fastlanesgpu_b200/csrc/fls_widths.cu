// fls_widths.cu -- GPU decode of FastLanes columns of 8-, 16- and 64-bit
// lanes (FOR with one base and bit width per column), to HBM and/or fused
// with a sum.  The reference decodes only 32-bit lanes on the GPU
// (fls_gen/unpack/unpack.cuh); its host packer covers all four widths
// (fastlanes/src/pack.cpp:29521, 29552, 29607, 29710), whose layout this
// reads: 1024/T lanes, row r of lane i is value (1024/T)*r + i, word k of
// lane i at (1024/T)*k + i, 128-byte rows, 128*bw bytes per vector.
//
// 8/16-bit lanes: one warp per vector; thread t reads the 32-bit word t of
// each 128-byte row, which holds 32/T consecutive lanes, and extracts row r
// of all of them at once (SIMD within a register: every lane of a word has
// the same bit offset r*bw, so one shift and a per-lane mask serve all; the
// base is added lane-wise without carries between lanes).  64-bit lanes: a
// half-warp per vector, one lane per thread.  Both read and write 128-byte
// rows per instruction.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "fls_pipeline.cuh"

namespace fls {
namespace {

template <int B>
struct Narrow {
	static constexpr uint32_t kRep  = B == 8 ? 0x01010101u : 0x00010001u; // one per lane of a word
	static constexpr uint32_t kLow  = (1u << B) - 1u;
	static constexpr uint32_t kHigh = (1u << (B - 1)) * kRep; // lane top bits
};

// Lane-wise sum of the 32/B lanes of x.
template <int B>
__device__ __forceinline__ uint32_t lane_sum(uint32_t x) {
	if constexpr (B == 8) {
		const uint32_t t = (x & 0x00ff00ffu) + ((x >> 8) & 0x00ff00ffu);
		return (t & 0xffffu) + (t >> 16);
	} else {
		return (x & 0xffffu) + (x >> 16);
	}
}

// One vector of 8/16-bit lanes: row r of the 32/B lanes of thread word t.
// OUT / SUM: write the values / add them to part; TAIL: the column's last,
// partial vector (rem values).  NOWRAP (sum only, whole vectors): the host
// proved base + 2^bw - 1 < 2^B, so no value wraps and the packed fields are
// summed in 2B-bit halves with the base added once per thread (32 values).
// Branch-free per row, so the loads of all rows can issue before the first
// is used.
template <int B, bool OUT, bool SUM, bool TAIL, bool NOWRAP = false>
__device__ __forceinline__ void narrow_vector(const uint32_t* __restrict src, uint32_t* __restrict dst, uint32_t bw,
                                              uint32_t vm, uint32_t base_rep, uint32_t t, uint64_t rem,
                                              uint32_t& part) {
	using N              = Narrow<B>;
	constexpr uint32_t L = 32u / B;   // lanes per thread word
	constexpr uint32_t S = 1024u / B; // lanes per vector
	const uint32_t     last = bw ? bw - 1u : 0u;
	static_assert(!NOWRAP || (SUM && !OUT && !TAIL), "NOWRAP sums whole vectors only");
	uint32_t           ev = 0, od = 0; // NOWRAP: even and odd lanes' fields, 2B-bit sums
#pragma unroll
	for (uint32_t r = 0; r < static_cast<uint32_t>(B); ++r) {
		// the second word row is read unconditionally, clamped inside the vector
		const uint32_t o = r * bw, k = o / B, s = o % B;
		const uint32_t lo_word = __ldg(src + 32u * k + t);
		const uint32_t hi_word = __ldg(src + 32u * min(k + 1u, last) + t);
		const uint32_t hi      = (hi_word << (B - s)) & (((N::kLow << (B - s)) & N::kLow) * N::kRep);
		const uint32_t x       = (((lo_word >> s) & ((N::kLow >> s) * N::kRep)) |
		                    (s + bw > static_cast<uint32_t>(B) ? hi : 0u)) & vm;
		if constexpr (NOWRAP) {
			// at most 8 (B = 8) or 16 (B = 16) rows of B-bit fields per half
			if constexpr (B == 8) {
				ev += x & 0x00ff00ffu;
				od += (x >> 8) & 0x00ff00ffu;
			} else {
				ev += x & 0xffffu;
				od += x >> 16;
			}
			continue;
		}
		const uint32_t y = ((x & ~N::kHigh) + (base_rep & ~N::kHigh)) ^ ((x ^ base_rep) & N::kHigh);
		if constexpr (OUT) { __stcs(dst + 32u * r + t, y); }
		if constexpr (SUM) {
			uint32_t keep = y;
			if constexpr (TAIL) {
				keep = 0;
#pragma unroll
				for (uint32_t j = 0; j < L; ++j) {
					keep |= (S * r + L * t + j < rem) ? (y & (N::kLow << (B * j))) : 0u;
				}
			}
			part += lane_sum<B>(keep);
		}
	}
	if constexpr (NOWRAP) {
		if constexpr (B == 8) {
			part += (ev & 0xffffu) + (ev >> 16) + (od & 0xffffu) + (od >> 16);
		} else {
			part += ev + od;
		}
		part += 32u * (base_rep & N::kLow); // the thread's 32 values
	}
}

// Resident 256-thread blocks per SM asked of the compiler (it trades
// registers for warps), measured per form on B200 at 2^28 values: decode to
// HBM 4, 8-bit sums and 64-bit lanes 3, 16-bit sums 2.
template <int B, bool OUT, bool SUM>
constexpr int narrow_min_blocks() {
	return OUT && !SUM ? 4 : (B == 16 && !OUT ? 2 : 3);
}

// 8/16-bit lanes: one warp per vector (a 0-bit column reads no payload).
template <int B, bool OUT, bool SUM>
__global__ void __launch_bounds__(256, narrow_min_blocks<B, OUT, SUM>()) decode_narrow_kernel(const uint32_t* __restrict in, uint64_t n, uint64_t n_vec,
                                                            uint32_t bw, uint32_t base_rep, uint32_t* __restrict out,
                                                            unsigned long long* sum, bool nowrap) {
	using N                = Narrow<B>;
	const uint32_t     t   = threadIdx.x & 31u;
	const uint64_t     wg  = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const uint64_t     nw  = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
	const uint32_t     vm  = (bw >= static_cast<uint32_t>(B) ? N::kLow : (1u << bw) - 1u) * N::kRep;
	unsigned long long acc = 0;
	for (uint64_t v = wg; v < n_vec; v += nw) {
		const uint32_t* src  = in + v * 32u * bw;
		uint32_t*       dst  = OUT ? out + v * 32u * B : nullptr;
		const uint64_t  rem  = n - v * 1024u;
		uint32_t        part = 0;
		if (bw == 0) {
			// every value is the base
			for (uint32_t r = 0; r < static_cast<uint32_t>(B); ++r) {
				if constexpr (OUT) { __stcs(dst + 32u * r + t, base_rep); }
			}
			if constexpr (SUM) {
				const uint64_t cnt = rem < 1024u ? rem : 1024u;
				if (t == 0) { acc += cnt * (base_rep & N::kLow); }
			}
		} else if (rem >= 1024u) {
			if constexpr (SUM && !OUT) {
				if (nowrap) {
					narrow_vector<B, OUT, SUM, false, true>(src, dst, bw, vm, base_rep, t, rem, part);
				} else {
					narrow_vector<B, OUT, SUM, false>(src, dst, bw, vm, base_rep, t, rem, part);
				}
			} else {
				narrow_vector<B, OUT, SUM, false>(src, dst, bw, vm, base_rep, t, rem, part);
			}
		} else {
			narrow_vector<B, OUT, SUM, true>(src, dst, bw, vm, base_rep, t, rem, part);
		}
		acc += part;
	}
	if constexpr (SUM) {
#pragma unroll
		for (int off = 16; off > 0; off >>= 1) { acc += __shfl_xor_sync(0xffffffffu, acc, off); }
		if (t == 0 && acc) { atomicAdd(sum, acc); }
	}
}

// 64-bit lanes: a half-warp per vector, one lane per thread.
template <bool OUT, bool SUM>
__global__ void __launch_bounds__(256, 3) decode_u64_kernel(const uint64_t* __restrict in, uint64_t n, uint64_t n_vec,
                                                         uint32_t bw, uint64_t base, uint64_t* __restrict out,
                                                         unsigned long long* sum) {
	const uint32_t     i   = threadIdx.x & 15u; // lane of the vector
	const uint64_t     h0  = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 4;
	const uint64_t     nh  = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 4;
	const uint64_t     m    = bw >= 64 ? ~0ull : (1ull << bw) - 1ull;
	const uint32_t     m_lo = static_cast<uint32_t>(m), m_hi = static_cast<uint32_t>(m >> 32);
	const uint32_t     last = bw ? bw - 1u : 0u;
	unsigned long long acc = 0;
	// every half-warp runs the same number of iterations, so full-warp
	// shuffles at the end see every lane
	const uint64_t iters = (n_vec + nh - 1) / nh;
	for (uint64_t it = 0; it < iters; ++it) {
		const uint64_t v = h0 + it * nh;
		if (v >= n_vec) { continue; }
		const auto*    src = reinterpret_cast<const unsigned long long*>(in + v * 16u * bw);
		const uint64_t rem = n - v * 1024u;
		if (bw == 0) { // every value is the base; no payload to read
			for (uint32_t r = 0; r < 64; ++r) {
				if constexpr (OUT) { __stcs(reinterpret_cast<unsigned long long*>(out) + v * 1024u + 16u * r + i, base); }
				if constexpr (SUM) { acc += 16u * r + i < rem ? base : 0ull; }
			}
			continue;
		}
		// Row r's field starts at bit s of word row k.  Both word rows are
		// read unconditionally (the second clamped inside the vector) and
		// the field is cut from their four 32-bit halves by two 32-bit
		// funnel shifts; bits of the second row past a field that does not
		// straddle fall under the mask.
		auto row = [&](uint32_t r) -> uint64_t {
			const uint32_t o = r * bw, k = o >> 6, s = o & 63u;
			const uint2    a = __ldg(reinterpret_cast<const uint2*>(src + 16u * k + i));
			const uint2    b = __ldg(reinterpret_cast<const uint2*>(src + 16u * min(k + 1u, last) + i));
			const bool     up = s >= 32u;
			const uint32_t w0 = up ? a.y : a.x, w1 = up ? b.x : a.y, w2 = up ? b.y : b.x;
			const uint32_t xl = __funnelshift_r(w0, w1, s) & m_lo, xh = __funnelshift_r(w1, w2, s) & m_hi;
			return ((static_cast<uint64_t>(xh) << 32) | xl) + base;
		};
		if (rem >= 1024u) {
#pragma unroll 16
			for (uint32_t r = 0; r < 64; ++r) {
				const uint64_t y = row(r);
				if constexpr (OUT) { __stcs(reinterpret_cast<unsigned long long*>(out) + v * 1024u + 16u * r + i, y); }
				if constexpr (SUM) { acc += y; }
			}
		} else {
#pragma unroll 4
			for (uint32_t r = 0; r < 64; ++r) {
				const uint64_t y = row(r);
				if constexpr (OUT) { __stcs(reinterpret_cast<unsigned long long*>(out) + v * 1024u + 16u * r + i, y); }
				if constexpr (SUM) { acc += 16u * r + i < rem ? y : 0ull; }
			}
		}
	}
	if constexpr (SUM) {
#pragma unroll
		for (int off = 16; off > 0; off >>= 1) { acc += __shfl_xor_sync(0xffffffffu, acc, off); }
		if ((threadIdx.x & 31u) == 0 && acc) { atomicAdd(sum, acc); }
	}
}

template <class K>
void launch_mode(bool out, bool sum, K&& k) {
	if (out && sum) {
		k(std::integral_constant<int, 3> {});
	} else if (out) {
		k(std::integral_constant<int, 1> {});
	} else {
		k(std::integral_constant<int, 2> {});
	}
}

fls_status launch_decode(uint32_t bits, const void* d_in, uint64_t n, uint8_t bw, uint64_t base, void* d_out,
                         uint64_t* d_sum, fls_stream_t stream, const char* who) {
	if (!d_in || n == 0 || (!d_out && !d_sum)) {
		return set_error(FLS_ERR_INVALID_ARG, std::string(who) + ": null pointer, n == 0 or no output");
	}
	if (bw > bits) { return set_error(FLS_ERR_BAD_BW, std::string(who) + ": bit width larger than the values"); }
	if (fls_status s = check_n_values(n, who); s != FLS_OK) { return s; }
	if ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 15u) {
		return set_error(FLS_ERR_ALIGNMENT, std::string(who) + ": buffers must be 16-byte aligned");
	}
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	cudaStream_t   st    = reinterpret_cast<cudaStream_t>(stream);
	const uint64_t n_vec = (n + 1023u) / 1024u;
	if (d_sum && (s = cuda_check(cudaMemsetAsync(d_sum, 0, sizeof(uint64_t), st), "cudaMemsetAsync")) != FLS_OK) {
		return s;
	}
	auto* sum = reinterpret_cast<unsigned long long*>(d_sum);
	if (bits == 64) {
		const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>((n_vec + 15u) / 16u, static_cast<uint64_t>(di.sms) * 16u));
		launch_mode(d_out != nullptr, d_sum != nullptr, [&](auto mode) {
			constexpr int M = decltype(mode)::value;
			decode_u64_kernel<(M & 1) != 0, (M & 2) != 0><<<grid, 256, 0, st>>>(
			    static_cast<const uint64_t*>(d_in), n, n_vec, bw, base, static_cast<uint64_t*>(d_out), sum);
		});
	} else {
		const uint32_t rep  = bits == 8 ? static_cast<uint32_t>(base & 0xffu) * 0x01010101u
		                                : static_cast<uint32_t>(base & 0xffffu) * 0x00010001u;
		// no decoded value wraps: base + 2^bw - 1 < 2^bits
		const bool nowrap = (base & ((1ull << bits) - 1u)) + ((1ull << bw) - 1u) < (1ull << bits);
		const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>((n_vec + 7u) / 8u, static_cast<uint64_t>(di.sms) * 16u));
		launch_mode(d_out != nullptr, d_sum != nullptr, [&](auto mode) {
			constexpr int M = decltype(mode)::value;
			if (bits == 8) {
				decode_narrow_kernel<8, (M & 1) != 0, (M & 2) != 0><<<grid, 256, 0, st>>>(
				    static_cast<const uint32_t*>(d_in), n, n_vec, bw, rep, static_cast<uint32_t*>(d_out), sum, nowrap);
			} else {
				decode_narrow_kernel<16, (M & 1) != 0, (M & 2) != 0><<<grid, 256, 0, st>>>(
				    static_cast<const uint32_t*>(d_in), n, n_vec, bw, rep, static_cast<uint32_t*>(d_out), sum, nowrap);
			}
		});
	}
	count_launch();
	return cuda_check(cudaGetLastError(), "decode kernel launch");
}

} // namespace
} // namespace fls

using namespace fls;

extern "C" {

fls_status fls_decode_u8(const uint8_t* d_in, uint64_t n, uint8_t bw, uint8_t base, uint8_t* d_out, uint64_t* d_sum,
                         fls_stream_t stream) {
	return launch_decode(8, d_in, n, bw, base, d_out, d_sum, stream, "fls_decode_u8");
}

fls_status fls_decode_u16(const uint16_t* d_in, uint64_t n, uint8_t bw, uint16_t base, uint16_t* d_out,
                          uint64_t* d_sum, fls_stream_t stream) {
	return launch_decode(16, d_in, n, bw, base, d_out, d_sum, stream, "fls_decode_u16");
}

fls_status fls_decode_u64(const uint64_t* d_in, uint64_t n, uint8_t bw, uint64_t base, uint64_t* d_out,
                          uint64_t* d_sum, fls_stream_t stream) {
	return launch_decode(64, d_in, n, bw, base, d_out, d_sum, stream, "fls_decode_u64");
}

} // extern "C"
