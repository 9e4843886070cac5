// fls_mlp.cu -- learned encoding selection on the GPU: per-vector statistics
// and a 16-64-64-5 FP32 MLP (forward, backward, Adam, inference) that picks a
// scheme per 1024-value vector.  The exhaustive encoder (fls_host.cpp) labels
// the training vectors and stays the fallback for low-confidence picks; the
// bit width is always recomputed exactly by the encoder, so any pick is
// lossless.  (No reference counterpart: the reference chooses encodings by hand
// per column, ssb_utils.h:37-83.)
//
// Parameter layout (FLS_MLP_N_PARAMS floats): W1[64][16], b1[64], W2[64][64],
// b2[64], W3[5][64], b3[5]; ReLU after layers 1 and 2, softmax cross-entropy.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "fls_pipeline.cuh"

namespace fls {
namespace {

constexpr int kIn = FLS_MLP_IN, kH = FLS_MLP_HIDDEN, kOut = FLS_MLP_OUT;
constexpr int kW1 = 0, kB1 = kW1 + kH * kIn, kW2 = kB1 + kH, kB2 = kW2 + kH * kH, kW3 = kB2 + kH,
              kB3 = kW3 + kOut * kH, kNP = kB3 + kOut;
static_assert(kNP == FLS_MLP_N_PARAMS, "parameter layout");

__device__ __forceinline__ uint32_t bits32(uint32_t v) { return 32u - static_cast<uint32_t>(__clz(v)); }

// ------------------------------------------------------ vector statistics

// Value j of a vector staged with one pad word per 32 values: lane L's
// chunk (values 32L..32L+31) is then read without bank conflicts.
__device__ __forceinline__ uint32_t pad33(uint32_t j) { return j + (j >> 5); }

// One warp per vector; exactly the features of vector_stats() (fls_host.cpp).
__global__ void __launch_bounds__(256) stats_kernel(const int32_t* __restrict__ values, uint64_t n, uint64_t n_vec,
                                                    float* __restrict__ out) {
	__shared__ int32_t  vbuf[8][1056];
	__shared__ uint32_t bmap[8][32];
	const uint32_t lane = threadIdx.x & 31u, wi = threadIdx.x >> 5;
	const uint64_t warps = static_cast<uint64_t>(gridDim.x) * 8u;
	int32_t*       v     = vbuf[wi];
	uint32_t*      bm    = bmap[wi];
	for (uint64_t vec = static_cast<uint64_t>(blockIdx.x) * 8u + wi; vec < n_vec; vec += warps) {
		const uint64_t start = vec * 1024u;
		const uint32_t cnt   = static_cast<uint32_t>(n - start < 1024u ? n - start : 1024u);
		int32_t        mn = INT32_MAX, mx = INT32_MIN;
		if (cnt == 1024u && (reinterpret_cast<uintptr_t>(values) & 15u) == 0) { // warp-uniform
			// eight 16-byte loads per lane (values 128 k + 4 lane .. + 3), all
			// in flight, then stored 33-padded (conflict-free: (j + j / 32)
			// mod 32 differs across lanes)
			int4 q[8];
#pragma unroll
			for (uint32_t k = 0; k < 8; ++k) { q[k] = __ldg(reinterpret_cast<const int4*>(values + start) + 32u * k + lane); }
#pragma unroll
			for (uint32_t k = 0; k < 8; ++k) {
				const uint32_t j    = 128u * k + 4u * lane;
				const int32_t  e[4] = {q[k].x, q[k].y, q[k].z, q[k].w};
#pragma unroll
				for (uint32_t t = 0; t < 4; ++t) {
					v[pad33(j + t)] = e[t];
					mn              = min(mn, e[t]);
					mx              = max(mx, e[t]);
				}
			}
		} else {
			for (uint32_t j = lane; j < 1024u; j += 32u) {
				// a partial last vector is padded with its last value (as the encoder does)
				const int32_t x = values[start + min(j, cnt - 1u)];
				v[pad33(j)]     = x;
				mn              = min(mn, x);
				mx              = max(mx, x);
			}
		}
		bm[lane] = 0u;
		__syncwarp();
		mn = __reduce_min_sync(0xffffffffu, mn);
		mx = __reduce_max_sync(0xffffffffu, mx);
		const uint32_t rbw = bits32(static_cast<uint32_t>(mx) - static_cast<uint32_t>(mn));
		const int32_t* c   = v + 33u * lane; // this lane's chunk: values 32 lane .. 32 lane + 31
		// u <= tm_h (tm_q): the value lies in the lower half (sixteenth) of the
		// range's bit width; every value counts when the width is 0 (<= 4)
		const uint32_t tm_h = rbw == 0 ? 0xffffffffu : (1u << (rbw / 2)) - 1u;
		const uint32_t tm_q = rbw <= 4 ? 0xffffffffu : (1u << (rbw - 4)) - 1u;
		const int32_t  c0   = c[0];
		// the value before the chunk; the vector's first value is compared
		// with itself (an equal pair, corrected below)
		const int32_t  pb   = lane ? v[pad33(32u * lane - 1u)] : c0;
		int32_t        p    = pb;
		uint32_t       max_d = 0, up = 0, eqs = 0, lh = 0, lq = 0;
		unsigned long long sabs = 0;
		bool               same = true;
#pragma unroll 8
		for (uint32_t s = 0; s < 32; ++s) {
			const int32_t  x = c[s];
			const uint32_t u = static_cast<uint32_t>(x) - static_cast<uint32_t>(mn);
			lh += u <= tm_h ? 1u : 0u;
			lq += u <= tm_q ? 1u : 0u;
			const uint32_t h = (static_cast<uint32_t>(x) * 0x9e3779b1u) >> 22;
			atomicOr(&bm[h >> 5], 1u << (h & 31u));
			same = same && x == c0;
			sabs += static_cast<uint32_t>(max(x, p)) - static_cast<uint32_t>(min(x, p));
			up += x > p ? 1u : 0u;
			eqs += x == p ? 1u : 0u;
			if (s != 0) { max_d = max(max_d, static_cast<uint32_t>(x) - static_cast<uint32_t>(p)); }
			p = x;
		}
		// deltas of the lane: 32 (31 for lane 0, whose first value has no
		// predecessor); runs (rle.hpp): a change of value, or every 256 values
		// (the chunks of lanes 0, 8, 16, 24 open one whether or not the value
		// changes, lane 0's first value included)
		uint32_t       eq   = eqs - (lane == 0 ? 1u : 0u);
		uint32_t       down = 32u - up - eqs;
		uint32_t       runs = 32u - eqs + (((lane & 7u) == 0 && c0 == pb) ? 1u : 0u);
		__syncwarp();
		const uint32_t occ = __reduce_add_sync(0xffffffffu, static_cast<uint32_t>(__popc(bm[lane])));
		max_d              = __reduce_max_sync(0xffffffffu, max_d);
		runs               = __reduce_add_sync(0xffffffffu, runs);
		up                 = __reduce_add_sync(0xffffffffu, up);
		down               = __reduce_add_sync(0xffffffffu, down);
		eq                 = __reduce_add_sync(0xffffffffu, eq);
		lh                 = __reduce_add_sync(0xffffffffu, lh);
		lq                 = __reduce_add_sync(0xffffffffu, lq);
		const uint32_t cc  = static_cast<uint32_t>(__popc(__ballot_sync(0xffffffffu, same)));
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) { sabs += __shfl_xor_sync(0xffffffffu, sabs, o); }
		const unsigned long long mean_d = sabs >> 10;
		const uint32_t amin = mn < 0 ? static_cast<uint32_t>(-static_cast<long long>(mn)) : static_cast<uint32_t>(mn);
		float f = 0.0f;
		switch (lane) {
		case 0: f = static_cast<float>(rbw) / 32.0f; break;
		case 1: f = static_cast<float>(bits32(max_d)) / 32.0f; break;
		case 2: f = static_cast<float>(runs) / 1024.0f; break;
		case 3: f = static_cast<float>(up) / 1024.0f; break;
		case 4: f = static_cast<float>(down) / 1024.0f; break;
		case 5: f = static_cast<float>(eq) / 1024.0f; break;
		case 6: f = static_cast<float>(occ) / 1024.0f; break;
		case 7: f = static_cast<float>(bits32(occ)) / 16.0f; break;
		case 8: f = static_cast<float>(bits32(static_cast<uint32_t>(min(mean_d, 0xffffffffull)))) / 32.0f; break;
		case 9: f = static_cast<float>(lh) / 1024.0f; break;
		case 10: f = static_cast<float>(lq) / 1024.0f; break;
		case 11: f = static_cast<float>(bits32(amin)) / 32.0f; break;
		case 12: f = mn == mx ? 1.0f : 0.0f; break;
		case 13: f = static_cast<float>(bits32(runs)) / 16.0f; break;
		case 14: f = static_cast<float>(cc) / 32.0f; break;
		case 15: f = 1.0f; break;
		default: break;
		}
		if (lane < 16) { out[vec * 16u + lane] = f; }
		__syncwarp();
	}
}

// ------------------------------------------------------------------ MLP

__device__ __forceinline__ uint32_t hash32(uint64_t x) {
	x ^= x >> 33;
	x *= 0xff51afd7ed558ccdull;
	x ^= x >> 33;
	x *= 0xc4ceb9fe1a85ec53ull;
	x ^= x >> 33;
	return static_cast<uint32_t>(x);
}

// He-uniform weights (bound sqrt(6 / fan_in)) from a counter hash; zero biases.
__global__ void mlp_init_kernel(float* __restrict__ p, uint64_t seed) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kNP; i += gridDim.x * blockDim.x) {
		int fan_in = 0;
		if (i < kB1) {
			fan_in = kIn;
		} else if (i >= kW2 && i < kB2) {
			fan_in = kH;
		} else if (i >= kW3 && i < kB3) {
			fan_in = kH;
		}
		float w = 0.0f;
		if (fan_in) {
			const float u = (hash32(seed * 0x9e3779b97f4a7c15ull + static_cast<uint64_t>(i)) >> 8) * (1.0f / 16777216.0f);
			w             = (2.0f * u - 1.0f) * sqrtf(6.0f / static_cast<float>(fan_in));
		}
		p[i] = w;
	}
}

__device__ __forceinline__ void load_params(const float* __restrict__ g, float* s) {
	for (int i = threadIdx.x; i < kNP; i += blockDim.x) { s[i] = g[i]; }
	__syncthreads();
}

// Forward of one sample with the parameters in shared memory: h1 in registers,
// h2 produced one unit at a time straight into the logits.
__device__ __forceinline__ void forward_one(const float* __restrict__ P, const float* __restrict__ x, float (&h1)[kH],
                                            float (&z)[kOut], float* h2_out) {
	float xin[kIn];
#pragma unroll
	for (int i = 0; i < kIn; ++i) { xin[i] = x[i]; }
	// P is 16-byte aligned and every weight row starts at a multiple of four
	// floats (kW1 = 0, kW2 = 1088): rows are read four weights per load
	static_assert(kW1 % 4 == 0 && kW2 % 4 == 0 && kIn % 4 == 0 && kH % 4 == 0, "float4 weight rows");
#pragma unroll
	for (int j = 0; j < kH; ++j) {
		const float4* w = reinterpret_cast<const float4*>(P + kW1 + j * kIn);
		float         a = P[kB1 + j];
#pragma unroll
		for (int i4 = 0; i4 < kIn / 4; ++i4) {
			const float4 q = w[i4];
			a = fmaf(q.x, xin[4 * i4], a);
			a = fmaf(q.y, xin[4 * i4 + 1], a);
			a = fmaf(q.z, xin[4 * i4 + 2], a);
			a = fmaf(q.w, xin[4 * i4 + 3], a);
		}
		h1[j] = fmaxf(a, 0.0f);
	}
#pragma unroll
	for (int k = 0; k < kOut; ++k) { z[k] = P[kB3 + k]; }
#pragma unroll 1
	for (int j = 0; j < kH; ++j) {
		// four partial sums: four independent FMA chains of 16 instead of one
		// of 64 (the sum's rounding is that of this order, fixed)
		const float4* w     = reinterpret_cast<const float4*>(P + kW2 + j * kH);
		float         a4[4] = {P[kB2 + j], 0.0f, 0.0f, 0.0f};
#pragma unroll
		for (int i4 = 0; i4 < kH / 4; ++i4) {
			const float4 q = w[i4];
			a4[0]          = fmaf(q.x, h1[4 * i4], a4[0]);
			a4[1]          = fmaf(q.y, h1[4 * i4 + 1], a4[1]);
			a4[2]          = fmaf(q.z, h1[4 * i4 + 2], a4[2]);
			a4[3]          = fmaf(q.w, h1[4 * i4 + 3], a4[3]);
		}
		float a = (a4[0] + a4[1]) + (a4[2] + a4[3]);
		a = fmaxf(a, 0.0f);
		if (h2_out) { h2_out[j] = a; }
#pragma unroll
		for (int k = 0; k < kOut; ++k) { z[k] = fmaf(P[kW3 + k * kH + j], a, z[k]); }
	}
}

__device__ __forceinline__ void softmax5(float (&z)[kOut]) {
	float m = z[0];
#pragma unroll
	for (int k = 1; k < kOut; ++k) { m = fmaxf(m, z[k]); }
	float s = 0.0f;
#pragma unroll
	for (int k = 0; k < kOut; ++k) {
		z[k] = expf(z[k] - m);
		s += z[k];
	}
	const float inv = 1.0f / s;
#pragma unroll
	for (int k = 0; k < kOut; ++k) { z[k] *= inv; }
}

__global__ void __launch_bounds__(256, 2) mlp_infer_kernel(const float* __restrict__ params, const float* __restrict__ x,
                                                        uint64_t n, float* __restrict__ probs, uint8_t* __restrict__ best,
                                                        float* __restrict__ conf) {
	// One sample per thread and no sample loop, so the compiler has no reason to
	// hoist the shared-memory weights into registers.  Every thread reads the
	// same weight at the same time: shared-memory broadcasts.
	__shared__ __align__(16) float P[kNP];
	load_params(params, P);
	const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (i < n) {
		float h1[kH], z[kOut];
		forward_one(P, x + i * kIn, h1, z, nullptr);
		softmax5(z);
		int   arg = 0;
		float top = z[0];
#pragma unroll
		for (int k = 1; k < kOut; ++k) {
			if (z[k] > top) {
				top = z[k];
				arg = k;
			}
		}
		if (probs) {
#pragma unroll
			for (int k = 0; k < kOut; ++k) { probs[i * kOut + k] = z[k]; }
		}
		if (best) { best[i] = static_cast<uint8_t>(arg); }
		if (conf) { conf[i] = top; }
	}
}

// Training forward: stores h1, h2 and (softmax - onehot)/B (the logit
// gradient of the mean cross-entropy); accumulates the loss sum.
__global__ void __launch_bounds__(256) mlp_train_fwd_kernel(const float* __restrict__ params,
                                                            const float* __restrict__ x, const uint8_t* __restrict__ y,
                                                            uint32_t B, float* __restrict__ H1, float* __restrict__ H2,
                                                            float* __restrict__ dZ, float* __restrict__ loss) {
	__shared__ __align__(16) float P[kNP];
	load_params(params, P);
	const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
	float          l = 0.0f;
	if (b < B) {
		float h1[kH], z[kOut];
		forward_one(P, x + static_cast<uint64_t>(b) * kIn, h1, z, H2 + static_cast<uint64_t>(b) * kH);
#pragma unroll
		for (int j = 0; j < kH; ++j) { H1[static_cast<uint64_t>(b) * kH + j] = h1[j]; }
		softmax5(z);
		const int   t   = y[b] < kOut ? y[b] : 0;
		const float inv = 1.0f / static_cast<float>(B);
#pragma unroll
		for (int k = 0; k < kOut; ++k) { dZ[static_cast<uint64_t>(b) * kOut + k] = (z[k] - (k == t ? 1.0f : 0.0f)) * inv; }
		l = -logf(fmaxf(z[t], 1e-30f));
	}
	for (int o = 16; o > 0; o >>= 1) { l += __shfl_xor_sync(0xffffffffu, l, o); }
	if ((threadIdx.x & 31) == 0 && loss) { atomicAdd(loss, l / static_cast<float>(B)); }
}

// Backward through the activations: dH2 = relu'(h2) * dZ W3, dH1 = relu'(h1) * dH2 W2.
__global__ void __launch_bounds__(256) mlp_train_bwd_kernel(const float* __restrict__ params, uint32_t B,
                                                            const float* __restrict__ H1, const float* __restrict__ H2,
                                                            const float* __restrict__ dZ, float* __restrict__ dH1,
                                                            float* __restrict__ dH2) {
	__shared__ __align__(16) float P[kNP];
	load_params(params, P);
	const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
	if (b >= B) { return; }
	float dz[kOut];
#pragma unroll
	for (int k = 0; k < kOut; ++k) { dz[k] = dZ[static_cast<uint64_t>(b) * kOut + k]; }
	float g2[kH];
#pragma unroll
	for (int j = 0; j < kH; ++j) {
		float a = 0.0f;
#pragma unroll
		for (int k = 0; k < kOut; ++k) { a = fmaf(P[kW3 + k * kH + j], dz[k], a); }
		g2[j] = H2[static_cast<uint64_t>(b) * kH + j] > 0.0f ? a : 0.0f;
		dH2[static_cast<uint64_t>(b) * kH + j] = g2[j];
	}
	for (int i = 0; i < kH; ++i) {
		float a = 0.0f;
#pragma unroll
		for (int j = 0; j < kH; ++j) { a = fmaf(P[kW2 + j * kH + i], g2[j], a); }
		dH1[static_cast<uint64_t>(b) * kH + i] = H1[static_cast<uint64_t>(b) * kH + i] > 0.0f ? a : 0.0f;
	}
}

// Weight gradients: block r < 64 -> row r of W1/b1 (inputs x), 64..127 -> W2/b2
// (inputs h1), 128..132 -> W3/b3 (inputs h2); sum over the batch.
__global__ void __launch_bounds__(256) mlp_grad_kernel(const float* __restrict__ x, uint32_t B,
                                                       const float* __restrict__ H1, const float* __restrict__ H2,
                                                       const float* __restrict__ dZ, const float* __restrict__ dH1,
                                                       const float* __restrict__ dH2, float* __restrict__ grads) {
	const int    row = blockIdx.x;
	const float* A;
	const float* dA;
	int          in_dim, stride_d, w_off, b_off, j;
	if (row < kH) {
		A = x, in_dim = kIn, dA = dH1, stride_d = kH, j = row, w_off = kW1, b_off = kB1;
	} else if (row < 2 * kH) {
		A = H1, in_dim = kH, dA = dH2, stride_d = kH, j = row - kH, w_off = kW2, b_off = kB2;
	} else {
		A = H2, in_dim = kH, dA = dZ, stride_d = kOut, j = row - 2 * kH, w_off = kW3, b_off = kB3;
	}
	float acc[kH];
#pragma unroll
	for (int i = 0; i < kH; ++i) { acc[i] = 0.0f; }
	float bacc = 0.0f;
	for (uint32_t b = threadIdx.x; b < B; b += blockDim.x) {
		const float d = dA[static_cast<uint64_t>(b) * stride_d + j];
		bacc += d;
		const float* a = A + static_cast<uint64_t>(b) * in_dim;
#pragma unroll
		for (int i = 0; i < kH; ++i) {
			if (i < in_dim) { acc[i] = fmaf(d, a[i], acc[i]); }
		}
	}
	__shared__ float red[8][kH + 1];
	const int        lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
	for (int i = 0; i < kH + 1; ++i) {
		float v = i < kH ? acc[i] : bacc;
		for (int o = 16; o > 0; o >>= 1) { v += __shfl_xor_sync(0xffffffffu, v, o); }
		if (lane == 0) { red[w][i] = v; }
	}
	__syncthreads();
	if (threadIdx.x <= kH) {
		const int i = threadIdx.x;
		float     s = 0.0f;
		for (int ww = 0; ww < static_cast<int>(blockDim.x >> 5); ++ww) { s += red[ww][i]; }
		if (i < in_dim) { grads[w_off + j * in_dim + i] = s; }
		if (i == kH) { grads[b_off + j] = s; }
	}
}

__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= kNP) { return; }
	const float gi = g[i];
	const float mi = b1 * m[i] + (1.0f - b1) * gi;
	const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
	m[i]           = mi;
	v[i]           = vi;
	p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

size_t align256(size_t x) { return (x + 255u) & ~static_cast<size_t>(255u); }

// Scratch of fls_mlp_gradients_static: h1, h2, dh1, dh2 (each
// FLS_MLP_STATIC_MAX_BATCH x 64 floats) and dz (FLS_MLP_STATIC_MAX_BATCH x 5
// floats), about 2.1 MB held by every device that loads this library.
constexpr uint32_t kStaticBatch        = FLS_MLP_STATIC_MAX_BATCH;
constexpr size_t   kStaticScratchFloats = 4u * kStaticBatch * kH + kStaticBatch * kOut;
static __device__ __align__(256) float g_mlp_static_scratch[kStaticScratchFloats];

// Device address of g_mlp_static_scratch, resolved once per device (host
// code may not use the symbol itself as a device pointer).
std::mutex          g_static_mu;
std::vector<float*> g_static_ptr;

fls_status static_scratch(float** out) {
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) {
		cudaGetLastError();
		return set_error(FLS_ERR_NO_DEVICE, "no CUDA device");
	}
	std::lock_guard<std::mutex> lk(g_static_mu);
	if (static_cast<int>(g_static_ptr.size()) <= dev) { g_static_ptr.resize(dev + 1, nullptr); }
	if (!g_static_ptr[dev]) {
		float*      ptr = nullptr;
		cudaError_t e   = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_mlp_static_scratch);
		if (e != cudaSuccess || !ptr) {
			return set_error(FLS_ERR_CUDA, std::string("cudaGetSymbolAddress(static MLP scratch): ") + cudaGetErrorString(e));
		}
		g_static_ptr[dev] = ptr;
	}
	*out = g_static_ptr[dev];
	return FLS_OK;
}

} // namespace
} // namespace fls

using namespace fls;

extern "C" {

fls_status fls_vector_stats_gpu(const int32_t* d_values, uint64_t n, float* d_stats, fls_stream_t stream) {
	if (!d_values || !d_stats || n == 0) { return set_error(FLS_ERR_INVALID_ARG, "fls_vector_stats_gpu: bad arguments"); }
	if (fls_status s = check_n_values(n, "fls_vector_stats_gpu"); s != FLS_OK) { return s; }
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	const uint64_t n_vec = (n + 1023u) / 1024u;
	const uint32_t grid  = static_cast<uint32_t>(std::min<uint64_t>((n_vec + 7u) / 8u, static_cast<uint64_t>(di.sms) * 4u));
	stats_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_values, n, n_vec, d_stats);
	count_launch();
	return cuda_check(cudaGetLastError(), "stats_kernel launch");
}

fls_status fls_mlp_init(float* d_params, uint64_t seed, fls_stream_t stream) {
	if (!d_params) { return set_error(FLS_ERR_INVALID_ARG, "fls_mlp_init: null params"); }
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	mlp_init_kernel<<<(kNP + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_params, seed);
	count_launch();
	return cuda_check(cudaGetLastError(), "mlp_init_kernel launch");
}

uint64_t fls_mlp_workspace_bytes(uint32_t batch) {
	const size_t b = batch;
	return align256(b * kH * 4) * 4 + align256(b * kOut * 4);
}

fls_status fls_mlp_gradients(const float* d_params, const float* d_x, const uint8_t* d_labels, uint32_t batch,
                             void* d_ws, uint64_t ws_bytes, float* d_grads, float* d_loss, fls_stream_t stream) {
	if (!d_params || !d_x || !d_labels || !d_ws || !d_grads || batch == 0) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_mlp_gradients: bad arguments");
	}
	if (ws_bytes < fls_mlp_workspace_bytes(batch)) { return set_error(FLS_ERR_CAPACITY, "MLP workspace too small"); }
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	char*        w   = static_cast<char*>(d_ws);
	const size_t hb  = align256(static_cast<size_t>(batch) * kH * 4);
	float*       H1  = reinterpret_cast<float*>(w);
	float*       H2  = reinterpret_cast<float*>(w + hb);
	float*       dH1 = reinterpret_cast<float*>(w + 2 * hb);
	float*       dH2 = reinterpret_cast<float*>(w + 3 * hb);
	float*       dZ  = reinterpret_cast<float*>(w + 4 * hb);
	cudaStream_t st  = reinterpret_cast<cudaStream_t>(stream);
	if (d_loss && (s = cuda_check(cudaMemsetAsync(d_loss, 0, sizeof(float), st), "cudaMemsetAsync")) != FLS_OK) {
		return s;
	}
	const uint32_t g = (batch + 255u) / 256u;
	mlp_train_fwd_kernel<<<g, 256, 0, st>>>(d_params, d_x, d_labels, batch, H1, H2, dZ, d_loss);
	mlp_train_bwd_kernel<<<g, 256, 0, st>>>(d_params, batch, H1, H2, dZ, dH1, dH2);
	mlp_grad_kernel<<<2 * kH + kOut, 256, 0, st>>>(d_x, batch, H1, H2, dZ, dH1, dH2, d_grads);
	count_launch(3);
	return cuda_check(cudaGetLastError(), "MLP gradient kernels launch");
}

// Same result as fls_mlp_gradients, for callers that cannot allocate device
// memory: the activation scratch lives in a fixed static device array instead
// of a caller workspace.  See include/fls_gpu.h.
fls_status fls_mlp_gradients_static(const float* d_params, const float* d_x, const uint8_t* d_labels, uint32_t batch,
                                    float* d_grads, float* d_loss, fls_stream_t stream) {
	if (!d_params || !d_x || !d_labels || !d_grads || batch == 0) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_mlp_gradients_static: bad arguments");
	}
	if (batch > kStaticBatch) {
		return set_error(FLS_ERR_CAPACITY, "fls_mlp_gradients_static: batch " + std::to_string(batch) +
		                                       " exceeds FLS_MLP_STATIC_MAX_BATCH (" + std::to_string(kStaticBatch) + ")");
	}
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	float* scratch = nullptr;
	if ((s = static_scratch(&scratch)) != FLS_OK) { return s; }
	float*       H1  = scratch;
	float*       H2  = H1 + static_cast<size_t>(kStaticBatch) * kH;
	float*       dH1 = H2 + static_cast<size_t>(kStaticBatch) * kH;
	float*       dH2 = dH1 + static_cast<size_t>(kStaticBatch) * kH;
	float*       dZ  = dH2 + static_cast<size_t>(kStaticBatch) * kH;
	cudaStream_t st  = reinterpret_cast<cudaStream_t>(stream);
	if (d_loss && (s = cuda_check(cudaMemsetAsync(d_loss, 0, sizeof(float), st), "cudaMemsetAsync")) != FLS_OK) {
		return s;
	}
	const uint32_t g = (batch + 255u) / 256u;
	mlp_train_fwd_kernel<<<g, 256, 0, st>>>(d_params, d_x, d_labels, batch, H1, H2, dZ, d_loss);
	mlp_train_bwd_kernel<<<g, 256, 0, st>>>(d_params, batch, H1, H2, dZ, dH1, dH2);
	mlp_grad_kernel<<<2 * kH + kOut, 256, 0, st>>>(d_x, batch, H1, H2, dZ, dH1, dH2, d_grads);
	count_launch(3);
	return cuda_check(cudaGetLastError(), "static-scratch MLP gradient kernels launch");
}

fls_status fls_mlp_adam_step(float* d_params, const float* d_grads, float* d_m, float* d_v, float lr, float beta1,
                             float beta2, float eps, uint32_t t, fls_stream_t stream) {
	if (!d_params || !d_grads || !d_m || !d_v || t == 0) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_mlp_adam_step: bad arguments");
	}
	const float c1 = 1.0f - powf(beta1, static_cast<float>(t));
	const float c2 = 1.0f - powf(beta2, static_cast<float>(t));
	mlp_adam_kernel<<<(kNP + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_params, d_grads, d_m, d_v,
	                                                                                      lr, beta1, beta2, eps, c1, c2);
	count_launch();
	return cuda_check(cudaGetLastError(), "mlp_adam_kernel launch");
}

fls_status fls_mlp_infer(const float* d_params, const float* d_x, uint64_t n, float* d_probs, uint8_t* d_best,
                         float* d_conf, fls_stream_t stream) {
	if (!d_params || !d_x || n == 0) { return set_error(FLS_ERR_INVALID_ARG, "fls_mlp_infer: bad arguments"); }
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	if (n > (static_cast<uint64_t>(1) << 36)) { return set_error(FLS_ERR_CAPACITY, "fls_mlp_infer: too many samples"); }
	const uint32_t grid = static_cast<uint32_t>((n + 255u) / 256u);
	mlp_infer_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_params, d_x, n, d_probs, d_best,
	                                                                          d_conf);
	count_launch();
	return cuda_check(cudaGetLastError(), "mlp_infer_kernel launch");
}

} // extern "C"
