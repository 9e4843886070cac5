// fls_jit.cu -- query specialisation for filter-aggregate on uniform FOR columns.
//
// fls_query_filter_agg hands queries whose columns are all uniform FOR (the
// reference's format, fls_q11.cu:202-223) to fls::jit_filter_agg.  It compiles
// fls::fixed::run (fls_fixed.cuh) for the query's exact shape with NVRTC the
// first time that shape is seen, loads the cubin with cudaLibraryLoadData and
// caches the kernel by shape for the life of the process.  NVRTC is opened
// with dlopen, so the library loads and the general kernel still runs where
// NVRTC is absent; a failed compile or load is cached as a failure and the
// caller falls back to the general kernel.
#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "fls_fixed.cuh"
#include "fls_internal.h"
#include "fls_jit_headers.inc" // kJitHeaders: the headers above as text (generated by build.py)
#include "fls_pipeline.cuh"

namespace fls {
namespace {

struct Nvrtc {
	decltype(&nvrtcCreateProgram)  create  = nullptr;
	decltype(&nvrtcCompileProgram) compile = nullptr;
	decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
	decltype(&nvrtcGetProgramLog)  log     = nullptr;
	decltype(&nvrtcGetCUBINSize)   cubin_size = nullptr;
	decltype(&nvrtcGetCUBIN)       cubin   = nullptr;
	decltype(&nvrtcDestroyProgram) destroy = nullptr;
	bool                           ok      = false;
};

const Nvrtc& nvrtc() {
	static Nvrtc n = [] {
		Nvrtc r;
		const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
		void*       h       = nullptr;
		for (const char* nm : names) {
			if ((h = dlopen(nm, RTLD_NOW | RTLD_LOCAL)) != nullptr) { break; }
		}
		if (!h) { return r; }
		r.create     = reinterpret_cast<decltype(r.create)>(dlsym(h, "nvrtcCreateProgram"));
		r.compile    = reinterpret_cast<decltype(r.compile)>(dlsym(h, "nvrtcCompileProgram"));
		r.log_size   = reinterpret_cast<decltype(r.log_size)>(dlsym(h, "nvrtcGetProgramLogSize"));
		r.log        = reinterpret_cast<decltype(r.log)>(dlsym(h, "nvrtcGetProgramLog"));
		r.cubin_size = reinterpret_cast<decltype(r.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
		r.cubin      = reinterpret_cast<decltype(r.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
		r.destroy    = reinterpret_cast<decltype(r.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
		r.ok = r.create && r.compile && r.log_size && r.log && r.cubin_size && r.cubin && r.destroy;
		return r;
	}();
	return n;
}

struct Entry {
	int                 state = 0; // 1 compiled, 2 loaded, -1 failed
	std::vector<char>   cubin;
	cudaLibrary_t       lib {};
	cudaKernel_t        kernel {};
	std::vector<size_t> smem_set; // per device: dynamic shared memory the attribute allows
};

std::mutex                             g_mu;
std::unordered_map<std::string, Entry> g_cache;
std::string                            g_last_log;
std::atomic<uint64_t>                  g_compiled {0}, g_launches {0}, g_failures {0};

// Headers NVRTC sees besides kJitHeaders: minimal stand-ins for the system
// headers they include (device code needs only the fixed-width types).
const char* const kStdint =
    "#pragma once\n"
    "typedef signed char int8_t; typedef short int16_t; typedef int int32_t; typedef long long int64_t;\n"
    "typedef unsigned char uint8_t; typedef unsigned short uint16_t; typedef unsigned int uint32_t;\n"
    "typedef unsigned long long uint64_t; typedef unsigned long long uintptr_t;\n";
const char* const kStddef = "#pragma once\ntypedef decltype(sizeof(0)) size_t;\n";
const char* const kEmpty  = "#pragma once\n";

// Kernel keys are "<op>:<warps>:<template arguments>"; op F = filter-aggregate,
// P = probe + group-by, D = decode.  The warp count fixes __launch_bounds__ so that the
// compiler may use every register the launch leaves.
std::string shape_source(const std::string& key) {
	const size_t a = key.find(':'), b = key.find(':', a + 1);
	const std::string op = key.substr(0, a), warps = key.substr(a + 1, b - a - 1), args = key.substr(b + 1);
	const char* params = op == "F" ? "FilterParams" : op == "P" ? "ProbeParams" : "DecodeParams";
	const char* body   = op == "F"   ? "filter_kernel<fls::fixed::FilterQuery<"
	                     : op == "P" ? "probe_kernel<fls::fixed::ProbeQuery<"
	                                 : "decode_kernel<fls::fixed::DecodeQuery<";
	return std::string("#include \"fls_fixed.cuh\"\n") + "extern \"C\" __global__ void __launch_bounds__(32 * " + warps +
	       ", 1)\nfls_fixed_kernel(const __grid_constant__ fls::fixed::" + params + " P) {\n\tfls::fixed::" + body +
	       args + ">>(P);\n}\n";
}

// NVRTC compile of one shape into e.cubin; false (log kept) on failure.
bool compile_shape(const std::string& key, Entry& e) {
	const Nvrtc& n = nvrtc();
	if (!n.ok) {
		g_last_log = "NVRTC library not found";
		return false;
	}
	std::vector<const char*> names, texts;
	for (const auto& h : kJitHeaders) {
		names.push_back(h.name);
		texts.push_back(h.text);
	}
	names.push_back("stdint.h");
	texts.push_back(kStdint);
	names.push_back("stddef.h");
	texts.push_back(kStddef);
	names.push_back("cuda_runtime.h");
	texts.push_back(kEmpty);
	const std::string src = shape_source(key);
	nvrtcProgram      prog;
	if (n.create(&prog, src.c_str(), "fls_fixed_query.cu", static_cast<int>(names.size()), texts.data(),
	             names.data()) != NVRTC_SUCCESS) {
		g_last_log = "nvrtcCreateProgram failed";
		return false;
	}
	// -default-device: the public header's host API declarations become unused
	// device declarations.
	const char*       opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-lineinfo", "-default-device",
	                            "-DFLS_JIT=1"};
	const nvrtcResult rc     = n.compile(prog, 5, opts);
	size_t            ls     = 0;
	n.log_size(prog, &ls);
	std::string log(ls, '\0');
	if (ls) { n.log(prog, &log[0]); }
	if (rc != NVRTC_SUCCESS) {
		g_last_log = key + ": " + log;
		n.destroy(&prog);
		return false;
	}
	size_t cs = 0;
	n.cubin_size(prog, &cs);
	e.cubin.resize(cs);
	n.cubin(prog, e.cubin.data());
	n.destroy(&prog);
	return cs > 0;
}

bool load_shape(Entry& e) {
	if (cudaLibraryLoadData(&e.lib, e.cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess) {
		g_last_log = std::string("cudaLibraryLoadData: ") + cudaGetErrorString(cudaGetLastError());
		return false;
	}
	if (cudaLibraryGetKernel(&e.kernel, e.lib, "fls_fixed_kernel") != cudaSuccess) {
		g_last_log = std::string("cudaLibraryGetKernel: ") + cudaGetErrorString(cudaGetLastError());
		cudaLibraryUnload(e.lib);
		return false;
	}
	return true;
}

// The cache entry of a shape, compiled if new (caller holds g_mu).
Entry& compiled_entry(const std::string& key) {
	auto it = g_cache.find(key);
	if (it == g_cache.end()) {
		Entry e;
		e.state = compile_shape(key, e) ? 1 : -1;
		(e.state > 0 ? g_compiled : g_failures).fetch_add(1);
		it = g_cache.emplace(key, std::move(e)).first;
	}
	return it->second;
}

// Stage plan of a specialised kernel: tiles of k vectors, S stages per warp,
// as many warps (up to the launch configuration's) as shared memory holds
// next to cta_words of CTA-wide tables.
// join: the probe + group-by kernels, which take up to jit_max_warps() warps;
// the filter and decode kernels keep the launch configuration's (16 by
// default: measured faster for them).
fls_status plan_fixed(const DeviceInfo& di, const fls_column* sc, uint32_t n, uint32_t cta_words,
                      fixed::StageParams& S, uint32_t& grid, size_t& smem, bool join = false, bool half = false) {
	fls_status st       = FLS_OK;
	uint32_t   W0 = 0, S0 = 0, ctas = 0, tile_bytes = 0;
	fls_get_launch_config(&W0, &S0, &ctas, &tile_bytes);
	if (join) {
		// half-vector stages fit about twice the warps; registers allow 28
		W0 = jit_max_warps();
		if (half && W0 == kJitDefaultWarps) { W0 = kJitHalfWarps; }
	}
	std::memset(&S, 0, sizeof(S));
	uint32_t sum_vec = 0;
	for (uint32_t c = 0; c < n; ++c) {
		DevCol d;
		if ((st = make_devcol(sc[c], d)) != FLS_OK) { return st; }
		if (sc[c].n_values != sc[0].n_values) { return set_error(FLS_ERR_INVALID_ARG, "columns differ in length"); }
		S.data[c] = sc[c].data;
		// half-vector tiles: ceil(bw/2) word rows of each column
		sum_vec += half ? 32u * ((sc[c].bw + 1u) / 2u) : 32u * sc[c].bw;
	}
	S.n_values = sc[0].n_values;
	S.n_vec    = (S.n_values + 1023u) / 1024u;
	const uint64_t total_warps = static_cast<uint64_t>(di.sms) * ctas * W0;
	uint32_t       k = sum_vec ? std::max<uint32_t>(1u, tile_bytes / (4u * sum_vec)) : kMaxTile;
	k                = half ? 1u : std::min<uint32_t>(k, kMaxTile);
	while (k > 1 && (S.n_vec + k - 1) / k < 4 * total_warps) { k /= 2; }
	const uint32_t avail = static_cast<uint32_t>(di.max_smem) / 4u;
	// a warp's area: its stages, the slack, one barrier per stage and (join
	// kernels) its row list
	const uint32_t list_words = join ? fixed::kRowListWords : 0u;
	auto warp_words = [&](uint32_t stages_) {
		return (stages_ * k * sum_vec + fixed::kSlack + 2u * stages_ + list_words + 3u) & ~3u;
	};
	auto warps_for  = [&](uint32_t per_) {
		return avail > cta_words ? std::min<uint32_t>(W0, (avail - cta_words) / per_) : 0u;
	};
	uint32_t stages = S0, W = 0, per = 0;
	for (;;) {
		per = warp_words(stages);
		W   = warps_for(per);
		if (W >= std::min<uint32_t>(W0, 8u) || (k == 1 && stages <= 2)) { break; }
		if (k > 1) {
			k /= 2;
		} else {
			--stages;
		}
	}
	// Wide rows (joins next to their tables): one stage per warp when that
	// holds more warps.  Warps hide the copy latency of each other's stages,
	// and the measured joins run faster with more warps than with more stages.
	if (W < W0 && k == 1 && stages > 1 && warps_for(warp_words(1)) > W) {
		stages = 1;
		per    = warp_words(1);
		W      = warps_for(per);
	}
	if (W == 0) { return set_error(FLS_ERR_CAPACITY, "vectors and tables too large for shared memory"); }
	S.tile            = k;
	S.n_tiles         = half ? 2u * S.n_vec : (S.n_vec + k - 1) / k;
	S.stages          = stages;
	S.warps           = W;
	S.stage_words     = k * sum_vec;
	S.bar_off         = stages * S.stage_words + fixed::kSlack;
	S.list_off        = S.bar_off + 2u * stages;
	S.warp_smem_words = per;
	S.cta_off         = W * per;
	smem              = 4ull * (static_cast<size_t>(S.cta_off) + cta_words);
	grid = static_cast<uint32_t>(std::min<uint64_t>((S.n_tiles + W - 1) / W, static_cast<uint64_t>(di.sms) * ctas));
	return FLS_OK;
}

// Loads (first use) and launches the kernel of `key`; used = false if the
// shape could not be compiled or loaded.
fls_status launch_fixed(const std::string& key, void* params, uint32_t grid, uint32_t threads, size_t smem,
                        cudaStream_t stream, bool& used) {
	used    = false;
	int dev = 0;
	fls_status s = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
	if (s != FLS_OK) { return s; }
	cudaKernel_t kernel {};
	{
		std::lock_guard<std::mutex> lk(g_mu);
		Entry&                      e = compiled_entry(key);
		if (e.state == 1) {
			e.state = load_shape(e) ? 2 : -1;
			if (e.state < 0) { g_failures.fetch_add(1); }
		}
		if (e.state != 2) { return FLS_OK; }
		if (e.smem_set.size() <= static_cast<size_t>(dev)) { e.smem_set.resize(dev + 1, 0); }
		if (smem > 48u * 1024u && e.smem_set[dev] < smem) {
			s = cuda_check(cudaKernelSetAttributeForDevice(e.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			                                               static_cast<int>(smem), dev),
			               "cudaKernelSetAttributeForDevice");
			if (s != FLS_OK) { return s; }
			e.smem_set[dev] = smem;
		}
		kernel = e.kernel;
	}
	void* argv[] = {params};
	s = cuda_check(cudaLaunchKernel(reinterpret_cast<const void*>(kernel), dim3(grid), dim3(threads), argv, smem, stream),
	               "cudaLaunchKernel (specialised kernel)");
	if (s != FLS_OK) { return s; }
	count_launch();
	g_launches.fetch_add(1);
	used = true;
	return FLS_OK;
}

std::string key_args(const fls_column* sc, uint32_t n, const char* head) {
	std::string k = head;
	for (uint32_t i = 0; i < n; ++i) { k += ", " + std::to_string(static_cast<unsigned>(sc[i].bw)); }
	return k;
}

std::string make_key(char op, uint32_t warps, const std::string& args) {
	return std::string(1, op) + ":" + std::to_string(warps) + ":" + args;
}

// The device a plan is made for: the current one, or (compiling ahead without
// a device) an sm_100 B200: 148 SMs, 227 KB of shared memory per CTA.
DeviceInfo plan_device(bool& have_device) {
	DeviceInfo di;
	have_device = device_info(di) == FLS_OK;
	if (!have_device) {
		di.sms      = 148;
		di.max_smem = 232448;
		di.major    = 10;
	}
	return di;
}

bool uniform_for(const fls_column& c, uint32_t layout) {
	return c.meta == nullptr && c.scheme == FLS_SCHEME_FOR && c.bw <= 32 && c.layout == layout;
}

} // namespace

bool jit_shape(const fls_column* cols, const fls_filter* filters, uint32_t n_filters, int32_t agg_a, int32_t agg_b,
               JitShape& sh) {
	sh.n_staged = 0;
	for (uint32_t f = 0; f < n_filters; ++f) {
		for (uint32_t g = 0; g < f; ++g) {
			if (filters[g].col == filters[f].col) { return false; } // two ranges on one column
		}
		sh.staged[sh.n_staged++] = filters[f].col;
	}
	auto slot_of = [&](int32_t c) -> int {
		if (c < 0) { return -1; }
		for (uint32_t i = 0; i < sh.n_staged; ++i) {
			if (sh.staged[i] == static_cast<uint32_t>(c)) { return static_cast<int>(i); }
		}
		sh.staged[sh.n_staged] = static_cast<uint32_t>(c);
		return static_cast<int>(sh.n_staged++);
	};
	sh.agg_a = slot_of(agg_a);
	sh.agg_b = slot_of(agg_b);
	if (sh.n_staged == 0) { return false; }
	fls_column sc[FLS_MAX_QUERY_COLS];
	for (uint32_t i = 0; i < sh.n_staged; ++i) {
		sc[i] = cols[sh.staged[i]];
		if (!uniform_for(sc[i], sc[0].layout)) { return false; }
	}
	// Filters that may test several packed fields at once: widths with a SWAR
	// form (4, or even up to 14) on columns whose decoded values cannot wrap.
	uint32_t swar = 0;
	for (uint32_t f = 0; f < n_filters; ++f) {
		const uint32_t bw = sc[f].bw;
		const bool     form = bw == 4 || (bw % 2 == 0 && bw >= 2 && bw <= 14);
		if (form && static_cast<int64_t>(sc[f].base) + (int64_t {1} << bw) - 1 <= INT32_MAX) { swar |= 1u << f; }
	}
	sh.swar = swar;
	char head[96];
	std::snprintf(head, sizeof(head), "%u, %u, %d, %d, %u", static_cast<unsigned>(sc[0].layout), n_filters, sh.agg_a,
	              sh.agg_b, swar);
	sh.key = key_args(sc, sh.n_staged, head);
	return true;
}

bool jit_compile(const fls_column* cols, const JitShape& sh) {
	fls_column sc[FLS_MAX_QUERY_COLS];
	for (uint32_t i = 0; i < sh.n_staged; ++i) { sc[i] = cols[sh.staged[i]]; }
	bool                have;
	const DeviceInfo    di = plan_device(have);
	fixed::StageParams  S;
	uint32_t            grid;
	size_t              smem;
	if (plan_fixed(di, sc, sh.n_staged, 0u, S, grid, smem) != FLS_OK) { return false; }
	std::lock_guard<std::mutex> lk(g_mu);
	return compiled_entry(make_key('F', S.warps, sh.key)).state > 0;
}

fls_status jit_filter_agg(const fls_column* cols, const fls_filter* filters, uint32_t n_filters, int32_t agg_a,
                          int32_t agg_b, int64_t* d_result, int32_t sparse_rows, cudaStream_t stream, bool& used) {
	used = false;
	JitShape sh;
	if (!jit_shape(cols, filters, n_filters, agg_a, agg_b, sh)) { return FLS_OK; }
	fls_column sc[FLS_MAX_QUERY_COLS];
	for (uint32_t i = 0; i < sh.n_staged; ++i) { sc[i] = cols[sh.staged[i]]; }
	fixed::FilterParams P {};
	uint32_t            grid;
	size_t              smem;
	DeviceInfo          di;
	fls_status          s = device_info(di);
	if (s != FLS_OK) { return s; }
	if ((s = plan_fixed(di, sc, sh.n_staged, 0u, P.S, grid, smem)) != FLS_OK) { return s; }
	P.S.err = device_error_word(stream);
	for (uint32_t i = 0; i < sh.n_staged; ++i) { P.base[i] = static_cast<uint32_t>(sc[i].base); }
	for (uint32_t f = 0; f < n_filters; ++f) {
		P.lo[f]    = static_cast<uint32_t>(filters[f].lo);
		P.range[f] = static_cast<uint32_t>(filters[f].hi) - static_cast<uint32_t>(filters[f].lo);
		if ((sh.swar >> f) & 1u) {
			// value = base + field exactly, so value in [lo, hi] <=> field in
			// [lo - base, hi - base] within the field's domain [0, 2^bw).
			const int64_t top = (int64_t {1} << sc[f].bw) - 1;
			const int64_t L   = std::max<int64_t>(0, static_cast<int64_t>(filters[f].lo) - sc[f].base);
			const int64_t H   = std::min<int64_t>(top, static_cast<int64_t>(filters[f].hi) - sc[f].base);
			P.field_lo[f]     = L <= H ? static_cast<uint32_t>(L) : 1u;
			P.field_hi[f]     = L <= H ? static_cast<uint32_t>(H) : 0u;
		}
	}
	P.sparse_rows = sparse_rows;
	P.result      = reinterpret_cast<unsigned long long*>(d_result);
	return launch_fixed(make_key('F', P.S.warps, sh.key), &P, grid, 32u * P.S.warps, smem, stream, used);
}

// Presence bitmaps of up to FLS_MAX_PROBES tables: bit i of word w of table j
// (at out + off[j]) is set when slot 32w + i is not zero (PHT_1) or its
// 64-bit entry is not zero (PHT_2).  One warp per word, coalesced reads.
struct PresenceJobs {
	const int32_t* ht[FLS_MAX_PROBES];
	uint32_t       len[FLS_MAX_PROBES];
	uint32_t       off[FLS_MAX_PROBES];
	uint32_t       two[FLS_MAX_PROBES];
	uint32_t       n;
};

__global__ void __launch_bounds__(256) presence_bits_kernel(const __grid_constant__ PresenceJobs J, uint32_t* out) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
	for (uint32_t j = 0; j < J.n; ++j) {
		const uint32_t len = J.len[j], n_words = (len + 31u) / 32u;
		for (uint32_t w = warp; w < n_words; w += nw) {
			const uint32_t idx = 32u * w + lane;
			int32_t        x   = 0;
			if (idx < len) {
				if (J.two[j]) {
					const int2 e = __ldg(reinterpret_cast<const int2*>(J.ht[j]) + idx);
					x            = e.x | e.y;
				} else {
					x = __ldg(J.ht[j] + idx);
				}
			}
			const uint32_t b = __ballot_sync(0xffffffffu, x != 0);
			if (lane == 0) { out[J.off[j] + w] = b; }
		}
	}
}

bool jit_probe_shape(const fls_join_groupby_desc* d, JitProbeShape& sh) {
	sh.n_staged = 0;
	for (uint32_t q = 0; q < d->n_probes; ++q) {
		for (uint32_t g = 0; g < q; ++g) {
			if (d->probes[g].col == d->probes[q].col) { return false; } // one column probed twice
		}
		sh.staged[sh.n_staged++] = d->probes[q].col;
	}
	auto slot_of = [&](int32_t c) -> int {
		if (c < 0) { return -1; }
		for (uint32_t i = 0; i < sh.n_staged; ++i) {
			if (sh.staged[i] == static_cast<uint32_t>(c)) { return static_cast<int>(i); }
		}
		sh.staged[sh.n_staged] = static_cast<uint32_t>(c);
		return static_cast<int>(sh.n_staged++);
	};
	// The measure columns: staged like the probe columns, or (late measures)
	// left in global memory, past the staged ones, and read for the selected
	// rows only.  A measure that is also a probe column is staged anyway.
	const uint32_t n_probe_cols = sh.n_staged;
	sh.agg                      = slot_of(static_cast<int32_t>(d->agg_col));
	sh.sub                      = slot_of(d->agg_sub_col);
	sh.n_global                 = tuning_late_measure() ? sh.n_staged - n_probe_cols : 0u;
	sh.n_staged -= sh.n_global;
	for (uint32_t i = 0; i < sh.n_staged + sh.n_global; ++i) {
		if (!uniform_for(d->cols[sh.staged[i]], d->cols[sh.staged[0]].layout)) { return false; }
	}
	// Tables go to shared memory in probe order while they fit the budget:
	// PHT_1 as bitmaps, PHT_2 verbatim or else as presence bitmaps (payloads
	// then come from global memory, for the selected rows only).  A probe is
	// direct when base + [0, 2^bw) - keys_min lies in [0, len).
	uint32_t kinds = 0, in_smem = 0, pbit = 0, direct = 0;
	sh.cta_words   = 0;
	const uint32_t budget = tuning_table_words();
	auto           place  = [&](uint64_t words, uint32_t q) {
        if (sh.cta_words + words > budget) { return false; }
        sh.smem_off[q] = sh.cta_words;
        sh.cta_words += static_cast<uint32_t>((words + 3u) & ~3ull);
        return true;
	};
	for (uint32_t q = 0; q < d->n_probes; ++q) {
		const fls_probe&  p  = d->probes[q];
		const fls_column& kc = d->cols[p.col];
		const int64_t     lo = static_cast<int64_t>(kc.base) - p.keys_min;
		const int64_t     hi = lo + (kc.bw >= 32 ? (int64_t {1} << 32) : (int64_t {1} << kc.bw)) - 1;
		if (kc.bw < 32 && lo >= 0 && hi < p.ht_len) { direct |= (lo == 0 ? 0x101u : 1u) << q; }
		const uint64_t bits_words = (static_cast<uint64_t>(p.ht_len) + 31u) / 32u;
		sh.smem_off[q]            = 0;
		if (p.kind == 1) {
			if (place(bits_words, q)) { in_smem |= 1u << q; }
		} else {
			kinds |= 1u << q;
			if (place(2ull * static_cast<uint64_t>(p.ht_len), q)) {
				in_smem |= 1u << q;
			} else if (place(bits_words, q)) {
				pbit |= 1u << q;
			}
		}
	}
	sh.tables_words = sh.cta_words;
	sh.bitmaps      = pbit | (in_smem & ~kinds);
	// The group-sum cache after the tables: slots of two sum words and a tag,
	// as many as the groups rounded up to a power of two, at most
	// kJitGroupSlots.
	const uint32_t ng = d->n_groups > 0 ? static_cast<uint32_t>(d->n_groups) : 0u;
	sh.gsm            = tuning_group_smem() && ng > 0;
	sh.gslots         = 1u;
	while (sh.gslots < ng && sh.gslots < kJitGroupSlots) { sh.gslots *= 2u; }
	sh.gsum_off = sh.cta_words;
	if (sh.gsm) { sh.cta_words += 3u * sh.gslots + (4u - (3u * sh.gslots) % 4u) % 4u; }
	fls_column sc[FLS_MAX_QUERY_COLS];
	for (uint32_t i = 0; i < sh.n_staged + sh.n_global; ++i) { sc[i] = d->cols[sh.staged[i]]; }
	int kp[FLS_MAX_GROUP_KEYS] = {-1, -1, -1};
	for (uint32_t k = 0; k < d->n_keys; ++k) { kp[k] = d->key_probe[k]; }
	sh.half = tuning_half_vectors() != 0;
	char head[160];
	std::snprintf(head, sizeof(head), "%u, %u, %d, %d, %u, %d, %d, %d, %u, %u, %u, %u, %d, %d, %u",
	              static_cast<unsigned>(sc[0].layout), d->n_probes, sh.agg, sh.sub, d->n_keys, kp[0], kp[1], kp[2], kinds,
	              in_smem, pbit, direct, sh.gsm ? 1 : 0, sh.half ? 1 : 0, sh.n_staged);
	sh.key = key_args(sc, sh.n_staged + sh.n_global, head);
	return true;
}

bool jit_compile(const fls_join_groupby_desc* d, const JitProbeShape& sh) {
	fls_column sc[FLS_MAX_QUERY_COLS];
	for (uint32_t i = 0; i < sh.n_staged; ++i) { sc[i] = d->cols[sh.staged[i]]; }
	bool               have;
	const DeviceInfo   di = plan_device(have);
	fixed::StageParams S;
	uint32_t           grid;
	size_t             smem;
	if (plan_fixed(di, sc, sh.n_staged, sh.cta_words, S, grid, smem, true, sh.half) != FLS_OK) { return false; }
	std::lock_guard<std::mutex> lk(g_mu);
	return compiled_entry(make_key('P', S.warps, sh.key)).state > 0;
}

uint64_t jit_probe_workspace_bytes(const fls_join_groupby_desc* d) {
	JitProbeShape sh;
	if (!tuning_jit() || !jit_probe_shape(d, sh) || !sh.bitmaps) { return 0u; }
	return 4ull * sh.tables_words;
}

fls_status jit_probe_groupby(const fls_join_groupby_desc* d, int32_t* d_res, int32_t sparse_rows, void* d_ws,
                             uint64_t ws_bytes, cudaStream_t stream, bool& used) {
	used = false;
	JitProbeShape sh;
	if (!jit_probe_shape(d, sh)) { return FLS_OK; }
	if (d_ws && sh.bitmaps && ws_bytes < 4ull * sh.tables_words) {
		return set_error(FLS_ERR_CAPACITY, "join workspace smaller than fls_join_workspace_bytes");
	}
	fls_column sc[FLS_MAX_QUERY_COLS];
	for (uint32_t i = 0; i < sh.n_staged; ++i) { sc[i] = d->cols[sh.staged[i]]; }
	fixed::ProbeParams P {};
	uint32_t           grid;
	size_t             smem;
	DeviceInfo         di;
	fls_status         s = device_info(di);
	if (s != FLS_OK) { return s; }
	if ((s = plan_fixed(di, sc, sh.n_staged, sh.cta_words, P.S, grid, smem, true, sh.half)) != FLS_OK) { return s; }
	P.S.err = device_error_word(stream);
	for (uint32_t i = 0; i < sh.n_staged + sh.n_global; ++i) {
		P.base[i] = static_cast<uint32_t>(d->cols[sh.staged[i]].base);
	}
	for (uint32_t g = 0; g < sh.n_global; ++g) { P.gcol[g] = d->cols[sh.staged[sh.n_staged + g]].data; }
	for (uint32_t q = 0; q < d->n_probes; ++q) {
		P.ht[q]       = d->probes[q].ht;
		P.len[q]      = d->probes[q].ht_len;
		P.kmin[q]     = d->probes[q].keys_min;
		P.smem_off[q] = sh.smem_off[q];
	}
	for (uint32_t k = 0; k < FLS_MAX_GROUP_KEYS; ++k) {
		P.key_mul[k]  = k < d->n_keys ? d->key_mul[k] : 0;
		P.key_slot[k] = k < d->n_keys ? d->key_slot[k] : -1;
	}
	P.sub         = d->group_sub;
	P.n_groups    = d->n_groups;
	P.stride      = d->res_stride;
	P.sum_slot    = d->sum_slot;
	P.sparse_rows = sparse_rows;
	P.gsum_off    = sh.gsum_off;
	P.gslot_mask  = sh.gslots - 1u;
	P.sum32       = d->sum_bits == 32 ? 1u : 0u;
	P.res         = d_res;
	// Presence bitmaps: with a workspace, built once per call for every CTA
	// to copy; without, each CTA builds its own (P.bits = null).
	uint32_t* bits = nullptr;
	if (sh.bitmaps && d_ws) {
		bits = static_cast<uint32_t*>(d_ws);
		PresenceJobs J {};
		for (uint32_t q = 0; q < d->n_probes; ++q) {
			if (!((sh.bitmaps >> q) & 1u)) { continue; }
			J.ht[J.n]  = d->probes[q].ht;
			J.len[J.n] = static_cast<uint32_t>(d->probes[q].ht_len);
			J.off[J.n] = sh.smem_off[q];
			J.two[J.n] = d->probes[q].kind == 2 ? 1u : 0u;
			++J.n;
		}
		presence_bits_kernel<<<2u * di.sms, 256, 0, stream>>>(J, bits);
		count_launch(1);
		if (cudaGetLastError() != cudaSuccess) { return set_error(FLS_ERR_CUDA, "presence bitmap kernel launch failed"); }
	}
	P.bits = bits;
	return launch_fixed(make_key('P', P.S.warps, sh.key), &P, grid, 32u * P.S.warps, smem, stream, used);
}

fls_status jit_decode(const fls_column* col, int mode, uint32_t* d_out, uint64_t* d_sum, cudaStream_t stream,
                      bool& used) {
	used = false;
	if (!uniform_for(*col, col->layout)) { return FLS_OK; }
	const bool no_wrap =
	    col->bw < 32 && static_cast<uint64_t>(static_cast<uint32_t>(col->base)) + (uint64_t {1} << col->bw) - 1u <
	                        (uint64_t {1} << 32);
	fixed::DecodeParams P {};
	uint32_t            grid;
	size_t              smem;
	DeviceInfo          di;
	fls_status          s = device_info(di);
	if (s != FLS_OK) { return s; }
	if ((s = plan_fixed(di, col, 1, 0u, P.S, grid, smem)) != FLS_OK) { return s; }
	P.S.err = device_error_word(stream);
	P.base  = static_cast<uint32_t>(col->base);
	P.sum   = reinterpret_cast<unsigned long long*>(d_sum);
	P.out   = d_out;
	const std::string args = std::to_string(static_cast<unsigned>(col->layout)) + ", " +
	                         std::to_string(static_cast<unsigned>(col->bw)) + ", " + std::to_string(mode) + ", " +
	                         (no_wrap ? "true" : "false");
	return launch_fixed(make_key('D', P.S.warps, args), &P, grid, 32u * P.S.warps, smem, stream, used);
}

} // namespace fls

using namespace fls;

extern "C" {

fls_status fls_get_jit_stats(fls_jit_stats* out) {
	if (!out) { return set_error(FLS_ERR_INVALID_ARG, "fls_get_jit_stats: null pointer"); }
	std::lock_guard<std::mutex> lk(g_mu);
	out->compiled = g_compiled.load();
	out->launches = g_launches.load();
	out->failures = g_failures.load();
	out->cached   = g_cache.size();
	return FLS_OK;
}

const char* fls_jit_last_log(void) {
	static thread_local std::string copy;
	std::lock_guard<std::mutex>     lk(g_mu);
	copy = g_last_log;
	return copy.c_str();
}

} // extern "C"
