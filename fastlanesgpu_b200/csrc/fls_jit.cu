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

#include <atomic>
#include <cstdio>
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

std::string shape_source(const std::string& args) {
	return "#include \"fls_fixed.cuh\"\n"
	       "extern \"C\" __global__ void __launch_bounds__(512, 1)\n"
	       "fls_fixed_kernel(const __grid_constant__ fls::fixed::FixedParams P) {\n"
	       "\tfls::fixed::run<fls::fixed::Query<" +
	       args + ">>(P);\n}\n";
}

// NVRTC compile of one shape into e.cubin; false (log kept) on failure.
bool compile_shape(const std::string& args, Entry& e) {
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
	const std::string src = shape_source(args);
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
		g_last_log = "Query<" + args + ">: " + log;
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
	for (uint32_t i = 0; i < sh.n_staged; ++i) {
		const fls_column& c = cols[sh.staged[i]];
		if (c.meta != nullptr || c.scheme != FLS_SCHEME_FOR || c.bw > 32 || c.layout != cols[sh.staged[0]].layout) {
			return false;
		}
	}
	char key[160];
	int  len = std::snprintf(key, sizeof(key), "%u, %u, %d, %d", static_cast<unsigned>(cols[sh.staged[0]].layout),
	                         n_filters, sh.agg_a, sh.agg_b);
	for (uint32_t i = 0; i < sh.n_staged; ++i) {
		len += std::snprintf(key + len, sizeof(key) - len, ", %u", static_cast<unsigned>(cols[sh.staged[i]].bw));
	}
	sh.key = key;
	return true;
}

bool jit_compile(const JitShape& sh) {
	std::lock_guard<std::mutex> lk(g_mu);
	return compiled_entry(sh.key).state > 0;
}

fls_status jit_filter_agg(const fls_column* cols, const fls_filter* filters, uint32_t n_filters, int32_t agg_a,
                          int32_t agg_b, int64_t* d_result, int32_t sparse_rows, cudaStream_t stream, bool& used) {
	used = false;
	JitShape sh;
	if (!jit_shape(cols, filters, n_filters, agg_a, agg_b, sh)) { return FLS_OK; }
	fls_column sc[FLS_MAX_QUERY_COLS];
	for (uint32_t i = 0; i < sh.n_staged; ++i) { sc[i] = cols[sh.staged[i]]; }
	StageCfg   cfg;
	uint32_t   grid, threads;
	size_t     smem;
	fls_status s = plan_stages(sc, sh.n_staged, 0u, 0u, cfg, grid, threads, smem);
	if (s != FLS_OK) { return s; }
	int dev = 0;
	if ((s = cuda_check(cudaGetDevice(&dev), "cudaGetDevice")) != FLS_OK) { return s; }

	fixed::FixedParams P {};
	for (uint32_t i = 0; i < sh.n_staged; ++i) {
		P.data[i] = sc[i].data;
		P.base[i] = static_cast<uint32_t>(sc[i].base);
	}
	for (uint32_t f = 0; f < n_filters; ++f) {
		P.lo[f]    = static_cast<uint32_t>(filters[f].lo);
		P.range[f] = static_cast<uint32_t>(filters[f].hi) - static_cast<uint32_t>(filters[f].lo);
	}
	P.n_values        = cfg.n_values;
	P.n_vec           = cfg.n_vec;
	P.n_tiles         = cfg.n_tiles;
	P.tile            = cfg.tile;
	P.stages          = cfg.stages;
	P.warps           = cfg.warps;
	P.stage_words     = cfg.stage_words;
	P.bar_off         = cfg.stages * cfg.stage_words + fixed::kSlack;
	P.warp_smem_words = (P.bar_off + 2u * cfg.stages + 3u) & ~3u;
	P.sparse_rows     = sparse_rows;
	P.result          = reinterpret_cast<unsigned long long*>(d_result);
	P.err             = cfg.err;
	const size_t fsmem = 4ull * P.warp_smem_words * cfg.warps;

	cudaKernel_t kernel {};
	{
		std::lock_guard<std::mutex> lk(g_mu);
		Entry&                      e = compiled_entry(sh.key);
		if (e.state == 1) {
			e.state = load_shape(e) ? 2 : -1;
			if (e.state < 0) { g_failures.fetch_add(1); }
		}
		if (e.state != 2) { return FLS_OK; }
		if (e.smem_set.size() <= static_cast<size_t>(dev)) { e.smem_set.resize(dev + 1, 0); }
		if (fsmem > 48u * 1024u && e.smem_set[dev] < fsmem) {
			s = cuda_check(cudaKernelSetAttributeForDevice(e.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			                                               static_cast<int>(fsmem), dev),
			               "cudaKernelSetAttributeForDevice");
			if (s != FLS_OK) { return s; }
			e.smem_set[dev] = fsmem;
		}
		kernel = e.kernel;
	}
	void* argv[] = {&P};
	s = cuda_check(cudaLaunchKernel(reinterpret_cast<const void*>(kernel), dim3(grid), dim3(threads), argv, fsmem,
	                                stream),
	               "cudaLaunchKernel (specialised filter-aggregate)");
	if (s != FLS_OK) { return s; }
	count_launch();
	g_launches.fetch_add(1);
	used = true;
	return FLS_OK;
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
