// fls_runtime.cu -- host runtime of the library: device properties, the device
// error word, launch configuration, shared-memory planning of the staged
// pipeline, and the C ABI entry points that are not operators.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "fls_pipeline.cuh"

namespace fls {

// The default error word of each device (a module-scope variable exists once
// per device context), for streams without a word of their own: [0] holds the
// bits kernels OR in, [1] receives the bits fls_check_device_error takes out of
// [0] with one atomic exchange.  Kernels receive the address as a parameter.
__device__ uint32_t g_err_word[2] = {0u, 0u};

namespace {
std::atomic<uint64_t> g_launches {0};

struct LaunchCfg {
	uint32_t warps = 16, stages = 2, ctas_per_sm = 1, tile_bytes = 6144;
};
std::mutex g_cfg_mu;
LaunchCfg  g_cfg;
bool       g_warps_set = false; // warps chosen by the caller (fls_set_launch_config)

LaunchCfg launch_cfg() {
	std::lock_guard<std::mutex> lk(g_cfg_mu);
	return g_cfg;
}

uint32_t round4(uint32_t w) { return (w + 3u) & ~3u; }

std::mutex              g_dev_mu;
std::vector<DeviceInfo> g_dev_cache;
std::vector<uint32_t*>  g_err_addr;

// Error words bound to streams by fls_bind_error_word: (device, stream) ->
// caller-owned pair of device words.  A short list: callers bind one word per
// stream they use.
struct ErrBinding {
	int          dev;
	cudaStream_t stream;
	uint32_t*    words;
};
constexpr size_t        kMaxBindings = 4096;
std::mutex              g_bind_mu;
std::vector<ErrBinding> g_bind;

// Moves the error bits of words[0] into words[1] with one atomic exchange, in
// stream order, so no bit raised after the read is lost.
__global__ void err_take_kernel(uint32_t* words) { words[1] = atomicExch(&words[0], 0u); }
} // namespace

void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

uint32_t jit_max_warps() {
	std::lock_guard<std::mutex> lk(g_cfg_mu);
	return g_warps_set ? g_cfg.warps : kJitDefaultWarps;
}

namespace {
constexpr int    kDefaultSparseRows = 4;
std::atomic<int> g_sparse_rows {kDefaultSparseRows};
std::atomic<int> g_jit {1};
std::atomic<int> g_group_smem {1};
std::atomic<int> g_late_measure {1};
std::atomic<int> g_half_vectors {0};
std::atomic<int> g_table_kb {kJitTableKB};
} // namespace

int tuning_sparse_rows() { return g_sparse_rows.load(std::memory_order_relaxed); }
int tuning_jit() { return g_jit.load(std::memory_order_relaxed); }
int tuning_group_smem() { return g_group_smem.load(std::memory_order_relaxed); }
int tuning_late_measure() { return g_late_measure.load(std::memory_order_relaxed); }
int tuning_half_vectors() { return g_half_vectors.load(std::memory_order_relaxed); }
uint32_t tuning_table_words() { return static_cast<uint32_t>(g_table_kb.load(std::memory_order_relaxed)) * 256u; }

fls_status cuda_check(cudaError_t e, const char* what) {
	if (e == cudaSuccess) { return FLS_OK; }
	return set_error(FLS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

fls_status device_info(DeviceInfo& di) {
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) {
		cudaGetLastError();
		return set_error(FLS_ERR_NO_DEVICE, "no CUDA device");
	}
	std::lock_guard<std::mutex> lk(g_dev_mu);
	if (static_cast<int>(g_dev_cache.size()) <= dev) {
		g_dev_cache.resize(dev + 1);
		g_err_addr.resize(dev + 1, nullptr);
	}
	if (g_dev_cache[dev].sms == 0) {
		cudaDeviceProp p;
		if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) {
			return set_error(FLS_ERR_NO_DEVICE, "cudaGetDeviceProperties failed");
		}
		void* addr = nullptr;
		if (cudaGetSymbolAddress(&addr, g_err_word) != cudaSuccess) {
			return set_error(FLS_ERR_CUDA, "cannot resolve the device error word");
		}
		g_err_addr[dev]           = static_cast<uint32_t*>(addr);
		g_dev_cache[dev].sms      = p.multiProcessorCount;
		g_dev_cache[dev].max_smem = static_cast<int>(p.sharedMemPerBlockOptin);
		g_dev_cache[dev].major    = p.major;
	}
	di = g_dev_cache[dev];
	if (di.major < 10) { return set_error(FLS_ERR_NO_DEVICE, "device is not sm_100 class"); }
	return FLS_OK;
}

uint32_t* device_error_word(cudaStream_t stream) {
	int dev = 0;
	cudaGetDevice(&dev);
	{
		std::lock_guard<std::mutex> lk(g_bind_mu);
		for (const ErrBinding& b : g_bind) {
			if (b.dev == dev && b.stream == stream) { return b.words; }
		}
	}
	std::lock_guard<std::mutex> lk(g_dev_mu);
	return dev < static_cast<int>(g_err_addr.size()) ? g_err_addr[dev] : nullptr;
}

// Validates one column descriptor and converts it for the kernel.
fls_status make_devcol(const fls_column& c, DevCol& d) {
	if (!c.data && c.n_words) { return set_error(FLS_ERR_INVALID_ARG, "column data is null"); }
	if (reinterpret_cast<uintptr_t>(c.data) & 15u) {
		return set_error(FLS_ERR_ALIGNMENT, "column data must be 16-byte aligned");
	}
	if (reinterpret_cast<uintptr_t>(c.meta) & 15u) {
		return set_error(FLS_ERR_ALIGNMENT, "column metadata must be 16-byte aligned");
	}
	if (c.layout > FLS_LAYOUT_TRANSPOSED) { return set_error(FLS_ERR_INVALID_ARG, "bad column layout"); }
	if (fls_status s = check_n_values(c.n_values, "column"); s != FLS_OK) { return s; }
	d.data    = c.data;
	d.meta    = c.meta;
	d.n_words = c.n_words;
	d.layout    = c.layout;
	d.vec_words = 0;
	if (c.meta == nullptr) {
		if (c.scheme != FLS_SCHEME_FOR && c.scheme != FLS_SCHEME_DELTA) {
			return set_error(FLS_ERR_INVALID_ARG, "uniform columns must be FOR or DELTA");
		}
		if (c.bw > 32) { return set_error(FLS_ERR_BAD_BW, "bit width > 32"); }
		if (c.scheme == FLS_SCHEME_DELTA && c.layout != FLS_LAYOUT_TRANSPOSED) {
			return set_error(FLS_ERR_INVALID_ARG, "DELTA columns are stored transposed");
		}
		d.scheme             = c.scheme;
		d.bw                 = c.bw;
		d.base               = c.base;
		d.slot_words         = dev::payload_words(c.scheme, c.bw, 0);
		d.vec_words          = d.slot_words;
		const uint64_t n_vec = (c.n_values + 1023u) / 1024u;
		if (d.slot_words != 0 && n_vec > c.n_words / d.slot_words) {
			return set_error(FLS_ERR_CAPACITY, "column data smaller than n_values at this bit width");
		}
	} else {
		if (c.max_vec_words > kMaxVecWords) { return set_error(FLS_ERR_INVALID_ARG, "max_vec_words too large"); }
		if ((c.scheme_mask & ((1u << FLS_SCHEME_DELTA) | (1u << FLS_SCHEME_RLE))) && c.layout != FLS_LAYOUT_TRANSPOSED) {
			return set_error(FLS_ERR_INVALID_ARG, "DELTA/RLE vectors need the transposed layout");
		}
		d.scheme     = 0;
		d.bw         = 0;
		d.base       = 0;
		d.slot_words = round4(c.max_vec_words);
	}
	return FLS_OK;
}

namespace {
bool needs_dict(const fls_column& c) {
	return c.meta != nullptr && (c.scheme_mask & ((1u << FLS_SCHEME_RLE) | (1u << FLS_SCHEME_DICT)));
}
} // namespace

fls_status plan_stages(const fls_column* cols, uint32_t n_cols, uint32_t extra_words, uint32_t cta_words,
                       StageCfg& cfg, uint32_t& grid, uint32_t& threads, size_t& smem_bytes) {
	if (!cols || n_cols == 0 || n_cols > kMaxCols) { return set_error(FLS_ERR_INVALID_ARG, "1..8 columns per query"); }
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	std::memset(&cfg, 0, sizeof(cfg));
	bool     dict     = false;
	bool     uniform  = true;
	uint32_t vec_words[kMaxCols];
	uint32_t sum_vec  = 0;
	cfg.n_values      = cols[0].n_values;
	cfg.layout        = cols[0].layout;
	for (uint32_t c = 0; c < n_cols; ++c) {
		if ((s = make_devcol(cols[c], cfg.cols[c])) != FLS_OK) { return s; }
		if (cols[c].n_values != cfg.n_values) { return set_error(FLS_ERR_INVALID_ARG, "columns differ in length"); }
		if (cols[c].layout != cfg.layout) {
			return set_error(FLS_ERR_UNSUPPORTED, "all columns of a query must share one layout");
		}
		vec_words[c] = cfg.cols[c].slot_words; // one vector's slot
		sum_vec += vec_words[c];
		dict    = dict || needs_dict(cols[c]);
		uniform = uniform && cols[c].meta == nullptr;
	}
	cfg.n_cols      = n_cols;
	cfg.all_uniform = uniform ? 1u : 0u;
	cfg.has_dict = dict ? 1u : 0u;
	cfg.n_vec    = (cfg.n_values + 1023u) / 1024u;
	cfg.err      = device_error_word(nullptr); // launch_staged sets the launching stream's word
	LaunchCfg lc = launch_cfg();
	uint32_t  W = lc.warps, S = lc.stages;
	// Tile: enough consecutive vectors for ~tile_bytes per stage, but keep at
	// least 4 tiles per warp of the grid for load balance.
	const uint64_t total_warps = static_cast<uint64_t>(di.sms) * lc.ctas_per_sm * W;
	uint32_t       k           = sum_vec ? std::max<uint32_t>(1u, lc.tile_bytes / (4u * sum_vec)) : kMaxTile;
	k                          = std::min<uint32_t>(k, kMaxTile / n_cols); // one lane per (vector, column) at issue
	while (k > 1 && (cfg.n_vec + k - 1) / k < 4 * total_warps) { k /= 2; }
	// Shrink the pipeline until it fits the shared-memory budget.
	for (;;) {
		cfg.stage_words = 0;
		for (uint32_t c = 0; c < n_cols; ++c) {
			cfg.cols[c].slot_words = k * vec_words[c];
			cfg.col_off[c]         = cfg.stage_words;
			cfg.stage_words += cfg.cols[c].slot_words;
		}
		uint32_t w   = S * cfg.stage_words + kSlotSlackWords;
		cfg.dict_off = w;
		w += dict ? kDictWords : 0u;
		cfg.extra_off = w;
		w += round4(extra_words);
		cfg.info_off = w;
		w += 4u * S * k * n_cols;
		cfg.bar_off = w;
		w += 2u * S;
		w                   = round4(w);
		cfg.warp_smem_words = w;
		smem_bytes          = 4ull * (static_cast<size_t>(w) * W + cta_words);
		if (smem_bytes <= static_cast<size_t>(di.max_smem)) { break; }
		if (k > 1) {
			k /= 2;
		} else if (S > 2) {
			--S;
		} else if (W > 1) {
			W /= 2;
		} else {
			return set_error(FLS_ERR_CAPACITY, "vectors too large for shared-memory staging");
		}
	}
	cfg.tile                 = k;
	cfg.n_tiles              = (cfg.n_vec + k - 1) / k;
	cfg.stages               = S;
	cfg.warps                = W;
	cfg.cta_extra_off        = cfg.warp_smem_words * W;
	const uint64_t need_ctas = (cfg.n_tiles + W - 1) / W;
	grid    = static_cast<uint32_t>(std::min<uint64_t>(need_ctas, static_cast<uint64_t>(di.sms) * lc.ctas_per_sm));
	threads = 32u * W;
	return FLS_OK;
}

namespace {
// Self-test of the bounded waits every pipeline uses: one warp waits on an
// mbarrier that nothing arrives on, with the pipelines' own bounded wait, so
// it gives up after `polls` tries, raises the timeout bit and returns; the
// host then reads FLS_ERR_TIMEOUT from fls_check_device_error and the context
// stays usable.  No fault, trap or unbounded wait is involved.
__global__ void wait_selftest_kernel(uint32_t polls, uint32_t* err) {
	__shared__ uint64_t bar;
	if (threadIdx.x == 0) {
		dev::mbar_init(&bar, 1);
		dev::fence_mbar_init();
	}
	__syncwarp();
	const bool done = dev::mbar_wait_bounded(&bar, 0, polls);
	if (!done && threadIdx.x == 0) { atomicOr(err, kErrTimeout); }
}

} // namespace

} // namespace fls

using namespace fls;

extern "C" {

fls_status fls_bind_error_word(fls_stream_t stream, uint32_t* d_words) {
	if (reinterpret_cast<uintptr_t>(d_words) & 7u) {
		return set_error(FLS_ERR_ALIGNMENT, "fls_bind_error_word: the word pair must be 8-byte aligned");
	}
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	int dev = 0;
	cudaGetDevice(&dev);
	const cudaStream_t          st = reinterpret_cast<cudaStream_t>(stream);
	std::lock_guard<std::mutex> lk(g_bind_mu);
	for (size_t i = 0; i < g_bind.size(); ++i) {
		if (g_bind[i].dev == dev && g_bind[i].stream == st) {
			if (d_words) {
				g_bind[i].words = d_words;
			} else {
				g_bind.erase(g_bind.begin() + static_cast<std::ptrdiff_t>(i));
			}
			return FLS_OK;
		}
	}
	if (!d_words) { return FLS_OK; }
	if (g_bind.size() >= kMaxBindings) {
		return set_error(FLS_ERR_CAPACITY, "fls_bind_error_word: too many bound streams (unbind with NULL)");
	}
	g_bind.push_back(ErrBinding {dev, st, d_words});
	return FLS_OK;
}

fls_status fls_check_device_error(fls_stream_t stream) {
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	cudaStream_t st    = reinterpret_cast<cudaStream_t>(stream);
	uint32_t*    words = device_error_word(st);
	if (!words) { return set_error(FLS_ERR_CUDA, "no error word for this device"); }
	err_take_kernel<<<1, 1, 0, st>>>(words);
	count_launch();
	if ((s = cuda_check(cudaGetLastError(), "err_take_kernel launch")) != FLS_OK) { return s; }
	uint32_t word = 0;
	if ((s = cuda_check(cudaMemcpyAsync(&word, words + 1, sizeof(word), cudaMemcpyDeviceToHost, st),
	                    "read error word")) != FLS_OK) {
		return s;
	}
	if ((s = cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize")) != FLS_OK) { return s; }
	if (word == 0) { return FLS_OK; }
	std::string msg = "device error:";
	if (word & kErrBadMeta) { msg += " bad-vector-metadata"; }
	if (word & kErrBounds) { msg += " vector-out-of-bounds"; }
	if (word & kErrHash) { msg += " hash-out-of-table"; }
	if (word & kErrCapacity) { msg += " vector-exceeds-slot"; }
	if (word & kErrTimeout) {
		msg += " wait-timeout";
		return set_error(FLS_ERR_TIMEOUT, msg);
	}
	return set_error(FLS_ERR_DEVICE, msg);
}

fls_status fls_selftest_bounded_wait(uint32_t polls, fls_stream_t stream) {
	if (polls == 0 || polls > 1024) { return set_error(FLS_ERR_INVALID_ARG, "fls_selftest_bounded_wait: polls in 1..1024"); }
	DeviceInfo di;
	fls_status s = device_info(di);
	if (s != FLS_OK) { return s; }
	wait_selftest_kernel<<<1, 32, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
	    polls, device_error_word(reinterpret_cast<cudaStream_t>(stream)));
	count_launch();
	return cuda_check(cudaGetLastError(), "wait_selftest_kernel launch");
}

fls_status fls_set_launch_config(uint32_t warps_per_cta, uint32_t stages, uint32_t ctas_per_sm, uint32_t tile_bytes) {
	if (warps_per_cta > kMaxWarps || stages > 8 || ctas_per_sm > 4 || tile_bytes > 65536) {
		return set_error(FLS_ERR_INVALID_ARG,
		                 "launch config out of range (warps <= 16, stages <= 8, ctas <= 4, tile_bytes <= 64K)");
	}
	const LaunchCfg d;
	std::lock_guard<std::mutex> lk(g_cfg_mu);
	g_cfg.warps       = warps_per_cta ? warps_per_cta : d.warps;
	g_warps_set       = warps_per_cta != 0;
	g_cfg.stages      = stages ? stages : d.stages;
	g_cfg.ctas_per_sm = ctas_per_sm ? ctas_per_sm : d.ctas_per_sm;
	g_cfg.tile_bytes  = tile_bytes ? tile_bytes : d.tile_bytes;
	return FLS_OK;
}

fls_status fls_get_launch_config(uint32_t* warps_per_cta, uint32_t* stages, uint32_t* ctas_per_sm,
                                 uint32_t* tile_bytes) {
	LaunchCfg c = launch_cfg();
	if (warps_per_cta) { *warps_per_cta = c.warps; }
	if (stages) { *stages = c.stages; }
	if (ctas_per_sm) { *ctas_per_sm = c.ctas_per_sm; }
	if (tile_bytes) { *tile_bytes = c.tile_bytes; }
	return FLS_OK;
}

uint64_t fls_kernel_launch_count(void) { return g_launches.load(); }

fls_status fls_set_tuning(uint32_t param, int64_t value) {
	switch (param) {
	case FLS_TUNE_SPARSE_ROWS:
		if (value < 0 || value > 32) { return set_error(FLS_ERR_INVALID_ARG, "sparse rows must be in [0, 32]"); }
		g_sparse_rows.store(value ? static_cast<int>(value) : kDefaultSparseRows);
		return FLS_OK;
	case FLS_TUNE_JIT:
		if (value < 0 || value > 1) { return set_error(FLS_ERR_INVALID_ARG, "jit must be 0 or 1"); }
		g_jit.store(static_cast<int>(value));
		return FLS_OK;
	case FLS_TUNE_GROUP_SMEM:
		if (value < 0 || value > 1) { return set_error(FLS_ERR_INVALID_ARG, "group smem must be 0 or 1"); }
		g_group_smem.store(static_cast<int>(value));
		return FLS_OK;
	case FLS_TUNE_LATE_MEASURE:
		if (value < 0 || value > 1) { return set_error(FLS_ERR_INVALID_ARG, "late measure must be 0 or 1"); }
		g_late_measure.store(static_cast<int>(value));
		return FLS_OK;
	case FLS_TUNE_TABLE_KB:
		if (value < 0 || value > static_cast<int64_t>(kJitMaxTableKB)) {
			return set_error(FLS_ERR_INVALID_ARG, "table budget must be in [0, 144] KB");
		}
		g_table_kb.store(value ? static_cast<int>(value) : static_cast<int>(kJitTableKB));
		return FLS_OK;
	case FLS_TUNE_HALF_VECTORS:
		if (value != 0 && value != 1) { return set_error(FLS_ERR_INVALID_ARG, "half vectors must be 0 or 1"); }
		g_half_vectors.store(static_cast<int>(value));
		return FLS_OK;
	default: return set_error(FLS_ERR_INVALID_ARG, "unknown tuning parameter");
	}
}

fls_status fls_get_tuning(uint32_t param, int64_t* value) {
	if (!value) { return set_error(FLS_ERR_INVALID_ARG, "fls_get_tuning: null pointer"); }
	switch (param) {
	case FLS_TUNE_SPARSE_ROWS: *value = tuning_sparse_rows(); return FLS_OK;
	case FLS_TUNE_JIT: *value = tuning_jit(); return FLS_OK;
	case FLS_TUNE_GROUP_SMEM: *value = tuning_group_smem(); return FLS_OK;
	case FLS_TUNE_LATE_MEASURE: *value = tuning_late_measure(); return FLS_OK;
	case FLS_TUNE_TABLE_KB: *value = g_table_kb.load(); return FLS_OK;
	case FLS_TUNE_HALF_VECTORS: *value = tuning_half_vectors(); return FLS_OK;
	default: return set_error(FLS_ERR_INVALID_ARG, "unknown tuning parameter");
	}
}

} // extern "C"
