// TEST INFRASTRUCTURE ONLY.  The reference's own GPU decoder of the
// tile-based RFOR format, LoadRBinPack (tile_based/src/include/
// rlebinpack_kernel.cuh:20-145, included where it lies, with CUB from the
// CUDA toolkit), run the way its benchmark runs it: one CTA of 128 threads x 4
// items per 512-value tile, the tile's items stored striped
// (tile_based_bench_rle_all_memory.cu:150-183, runRBinKernel).  The tests use
// it to pin the decoding semantics of RFOR streams on the GPU.
#include "rlebinpack_kernel.cuh"

namespace {
constexpr int kThreads = 128, kItems = 4, kTile = kThreads * kItems;

__global__ void ref_rfor_tiles(int* col, uint* val_block_start, uint* val_data, uint* rl_block_start, uint* rl_data,
                               int num_entries) {
	extern __shared__ uint shared_buffer[];
	int        val_block[kItems];
	int        rl_block[kItems];
	const int  tile_offset    = blockIdx.x * kTile;
	const bool is_last_tile   = blockIdx.x == gridDim.x - 1;
	const int  num_tile_items = is_last_tile ? num_entries - tile_offset : kTile;
	LoadRBinPack<kThreads, kItems>(val_block_start, rl_block_start, val_data, rl_data, shared_buffer, val_block, rl_block,
	                               is_last_tile, num_tile_items);
	__syncthreads();
	for (int i = 0; i < kItems; i++) {
		const int p = i * kThreads + threadIdx.x;
		if (p < num_tile_items) { col[tile_offset + p] = val_block[i]; }
	}
}
} // namespace

// Launches the decode of every tile of the streams into out (n values) on the
// legacy default stream, without waiting; device pointers.  Returns the
// launch status.
extern "C" int ref_rfor_decode_gpu_launch(const uint32_t* val, const uint32_t* val_offsets, const uint32_t* rl,
                                          const uint32_t* rl_offsets, uint32_t n, int32_t* out) {
	const unsigned tiles = (n + kTile - 1) / kTile;
	// 8 KB of shared memory: the 4 KB the benchmark gives, plus room for CUB's
	// scan and exchange storage, which LoadRBinPack places in its second half.
	ref_rfor_tiles<<<tiles, kThreads, 8192>>>(out, const_cast<uint*>(val_offsets), const_cast<uint*>(val),
	                                          const_cast<uint*>(rl_offsets), const_cast<uint*>(rl),
	                                          static_cast<int>(n));
	return static_cast<int>(cudaGetLastError());
}

// Decodes every tile of the streams into out (n values) and waits; device
// pointers.
extern "C" int ref_rfor_decode_gpu(const uint32_t* val, const uint32_t* val_offsets, const uint32_t* rl,
                                   const uint32_t* rl_offsets, uint32_t n, int32_t* out) {
	const int s = ref_rfor_decode_gpu_launch(val, val_offsets, rl, rl_offsets, n, out);
	return s != 0 ? s : static_cast<int>(cudaDeviceSynchronize());
}
