// fls_crystal_ops.cu -- the reference's query kernels written against the
// drop-in primitive API (include/fls_crystal.cuh), one 1024-value vector per
// 32-thread CTA exactly as the reference launches them.  They show that
// kernels written for the reference's primitives run unchanged on this
// library, and give parity tests a second, independent code path.
//
//   fls_crystal_q11        fastlanes/src/ssb/fls_q11.cu:29-81  QueryKernel_v1
//   fls_crystal_q21_probe  fastlanes/src/ssb/fls_q21.cu:21-78  probe_v1
#include "../../include/fls_crystal.cuh"
#include "fls_pipeline.cuh"

namespace fls {
namespace {
using namespace fls::crystal;

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
__global__ void crystal_q11_kernel(const int* enc_date, int date_bw, const int* enc_disc, int disc_bw,
                                   const int* enc_qty, int qty_bw, const int* enc_price, int price_bw, long long n_rows,
                                   int date_gt, int date_lt, int qty_lt, int disc_ge, int disc_le,
                                   unsigned long long* revenue) {
	constexpr int TILE = BLOCK_THREADS * ITEMS_PER_THREAD;
	int           items[ITEMS_PER_THREAD];
	int           items2[ITEMS_PER_THREAD];
	int           flags[ITEMS_PER_THREAD];
	const long long tile_offset = static_cast<long long>(blockIdx.x) * TILE;
	const int       num_tile    = static_cast<int>(min(static_cast<long long>(TILE), n_rows - tile_offset));

	unpack_device(enc_date + static_cast<long long>(blockIdx.x) * date_bw * 32, items, static_cast<uint8_t>(date_bw));
	BlockPredGT<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(items, date_gt, flags, num_tile);
	BlockPredAndLT<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(items, date_lt, flags, num_tile);
	unpack_device(enc_qty + static_cast<long long>(blockIdx.x) * qty_bw * 32, items, static_cast<uint8_t>(qty_bw));
	BlockPredAndLT<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(items, qty_lt, flags, num_tile);
	unpack_device(enc_disc + static_cast<long long>(blockIdx.x) * disc_bw * 32, items, static_cast<uint8_t>(disc_bw));
	BlockPredAndGTE<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(items, disc_ge, flags, num_tile);
	BlockPredAndLTE<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(items, disc_le, flags, num_tile);
	unpack_device(enc_price + static_cast<long long>(blockIdx.x) * price_bw * 32, items2,
	              static_cast<uint8_t>(price_bw));
	long long sum = 0;
#pragma unroll
	for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
		if (static_cast<int>(threadIdx.x) + BLOCK_THREADS * i < num_tile && flags[i]) {
			sum += static_cast<long long>(items[i]) * items2[i];
		}
	}
	__shared__ long long buffer[(BLOCK_THREADS + 31) / 32];
	const long long      total = BlockSum<long long, BLOCK_THREADS, ITEMS_PER_THREAD>(sum, buffer);
	if (threadIdx.x == 0) { atomicAdd(revenue, static_cast<unsigned long long>(total)); }
}

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
__global__ void crystal_q21_kernel(const int* lo_suppkey, int supp_bw, const int* lo_partkey, int part_bw,
                                   const int* lo_orderdate, int date_bw, const int* lo_revenue, int rev_bw,
                                   long long n_rows, const int* ht_s, int s_len, const int* ht_p, int p_len,
                                   const int* ht_d, int d_len, int d_keys_min, int* res) {
	constexpr int TILE = BLOCK_THREADS * ITEMS_PER_THREAD;
	int           items[ITEMS_PER_THREAD];
	int           flags[ITEMS_PER_THREAD];
	int           brand[ITEMS_PER_THREAD];
	int           year[ITEMS_PER_THREAD];
	int           revenue[ITEMS_PER_THREAD];
	const long long tile_offset = static_cast<long long>(blockIdx.x) * TILE;
	const int       num_tile    = static_cast<int>(min(static_cast<long long>(TILE), n_rows - tile_offset));
	const long long v           = blockIdx.x;

	InitFlags<BLOCK_THREADS, ITEMS_PER_THREAD>(flags);
	unpack_device(lo_suppkey + v * supp_bw * 32, items, static_cast<uint8_t>(supp_bw));
	BlockProbeAndPHT_1<int, BLOCK_THREADS, ITEMS_PER_THREAD>(items, flags, ht_s, s_len, num_tile);
	unpack_device(lo_partkey + v * part_bw * 32, items, static_cast<uint8_t>(part_bw));
	BlockProbeAndPHT_2<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(items, brand, flags, ht_p, p_len, num_tile);
	unpack_device(lo_orderdate + v * date_bw * 32, items, static_cast<uint8_t>(date_bw));
	BlockProbeAndPHT_2<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(items, year, flags, ht_d, d_len, d_keys_min,
	                                                              num_tile);
	unpack_device(lo_revenue + v * rev_bw * 32, revenue, static_cast<uint8_t>(rev_bw));
#pragma unroll
	for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
		if (static_cast<int>(threadIdx.x) + BLOCK_THREADS * i < num_tile && flags[i]) {
			const int hash = (brand[i] * 7 + (year[i] - 1992)) % ((1998 - 1992 + 1) * (5 * 5 * 40));
			if (hash >= 0) {
				res[hash * 4]     = year[i];
				res[hash * 4 + 1] = brand[i];
				atomicAdd(reinterpret_cast<unsigned long long*>(&res[hash * 4 + 2]),
				          static_cast<unsigned long long>(static_cast<long long>(revenue[i])));
			}
		}
	}
}

fls_status check_uniform_col(const int32_t* p, uint32_t bw) {
	if (!p) { return set_error(FLS_ERR_INVALID_ARG, "null column"); }
	if (bw > 32) { return set_error(FLS_ERR_BAD_BW, "bit width > 32"); }
	return FLS_OK;
}

} // namespace
} // namespace fls

using namespace fls;

extern "C" {

fls_status fls_crystal_q11(const int32_t* date, uint32_t date_bw, const int32_t* disc, uint32_t disc_bw,
                           const int32_t* qty, uint32_t qty_bw, const int32_t* price, uint32_t price_bw,
                           uint64_t n_rows, int32_t date_gt, int32_t date_lt, int32_t qty_lt, int32_t disc_ge,
                           int32_t disc_le, uint64_t* d_revenue, fls_stream_t stream) {
	fls_status s;
	if ((s = check_uniform_col(date, date_bw)) || (s = check_uniform_col(disc, disc_bw)) ||
	    (s = check_uniform_col(qty, qty_bw)) || (s = check_uniform_col(price, price_bw))) {
		return s;
	}
	if (!d_revenue || n_rows == 0) { return set_error(FLS_ERR_INVALID_ARG, "fls_crystal_q11: bad arguments"); }
	DeviceInfo di;
	if ((s = device_info(di)) != FLS_OK) { return s; }
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	if ((s = cuda_check(cudaMemsetAsync(d_revenue, 0, sizeof(uint64_t), st), "cudaMemsetAsync")) != FLS_OK) {
		return s;
	}
	const uint64_t n_vec = (n_rows + 1023u) / 1024u;
	crystal_q11_kernel<32, 32><<<static_cast<unsigned>(n_vec), 32, 0, st>>>(
	    date, static_cast<int>(date_bw), disc, static_cast<int>(disc_bw), qty, static_cast<int>(qty_bw), price,
	    static_cast<int>(price_bw), static_cast<long long>(n_rows), date_gt, date_lt, qty_lt, disc_ge, disc_le,
	    reinterpret_cast<unsigned long long*>(d_revenue));
	count_launch();
	return cuda_check(cudaGetLastError(), "crystal_q11_kernel launch");
}

fls_status fls_crystal_q21_probe(const int32_t* suppkey, uint32_t supp_bw, const int32_t* partkey, uint32_t part_bw,
                                 const int32_t* orderdate, uint32_t date_bw, const int32_t* revenue, uint32_t rev_bw,
                                 uint64_t n_rows, const int32_t* ht_s, int32_t s_len, const int32_t* ht_p,
                                 int32_t p_len, const int32_t* ht_d, int32_t d_len, int32_t d_keys_min, int32_t* d_res,
                                 fls_stream_t stream) {
	fls_status s;
	if ((s = check_uniform_col(suppkey, supp_bw)) || (s = check_uniform_col(partkey, part_bw)) ||
	    (s = check_uniform_col(orderdate, date_bw)) || (s = check_uniform_col(revenue, rev_bw))) {
		return s;
	}
	if (!ht_s || !ht_p || !ht_d || !d_res || s_len <= 0 || p_len <= 0 || d_len <= 0 || n_rows == 0) {
		return set_error(FLS_ERR_INVALID_ARG, "fls_crystal_q21_probe: bad arguments");
	}
	DeviceInfo di;
	if ((s = device_info(di)) != FLS_OK) { return s; }
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	if ((s = cuda_check(cudaMemsetAsync(d_res, 0, sizeof(int32_t) * 4u * 7000u, st), "cudaMemsetAsync")) != FLS_OK) {
		return s;
	}
	const uint64_t n_vec = (n_rows + 1023u) / 1024u;
	crystal_q21_kernel<32, 32><<<static_cast<unsigned>(n_vec), 32, 0, st>>>(
	    suppkey, static_cast<int>(supp_bw), partkey, static_cast<int>(part_bw), orderdate, static_cast<int>(date_bw),
	    revenue, static_cast<int>(rev_bw), static_cast<long long>(n_rows), ht_s, s_len, ht_p, p_len, ht_d, d_len,
	    d_keys_min, d_res);
	count_launch();
	return cuda_check(cudaGetLastError(), "crystal_q21_kernel launch");
}

} // extern "C"
