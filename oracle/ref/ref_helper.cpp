// TEST INFRASTRUCTURE ONLY: exposes the reference's golden unpack-test arrays
// (rand_arr_{bw}_b{bw}_w32_arr, one per bit width 0..32).
#include <cstdint>
#include "cuda_normal_t32_1024_uf1_unpack_helper.hpp"
#include "ref_api.h"

#define FLS_REF_ARR(BW) case BW: return helper::rand_arr_##BW##_b##BW##_w32_arr;
extern "C" const uint32_t* ref_helper_arr(unsigned bw) {
	switch (bw) {
		FLS_REF_ARR(0) FLS_REF_ARR(1) FLS_REF_ARR(2) FLS_REF_ARR(3) FLS_REF_ARR(4) FLS_REF_ARR(5)
		FLS_REF_ARR(6) FLS_REF_ARR(7) FLS_REF_ARR(8) FLS_REF_ARR(9) FLS_REF_ARR(10) FLS_REF_ARR(11)
		FLS_REF_ARR(12) FLS_REF_ARR(13) FLS_REF_ARR(14) FLS_REF_ARR(15) FLS_REF_ARR(16) FLS_REF_ARR(17)
		FLS_REF_ARR(18) FLS_REF_ARR(19) FLS_REF_ARR(20) FLS_REF_ARR(21) FLS_REF_ARR(22) FLS_REF_ARR(23)
		FLS_REF_ARR(24) FLS_REF_ARR(25) FLS_REF_ARR(26) FLS_REF_ARR(27) FLS_REF_ARR(28) FLS_REF_ARR(29)
		FLS_REF_ARR(30) FLS_REF_ARR(31) FLS_REF_ARR(32)
	default: return nullptr;
	}
}
