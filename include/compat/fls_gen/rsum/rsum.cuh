/* fls_gen/rsum/rsum.cuh under the reference's path
 * (fastlanes/src/include/fls_gen/rsum/rsum.cuh:4): d_rsum_32 of
 * fls_crystal.cuh, visible unqualified as the reference's is. */
#pragma once
#include "../../../fls_crystal.cuh"
using fls::crystal::d_rsum_32;
