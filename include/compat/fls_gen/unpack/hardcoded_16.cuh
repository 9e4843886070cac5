/* fls_gen/unpack/hardcoded_16.cuh under the reference's path: the
 * namespaces unpack_8_at_a_time, hardcoded and hardcoded_16 of fls_crystal.cuh
 * (the reference's fastlanes/src/include/fls_gen/unpack/hardcoded_16.cuh:16-1206),
 * visible unqualified as the reference's are. */
#pragma once
#include "../../../fls_crystal.cuh"
using namespace fls::crystal;
