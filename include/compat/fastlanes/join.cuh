/* fastlanes/join.cuh under the reference's path: the tile primitives of fls_crystal.cuh
 * (the reference's fastlanes/src/include/fastlanes/join.cuh), visible
 * unqualified as the reference's are.  Put include/compat first on the
 * include path. */
#pragma once
#include "../../fls_crystal.cuh"
using namespace fls::crystal;
