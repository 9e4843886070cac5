/* TEST INFRASTRUCTURE ONLY: stands in for CUB's test utility header, which
 * the reference's SSB query files include (fastlanes/src/ssb/fls_q21.cu:3)
 * for CubDebugExit; the toolkit's CUB provides that macro. */
#pragma once
#include <cub/util_allocator.cuh>
#include <cub/util_debug.cuh>
