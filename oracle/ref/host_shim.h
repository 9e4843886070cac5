/*
 * host_shim.h -- TEST INFRASTRUCTURE ONLY (oracle build of the reference).
 *
 * Lets the reference's warp-level CUDA decoder headers compile as plain host
 * C++ so that the reference's own arithmetic can be run on the CPU and used to
 * pin the oracle and to time the reference CPU arm:
 *   fastlanes/src/include/fls_gen/unpack/unpack.cuh        (normal unpack)
 *   fastlanes/src/include/fls_gen/unpack/unpack_fused.cuh  (register unpack)
 *   fastlanes/src/include/fls_gen/unpack/hardcoded_16.cuh  (8-at-a-time etc.)
 *   fastlanes/src/include/fls_gen/rsum/rsum.cuh            (transposed delta)
 *
 * A "warp" is emulated by looping lanes 0..31 and setting the thread index
 * between calls.  Device qualifiers become host ones; the only inline PTX in
 * those headers is a trap on unsupported bit widths, which the wrappers never
 * reach because they validate the bit width first.
 */
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>

struct fls_shim_idx3 {
	unsigned x, y, z;
};
extern thread_local fls_shim_idx3 fls_shim_thread_idx;
extern thread_local fls_shim_idx3 fls_shim_block_idx;

#define threadIdx       fls_shim_thread_idx
#define blockIdx        fls_shim_block_idx
#define __device__
#define __host__
#define __global__      static inline
#define __forceinline__ inline
#define __shared__      static
#define asm(x)          abort()
