// TEST INFRASTRUCTURE ONLY: the reference's tile-based RFOR encoder
// (tile_based/src/rlebinpack.cpp:9-146, included where it lies; its main
// renamed away) behind a C entry point.  Its progress line on stdout is
// discarded.
#include <fcntl.h>
#include <unistd.h>

#define main fls_ref_rfor_main
#include "rlebinpack.cpp"
#undef main

#include "ref_api.h"

extern "C" void ref_rfor_encode(const uint32_t* in, uint32_t n, uint32_t* value, uint32_t* run_length,
                                uint32_t* val_offsets, uint32_t* rl_offsets, uint32_t* sizes2) {
	fflush(stdout);
	int saved   = dup(1);
	int devnull = open("/dev/null", O_WRONLY);
	if (saved >= 0 && devnull >= 0) { dup2(devnull, 1); }
	uint* inp = const_cast<uint*>(in); // rleBinPack advances its pointer arguments
	uint* v   = value;
	uint* r   = run_length;
	uint* vo  = val_offsets;
	uint* ro  = rl_offsets;
	std::pair<uint, uint> p = rleBinPack(inp, v, r, vo, ro, n);
	std::cout.flush();
	fflush(stdout);
	if (saved >= 0 && devnull >= 0) { dup2(saved, 1); }
	if (devnull >= 0) { close(devnull); }
	if (saved >= 0) { close(saved); }
	sizes2[0] = p.first;
	sizes2[1] = p.second;
}
