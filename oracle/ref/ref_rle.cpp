// TEST INFRASTRUCTURE ONLY: the reference's FastLanes RLE encoder (rle.hpp).
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <fcntl.h>
#include <unistd.h>
#include "fls_gen/rle/rle.hpp"
#include "ref_api.h"

extern "C" int ref_vector_rle(const int32_t* vec, uint8_t* idx, int32_t* dict, uint16_t* dict4) {
	// VECTOR_RLE prints 2x1024 debug entries to stdout (rle.hpp:37-38); discard them.
	fflush(stdout);
	int saved = dup(1);
	int devnull = open("/dev/null", O_WRONLY);
	if (saved >= 0 && devnull >= 0) { dup2(devnull, 1); }
	uint16_t last = fastlanes::VECTOR_RLE(vec, idx, dict, dict4);
	fflush(stdout);
	if (saved >= 0 && devnull >= 0) { dup2(saved, 1); }
	if (devnull >= 0) { close(devnull); }
	if (saved >= 0) { close(saved); }
	return static_cast<int>(dict4[3]) + static_cast<int>(last);
}
