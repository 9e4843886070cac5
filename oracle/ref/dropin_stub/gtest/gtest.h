/* TEST INFRASTRUCTURE ONLY: the two gtest assertions the reference's SSB
 * query files use in their host code (fastlanes/src/ssb/fls_q21.cu:349-350,
 * compress_ssb.cu:346-347), so those files compile without gtest (the
 * drop-in test calls only their kernels). */
#pragma once
#include <cstdio>
#define ASSERT_EQ(a, b)                                                                                                \
	do {                                                                                                               \
		if (!((a) == (b))) {                                                                                           \
			std::fprintf(stderr, "ASSERT_EQ failed: %s == %s\n", #a, #b);                                           \
			return;                                                                                                    \
		}                                                                                                              \
	} while (0)
#define EXPECT_EQ(a, b)                                                                                                \
	do {                                                                                                               \
		if (!((a) == (b))) { std::fprintf(stderr, "EXPECT_EQ failed: %s == %s\n", #a, #b); }                         \
	} while (0)
