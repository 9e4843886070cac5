"""The C ABI from plain C: a C11 program compiled against include/fls_gpu.h
and linked with libfls_gpu.so (as a reference user's host code would be)
packs and unpacks vectors of every lane width, encodes a column, writes and
reopens an encoded-column container, sizes a vector exhaustively and reads
an error message -- all host calls, no GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "fls_gpu.h"

#define CHECK(x) do { fls_status s_ = (x); if (s_ != FLS_OK) { \
    printf("FAIL %s: %d %s\n", #x, (int)s_, fls_last_error()); return 1; } } while (0)

int main(void) {
    /* 8-bit lanes: reference pack.cpp:29521 layout, round trip */
    uint8_t v8[1024], p8[1024], u8[1024];
    for (int i = 0; i < 1024; ++i) v8[i] = (uint8_t)((i * 37) & 31);
    CHECK(fls_pack_u8(v8, p8, 5));
    CHECK(fls_unpack_u8(p8, u8, 5));
    if (memcmp(v8, u8, sizeof(v8)) != 0) { printf("FAIL u8 round trip\n"); return 1; }
    /* 64-bit lanes */
    static uint64_t v64[1024], p64[1024], u64[1024];
    for (int i = 0; i < 1024; ++i) v64[i] = ((uint64_t)i * 0x9E3779B97F4A7C15ull) >> 23; /* 41 bits */
    CHECK(fls_pack_u64(v64, p64, 41));
    CHECK(fls_unpack_u64(p64, u64, 41));
    if (memcmp(v64, u64, sizeof(v64)) != 0) { printf("FAIL u64 round trip\n"); return 1; }
    /* a uniform 32-bit column and its container */
    enum { N = 5000 };
    static int32_t vals[N];
    for (int i = 0; i < N; ++i) vals[i] = 100000 + (i * 7919) % 4096;
    uint64_t bound = fls_encode_bound_words(N), words = 0;
    uint32_t* enc = (uint32_t*)calloc(bound, 4);
    uint8_t bw = 0;
    CHECK(fls_encode_uniform(vals, N, FLS_SCHEME_FOR, FLS_LAYOUT_NORMAL, 0xff, 100000, enc, &words, &bw));
    if (bw != 12) { printf("FAIL bw %u\n", bw); return 1; }
    fls_column col;
    memset(&col, 0, sizeof(col));
    col.data = enc; col.meta = NULL; col.n_values = N; col.n_words = words; col.layout = FLS_LAYOUT_NORMAL;
    col.scheme = FLS_SCHEME_FOR; col.bw = bw; col.base = 100000; col.max_vec_words = 32u * bw;
    col.scheme_mask = 1u << FLS_SCHEME_FOR;
    uint64_t bytes = fls_column_container_bytes(&col), written = 0;
    void* buf = NULL;
    if (posix_memalign(&buf, 16, bytes) != 0) return 1;
    CHECK(fls_column_write_container(&col, buf, bytes, &written));
    fls_column back;
    CHECK(fls_column_open_container(buf, written, &back));
    if (back.n_values != N || back.bw != bw || back.base != 100000 || back.n_words != words ||
        memcmp(back.data, enc, 4 * words) != 0) { printf("FAIL container\n"); return 1; }
    ((uint8_t*)buf)[3] ^= 1;
    if (fls_column_open_container(buf, written, &back) != FLS_ERR_INVALID_ARG) { printf("FAIL damage\n"); return 1; }
    printf("refused: %s\n", fls_last_error());
    /* exhaustive sizing of one vector */
    uint32_t sizes[5];
    uint8_t best;
    CHECK(fls_encode_exhaustive(vals, 1024, sizes, &best, 1));
    if (best > 4 || sizes[FLS_SCHEME_FOR] != 16u + 4u * 32u * 12u) { printf("FAIL exhaustive %u\n", sizes[0]); return 1; }
    /* errors are status codes with messages */
    if (fls_pack_u8(v8, p8, 9) != FLS_ERR_BAD_BW || strlen(fls_last_error()) == 0) { printf("FAIL error\n"); return 1; }
    printf("OK\n");
    free(buf);
    free(enc);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_c_program_against_the_abi(tmp_path):
    lib_dir = os.path.join(ROOT, "fastlanesgpu_b200")
    assert os.path.exists(os.path.join(lib_dir, "libfls_gpu.so"))
    src = tmp_path / "user.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "user"
    subprocess.run(["gcc", "-std=c11", "-D_POSIX_C_SOURCE=200112L", "-Wall", "-Werror", "-o", str(exe), str(src),
                    "-I", os.path.join(ROOT, "include"), "-L", lib_dir, "-lfls_gpu", f"-Wl,-rpath,{lib_dir}"],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip().endswith("OK"), out.stdout + out.stderr
    assert "checksum" in out.stdout
