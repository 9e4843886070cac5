"""The C ABI from plain C on the GPU: a C11 program using the CUDA runtime
API for its own device memory (as the reference's host code does) encodes a
Q1.1-shaped table with fls_encode_uniform, runs fls_decode_sum_u32 and
fls_query_filter_agg on the device, and checks both against sums it computes
itself on the host."""
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime_api.h>
#include "fls_gpu.h"

#define CHECK(x) do { fls_status s_ = (x); if (s_ != FLS_OK) { \
    printf("FAIL %s: %d %s\n", #x, (int)s_, fls_last_error()); return 1; } } while (0)
#define CU(x) do { if ((x) != cudaSuccess) { printf("FAIL %s\n", #x); return 1; } } while (0)

enum { N = 3 * 1024 * 1024 + 77 };

static int encode(const int32_t* v, uint8_t bw, fls_column* col, void** d_words) {
    uint64_t bound = fls_encode_bound_words(N), words = 0;
    uint32_t* enc = (uint32_t*)calloc(bound, 4);
    uint8_t out_bw = 0;
    CHECK(fls_encode_uniform(v, N, FLS_SCHEME_FOR, FLS_LAYOUT_NORMAL, bw, 0, enc, &words, &out_bw));
    CU(cudaMalloc(d_words, 4 * words));
    CU(cudaMemcpy(*d_words, enc, 4 * words, cudaMemcpyHostToDevice));
    memset(col, 0, sizeof(*col));
    col->data = (const uint32_t*)*d_words; col->n_values = N; col->n_words = words;
    col->layout = FLS_LAYOUT_NORMAL; col->scheme = FLS_SCHEME_FOR; col->bw = out_bw; col->base = 0;
    col->max_vec_words = 32u * out_bw; col->scheme_mask = 1u << FLS_SCHEME_FOR;
    free(enc);
    return 0;
}

int main(void) {
    static int32_t date[N], disc[N], qty[N], price[N];
    uint64_t seed = 12345;
    for (int i = 0; i < N; ++i) {
        seed = seed * 6364136223846793005ull + 1442695040888963407ull;
        date[i] = (int32_t)((seed >> 33) % 2556); disc[i] = (int32_t)((seed >> 20) % 11);
        qty[i] = 1 + (int32_t)((seed >> 40) % 50); price[i] = 90000 + (int32_t)((seed >> 10) % 10000000);
    }
    fls_column cols[4];
    void* d[4];
    const int32_t* src[4] = {date, disc, qty, price};
    const uint8_t bws[4] = {12, 4, 6, 24};
    for (int c = 0; c < 4; ++c) { if (encode(src[c], bws[c], &cols[c], &d[c])) return 1; }
    uint64_t* d_sum; int64_t* d_res;
    CU(cudaMalloc((void**)&d_sum, 8)); CU(cudaMalloc((void**)&d_res, 8));
    /* decode fused with a sum (bitpack_shared_memory.cu QueryKernel) */
    CHECK(fls_decode_sum_u32(&cols[3], d_sum, NULL));
    uint64_t got_sum = 0, want_sum = 0;
    CU(cudaMemcpy(&got_sum, d_sum, 8, cudaMemcpyDeviceToHost));
    for (int i = 0; i < N; ++i) want_sum += (uint32_t)price[i];
    /* the Q1.1 filter-aggregate (fls_q11.cu QueryKernel_v1) */
    fls_filter_agg_desc q;
    memset(&q, 0, sizeof(q));
    q.cols = cols; q.n_cols = 4;
    q.filters[0].col = 0; q.filters[0].lo = 366; q.filters[0].hi = 730;
    q.filters[1].col = 1; q.filters[1].lo = 1; q.filters[1].hi = 3;
    q.filters[2].col = 2; q.filters[2].lo = -2147483647 - 1; q.filters[2].hi = 24;
    q.n_filters = 3; q.agg_a = 3; q.agg_b = 1;
    CHECK(fls_query_filter_agg(&q, d_res, NULL));
    CHECK(fls_check_device_error(NULL));
    int64_t got_q = 0, want_q = 0;
    CU(cudaMemcpy(&got_q, d_res, 8, cudaMemcpyDeviceToHost));
    for (int i = 0; i < N; ++i)
        if (date[i] >= 366 && date[i] <= 730 && disc[i] >= 1 && disc[i] <= 3 && qty[i] <= 24)
            want_q += (int64_t)price[i] * disc[i];
    printf("sum %llu/%llu query %lld/%lld\n", (unsigned long long)got_sum, (unsigned long long)want_sum,
           (long long)got_q, (long long)want_q);
    for (int c = 0; c < 4; ++c) cudaFree(d[c]);
    cudaFree(d_sum); cudaFree(d_res);
    if (got_sum != want_sum || got_q != want_q || want_q == 0) { printf("FAIL results\n"); return 1; }
    printf("OK\n");
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_c_program_on_the_gpu(cuda, tmp_path):
    lib_dir = os.path.join(ROOT, "fastlanesgpu_b200")
    src = tmp_path / "user_gpu.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "user_gpu"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-o", str(exe), str(src), "-I", os.path.join(ROOT, "include"),
                    "-I", f"{CUDA}/include", "-L", lib_dir, "-L", f"{CUDA}/lib64", "-lfls_gpu", "-lcudart",
                    f"-Wl,-rpath,{lib_dir}", f"-Wl,-rpath,{CUDA}/lib64"], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip().endswith("OK"), out.stdout + out.stderr
