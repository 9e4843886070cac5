"""Builds libfls_gpu.so in-tree: CUDA sources for sm_100a with nvcc, host
encoders with g++ (OpenMP), linked into one shared library next to this file.

    python -m fastlanesgpu_b200.build          # incremental
    python -m fastlanesgpu_b200.build --clean  # from scratch
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
GEN = os.path.join(ROOT, "_build", "gen")
# Headers compiled again at run time by NVRTC (query specialisation), embedded
# as text under the names their #include lines use.
JIT_HEADERS = [("fls_fixed.cuh", os.path.join(CSRC, "fls_fixed.cuh")),
               ("fls_device.cuh", os.path.join(CSRC, "fls_device.cuh")),
               ("../../include/fls_gpu.h", os.path.join(ROOT, "include", "fls_gpu.h"))]
LIB = os.path.join(PKG, "libfls_gpu.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp"]
CXX = "g++"  # the system compiler (some images export a CXX without libgomp)
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wextra", "-march=x86-64-v3"]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "fls_gpu.h"))
    return hs


def _gen_jit_headers() -> None:
    """Writes _build/gen/fls_jit_headers.inc (only when its text changes)."""
    os.makedirs(GEN, exist_ok=True)
    delim = "FLSJIT"
    out = ["// generated by fastlanesgpu_b200/build.py from the headers it names",
           "struct JitHeader { const char* name; const char* text; };",
           "static const JitHeader kJitHeaders[] = {"]
    for name, path in JIT_HEADERS:
        text = open(path).read()
        if ")" + delim + '"' in text:
            raise RuntimeError(f"{path} contains the raw-string delimiter")
        out.append(f'\t{{"{name}", R"{delim}(' + text + f'){delim}"}},')
    out.append("};")
    body = "\n".join(out) + "\n"
    dst = os.path.join(GEN, "fls_jit_headers.inc")
    if not os.path.exists(dst) or open(dst).read() != body:
        with open(dst, "w") as f:
            f.write(body)


def _stale(obj: str, src: str, headers) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src, *headers])


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(clean: bool = False, verbose: bool = False) -> str:
    """Compile every CUDA / C++ source and link libfls_gpu.so; returns its path."""
    if clean and os.path.isdir(OBJ):
        shutil.rmtree(OBJ)
    os.makedirs(OBJ, exist_ok=True)
    cu, cpp = _sources()
    _gen_jit_headers()
    headers = _headers()
    jobs, objs = [], []
    for f in cu:
        src, obj = os.path.join(CSRC, f), os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if _stale(obj, src, headers):
            jobs.append([NVCC, *NVCC_FLAGS, "-I", GEN, "-Xptxas", "-v", "-c", src, "-o", obj])
    for f in cpp:
        src, obj = os.path.join(CSRC, f), os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if _stale(obj, src, headers):
            jobs.append([CXX, *CXX_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
            for log in ex.map(_compile, jobs):
                if verbose and log:
                    print(log, file=sys.stderr)
    if jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        link = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fopenmp", "-lgomp", "-ldl", "-cudart",
                "static"]
        _compile(link)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(clean=a.clean, verbose=a.verbose))
