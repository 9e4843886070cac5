"""Generates the committed golden fixtures from the reference's own code.

Run in a container that has the reference sources (they are compiled into
oracle/_ref/libflsref.so by `make -C oracle ref`):

    python tests/golden/make_golden.py

Outputs (all produced by the reference's functions, on seeded inputs that the
tests regenerate with fastlanesgpu_b200.datagen / numpy):
  * reference_pack.npz -- pack.cpp output for bit widths 0..32 of
    uniform_bits(1024, bw, seed=1000+bw); transpose_i/unrsum/pack of a sorted
    vector (delta); VECTOR_RLE of a run vector; the reference's
    unpack_8_at_a_time quarters for bw 4..20.
  * reference_helper_digest.json -- sha256 of the reference's golden unpack-test
    arrays rand_arr_{bw}_b{bw}_w32_arr and of their packed form, so the oracle
    can be checked against them even where the reference is absent.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from fastlanesgpu_b200 import datagen  # noqa: E402
from oracle import Reference, build  # noqa: E402


def main() -> None:
    build(with_reference=True)
    R = Reference()
    out = {}
    for bw in range(33):
        x = datagen.uniform_bits(1024, bw, seed=1000 + bw).view(np.uint32)
        out[f"pack_{bw}"] = R.pack(x, bw)
    s = datagen.sorted_geometric(1024, seed=77).view(np.uint32)
    t = R.transpose_i(s)
    d = R.unrsum(t)
    bw = int(max(int(d.max()), 1)).bit_length()
    out["delta_transposed"] = t
    out["delta_deltas"] = d
    out["delta_bw"] = np.array([bw], np.uint32)
    out["delta_packed"] = R.pack(d, bw)
    out["delta_rsum"] = R.rsum(R.unpack(R.pack(d, bw), bw), t[:32].copy())
    r = datagen.geometric_runs(1024, seed=78)
    n, idx, dic, d4 = R.vector_rle(r)
    out["rle_n"] = np.array([n], np.uint32)
    out["rle_idx"] = idx
    out["rle_dict"] = dic
    out["rle_dict4"] = d4
    for bw in (4, 8, 12, 16, 20):
        x = datagen.uniform_bits(1024, bw, seed=2000 + bw).view(np.uint32)
        p = R.pack(x, bw)
        out[f"quarter_{bw}"] = np.concatenate([R.unpack_quarter(p[q * bw * 8:], bw) for q in range(4)])
    np.savez_compressed(os.path.join(HERE, "reference_pack.npz"), **out)

    dig = {}
    for bw in range(33):
        a = R.helper_arr(bw)
        dig[str(bw)] = {"array_sha256": hashlib.sha256(a.tobytes()).hexdigest(),
                        "packed_sha256": hashlib.sha256(R.pack(a, bw).tobytes()).hexdigest()}
    with open(os.path.join(HERE, "reference_helper_digest.json"), "w") as f:
        json.dump(dig, f, indent=1, sort_keys=True)
    print("wrote", len(out), "arrays and", len(dig), "digests")


if __name__ == "__main__":
    main()
