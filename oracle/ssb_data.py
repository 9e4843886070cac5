"""TEST INFRASTRUCTURE ONLY: Star Schema Benchmark tables generated by the
reference's own dbgen (data/ssb/dbgen, compiled from its C sources into
_ref/dbgen by the Makefile here) and loaded into int32 columns by ssb_load.c
with the reference loader's integer encoding (data/ssb/loader/convert.py,
load_modified.c).  On these tables the reference holds query answers
(fastlanes/src/include/ssb_utils.h:178-183, data/result_of_queries/q21,q31,
q41; committed as tests/golden/ssb_answers.json by make_ssb_answers.py).

dbgen runs as the reference's data/util.py runs it (`dbgen -s SF -T a`, one
process): its tables share random streams, so generating them one by one
(-T l, -T p, ...) or in parallel chunks (-C/-S) gives other rows.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DBGEN_DIR = os.path.join(HERE, "_ref", "dbgen")
DBGEN = os.path.join(DBGEN_DIR, "dbgen")
DISTS = os.path.join(DBGEN_DIR, "dists.dss")
LOADER = os.path.join(DBGEN_DIR, "ssb_load")

LINEORDER = ["lo_custkey", "lo_partkey", "lo_suppkey", "lo_orderdate", "lo_quantity", "lo_extendedprice",
             "lo_discount", "lo_revenue", "lo_supplycost"]
DIMENSIONS = ["s_suppkey", "s_city", "s_nation", "s_region", "c_custkey", "c_city", "c_nation", "c_region",
              "p_partkey", "p_mfgr", "p_category", "p_brand1", "d_datekey", "d_year", "d_yearmonthnum",
              "d_weeknuminyear"]
# lineorder rows per scale factor (fastlanes/src/include/ssb_utils.h:168-170)
LINEORDER_ROWS = {0.1: 600597, 1: 6001171, 10: 59986214}


def available() -> bool:
    """dbgen and the loader are built (they need the reference's sources)."""
    return all(os.path.exists(p) for p in (DBGEN, DISTS, LOADER))


def default_dir(sf: float) -> str:
    base = os.environ.get("FLS_SSB_DIR") or os.path.join(tempfile.gettempdir(), "fls_ssb")
    return os.path.join(base, f"sf{sf:g}")


def generate(sf: float, out_dir: str | None = None) -> str:
    """dbgen's tables at scale factor `sf` loaded into out_dir/<column>.i32
    (nothing is done when out_dir already holds a complete load).  Returns
    out_dir.  SF 10 takes about two minutes of one core and 6 GB of text on
    the way (deleted after loading)."""
    out_dir = out_dir or default_dir(sf)
    done = os.path.join(out_dir, "complete")
    if os.path.exists(done):
        return out_dir
    if not available():
        raise FileNotFoundError(f"dbgen is not built in {DBGEN_DIR} (make -C oracle dbgen, with the reference "
                                "sources present)")
    os.makedirs(out_dir, exist_ok=True)
    tbl = os.path.join(out_dir, "tbl")
    os.makedirs(tbl, exist_ok=True)
    try:
        subprocess.run([DBGEN, "-s", f"{sf:g}", "-T", "a", "-f", "-b", DISTS], cwd=tbl, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        subprocess.run([LOADER, tbl, out_dir], check=True, stdout=subprocess.DEVNULL)
    finally:
        shutil.rmtree(tbl, ignore_errors=True)
    with open(done, "w") as f:
        f.write(f"sf {sf:g}\n")
    return out_dir


def load(out_dir: str) -> dict:
    """The loaded columns of a generate() directory, name -> int32 array."""
    return {k: np.fromfile(os.path.join(out_dir, k + ".i32"), dtype=np.int32) for k in LINEORDER + DIMENSIONS}


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="generate and load the SSB tables with dbgen")
    ap.add_argument("--sf", type=float, default=10)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    print(generate(args.sf, args.out))
