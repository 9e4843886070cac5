#!/usr/bin/env python
"""Benchmark of the fused FastLanes decode + query path on B200.

Headline workload (one "step" = one pass of the hot path over the table):
fused decode + filter-aggregate over a synthetic 2^27-row fact table
(date 12 bit, discount 4 bit, quantity 6 bit, price 24 bit, FastLanes
bit-packed; year-1993 AND discount in [1,3] AND quantity < 25; exact int64
sum(price*discount)) -- the Q1.1 shape of fastlanes/src/ssb/fls_q11.cu.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload q11|q21|decode]

Prints ONE JSON line on rank 0.  With --gpus N > 1 it is launched under
torchrun: each rank holds its own shard of 2^27 rows (weak scaling) and the
per-step int64 partial aggregates are summed with one NCCL all-reduce.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["q11", "q21", "q31", "q41", "ssb", "ssb-real", "decode", "mixed"],
                    default="q11")
    ap.add_argument("--ssb-dir", default="",
                    help="ssb-real: directory of the Star Schema Benchmark columns loaded from dbgen's tables "
                         "(<column>.i32; default $FLS_SSB_DIR/sf10 or <tmp>/fls_ssb/sf10)")
    ap.add_argument("--rows", type=int, default=0, help="rows per GPU (0 = 2^27 for queries, 2^28 for decode)")
    ap.add_argument("--decode-bw", type=int, default=16, help="bit width of the FOR decode workload")
    ap.add_argument("--decode-width", type=int, choices=[8, 16, 32, 64], default=32,
                    help="decode workload, FOR: value width of the FastLanes lanes (8/16/64: fls_decode_u8/u16/u64)")
    ap.add_argument("--decode-scheme", choices=["for", "delta", "rle", "dict", "rfor"], default="for",
                    help="decode input: uniform FOR bit-packing, delta over sorted keys (geometric gaps p=0.3), "
                         "RLE (geometric runs of mean 16, values in [0,2^16)), dictionary (Zipf 1.1 over 2^20), "
                         "the reference's tile-based RLE format (rfor; the same runs)")
    ap.add_argument("--decode-out", choices=["sum", "hbm"], default="sum",
                    help="decode fused with a uint64 sum, or decode to HBM")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--secondary", choices=["all", "none"], default="all",
                    help="with the default workload on 1 GPU: also measure the other configurations (Q2.1, Q3.1 and "
                         "Q4.1 joins, the FOR decode sweep over bit widths 1..32 and DELTA/RLE/DICT decode at 2^28 "
                         "values, learned vs exhaustive encoding and the batch) and add them to the line")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--launch", default="", help="warps,stages,ctas_per_sm,tile_bytes (0 = default)")
    ap.add_argument("--sparse-rows", type=int, default=0, help="FLS_TUNE_SPARSE_ROWS (0 = default)")
    ap.add_argument("--jit", type=int, choices=[0, 1], default=1,
                    help="FLS_TUNE_JIT: 1 = kernel specialised to the query's shape, 0 = general kernel")
    ap.add_argument("--late-measure", type=int, choices=[0, 1], default=None,
                    help="FLS_TUNE_LATE_MEASURE: 1 = join measures read from global memory for selected rows only")
    ap.add_argument("--tune-joins", type=int, choices=[0, 1], default=None,
                    help="join workloads (q21, q31, q41, each join of ssb): choose the join variants with the "
                         "autotuner (JOIN_SPACE) before timing; default 1 unless --late-measure, --table-kb or "
                         "--group-smem is given (ssb: always 1 by default)")
    ap.add_argument("--table-kb", type=int, default=0,
                    help="FLS_TUNE_TABLE_KB: shared-memory budget of the join kernels' hash tables (0 = default 72)")
    ap.add_argument("--half-vectors", type=int, choices=[0, 1], default=None,
                    help="FLS_TUNE_HALF_VECTORS: join kernels stage half vectors (1) or whole ones (0)")
    ap.add_argument("--group-smem", type=int, choices=[0, 1], default=None,
                    help="FLS_TUNE_GROUP_SMEM: 1 = per-CTA group sums in shared memory, 0 = a global atomic per row")
    ap.add_argument("--mixed-columns", type=int, default=64, help="mixed workload: number of columns")
    ap.add_argument("--mixed-max-log", type=int, default=26, help="mixed workload: longest column is 2^this rows")
    ap.add_argument("--train-vectors", type=int, default=1 << 20, help="mixed workload: MLP training vectors")
    ap.add_argument("--train-epochs", type=int, default=6)
    ap.add_argument("--queries", type=int, default=256, help="mixed workload: batched filter-aggregate queries")
    ap.add_argument("--threshold", type=float, default=0.9, help="selector confidence below which the "
                                                                    "exhaustive encoder decides")
    ap.add_argument("--decode-kappa", type=float, default=0.03,
                    help="training labels: argmin size * (1 + kappa * (decode cost - 1))")
    a = ap.parse_args()
    if not a.rows:
        a.rows = (1 << 28) if a.workload == "decode" else (1 << 27)
    return a


# ------------------------------------------------------------------ helpers

class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, backend="nccl"):
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(self.local)
        if self.world > 1:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", self.local))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples of this rank's GPU."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        import torch
        self.proc = None
        self.window = None
        try:
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            sel = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
        except Exception:
            sel = str(device_index)
        self.cmd = ["nvidia-smi", "-i", sel, f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                    "-lms", "50"]

    def start(self):
        try:
            self.proc = subprocess.Popen(self.cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        self.t_start = time.time()

    def mark(self, t0: float, t1: float):
        self.window = (t0, t1)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        rows = [r for r in csv.reader(io.StringIO(out)) if len(r) >= 9]
        n = len(rows)
        if n == 0:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        # nvidia-smi -lms emits at a fixed period; map samples to wall time.
        t_end = time.time()
        period = (t_end - self.t_start) / n
        stamps = [self.t_start + (i + 1) * period for i in range(n)]
        sel = [r for r, t in zip(rows, stamps) if self.window and self.window[0] <= t <= self.window[1]]
        scope = "timed"
        if not sel:
            sel, scope = rows, "run"
        sm = [float(r[1]) for r in sel if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in sel if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in sel for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sel), "window": scope}


def measured_peak_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(key: str):
    """DRAM bytes per launch of the dominant kernel from a committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(key)
    except Exception:
        return None


# --------------------------------------------------------------- workloads

def build_q11(rows: int, seed: int):
    from fastlanesgpu_b200 import EncodedColumn, datagen
    t = datagen.lineorder_q11(rows, seed=seed)
    names = ["date", "discount", "quantity", "price"]
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q11_BITS[k]) for k in names]
    f = datagen.Q11_FILTER
    filters = [(0, *f["date"]), (1, *f["discount"]), (2, *f["quantity"])]
    return t, cols, filters


def build_q21(rows: int, seed: int):
    from fastlanesgpu_b200 import EncodedColumn, datagen
    t = datagen.q21_tables(rows, seed=seed)
    names = ["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"]
    cols = [EncodedColumn.uniform(t[k], bw=datagen.Q21_BITS[k]) for k in names]
    return t, cols


def run_ours(a, dist: Dist):
    import numpy as np
    import torch

    from fastlanesgpu_b200 import EncodedColumn, datagen, ops
    dev = torch.device("cuda", dist.local)
    stream = torch.cuda.current_stream()
    if a.launch:
        ops.set_launch_config(*[int(x) for x in a.launch.split(",")])
    if a.sparse_rows:
        ops.set_tuning(0, a.sparse_rows)
    ops.set_tuning(1, a.jit)
    if a.group_smem is not None:
        ops.set_tuning(2, a.group_smem)
    if a.late_measure is not None:
        ops.set_tuning(3, a.late_measure)
    ops.set_tuning(4, a.table_kb)
    if a.half_vectors is not None:
        ops.set_tuning(5, a.half_vectors)
    explicit_variants = (a.late_measure is not None or a.table_kb != 0 or a.group_smem is not None or
                         a.half_vectors is not None)
    tune_joins = a.tune_joins if a.tune_joins is not None else int(a.workload in ("ssb", "ssb-real") or
                                                                    not explicit_variants)
    from fastlanesgpu_b200.shard import allreduce_sum, combine_group_records, shard_seed
    seed = shard_seed(1000, dist.rank)
    # ---------------------------------------------------------------- setup
    if a.workload == "q11":
        t, hcols, filters = build_q11(a.rows, seed)
        dcols = [c.to_device(dev) for c in hcols]
        res = torch.zeros(1, dtype=torch.int64, device=dev)

        def step():
            ops.query_filter_agg(dcols, filters, agg_a=3, agg_b=1, out=res)
            return res
        workload = {"workload": "fused decode + filter-aggregate (Q1.1 shape)", "rows_per_gpu": a.rows,
                    "columns": "date 12b, discount 4b, quantity 6b, price 24b (FastLanes bit-packed, uniform)",
                    "predicate": "date in year 1993 AND discount in [1,3] AND quantity < 25",
                    "aggregate": "int64 sum(price*discount)"}
        metric_key = "q11"
    elif a.workload == "q21":
        t, hcols = build_q21(a.rows, seed)
        dcols = [c.to_device(dev) for c in hcols]
        dt = {k: torch.from_numpy(v).to(dev) for k, v in t.items() if not k.startswith("lo_")}
        ht_s = ops.build_pht(dt["s_suppkey"], dt["s_suppkey"].numel(), filt=dt["s_region"], filter_eq=1)
        ht_p = ops.build_pht(dt["p_partkey"], dt["p_partkey"].numel(), vals=dt["p_brand1"], filt=dt["p_category"],
                             filter_eq=1)
        ht_d = ops.build_pht(dt["d_datekey"], datagen.N_DAYS, vals=dt["d_year"])
        tabs = {"ht_s": ht_s, "ht_p": ht_p, "ht_d": ht_d}
        probes = [(0, ht_s, ht_s.numel(), 0, 1), (1, ht_p, ht_p.numel() // 2, 0, 2),
                  (2, ht_d, ht_d.numel() // 2, 0, 2)]
        res = torch.zeros(4 * datagen.N_GROUPS, dtype=torch.int32, device=dev)

        def step():
            ops.probe_groupby(dcols, probes, 3, 1, 2, 7, 1992, datagen.N_GROUPS, out=res)
            return res
        workload = {"workload": "fused decode + 3-way perfect-hash probe + 7000-group int64 group-by (Q2.1 shape)",
                    "rows_per_gpu": a.rows, "columns": "supp 17b, part 19b, date 12b, revenue 24b",
                    "filters": "part category 1/5, supplier region 1/25"}
        metric_key = "q21"
    elif a.workload in ("q31", "q41"):
        t, tables, hcols, dcols, probes, jkw = datagen.ssb_join(a.workload, a.rows, seed, device=dev)
        tabs = tables
        res = torch.zeros(jkw["res_stride"] * jkw["n_groups"], dtype=torch.int32, device=dev)

        def step():
            ops.join_groupby(dcols, probes, out=res, **jkw)
            return res
        if a.workload == "q31":
            workload = {"workload": "fused decode + 3 perfect-hash probes + 4375-group int64 group-by (Q3.1 shape, "
                                    "fls_q31.cu)", "rows_per_gpu": a.rows,
                        "columns": "supp 17b, cust 18b, date 12b, revenue 24b",
                        "filters": "supplier region 1/5, customer region 1/5, years 1992-1997"}
        else:
            workload = {"workload": "fused decode + 4 perfect-hash probes + 175-group int64 sum(revenue - supplycost) "
                                    "(Q4.1 shape, fls_q41.cu)", "rows_per_gpu": a.rows,
                        "columns": "supp 17b, cust 18b, part 19b, date 12b, revenue 24b, supplycost 18b",
                        "filters": "supplier region 1/5, customer region 1/5, part manufacturer 2/5"}
        metric_key = a.workload
    elif a.workload in ("ssb", "ssb-real"):
        # the thirteen SSB queries over one lineorder table (dimension tables
        # and hash tables replicated per rank); results side by side in one
        # int32 buffer, 8-byte aligned per query
        if a.workload == "ssb":
            t = datagen.ssb_tables(a.rows, seed=seed)
            names = list(datagen.SSB_BITS)
            hcols = [EncodedColumn.uniform(t[k], bw=datagen.SSB_BITS[k]) for k in names]
            make_query = datagen.ssb_device_query
        else:
            # dbgen's tables in the reference loader's encoding, every rank the same
            t = datagen.ssb_dbgen_load(a.ssb_dir or datagen.ssb_dbgen_default_dir(10))
            a.rows = int(t["lo_orderdate"].size)
            enc = datagen.ssb_dbgen_columns(t)
            names = list(enc)
            hcols = [enc[k] for k in names]
            make_query = datagen.ssb_dbgen_query
        dcols = [c.to_device(dev) for c in hcols]
        dmap = dict(zip(names, dcols))
        suite, off = [], 0
        for name in datagen.SSB_QUERIES:
            dq = make_query(name, t, dmap, device=dev)
            words = 2 if dq["kind"] == "filter" else dq["kw"]["res_stride"] * dq["kw"]["n_groups"]
            suite.append((name, dq, off, words))
            off += words + (words & 1)
        dims = ("supplier 2^17, customer 2^18, part 2^19 keys, 2556 days; cities/nations/regions and "
                "brands/categories/manufacturers in dbgen's hierarchy") if a.workload == "ssb" else \
            ", ".join(f"{k} {t[k].size}" for k in ("s_suppkey", "c_custkey", "p_partkey", "d_datekey"))
        del t
        res = torch.zeros(off, dtype=torch.int32, device=dev)
        suite_bytes = sum(sum(c.nbytes for c in dq["cols"]) for _, dq, _, _ in suite)

        def run_query(dq, o, w):
            if dq["kind"] == "filter":
                ops.query_filter_agg(dq["cols"], dq["filters"], agg_a=3, agg_b=1, out=res[o:o + 2].view(torch.int64))
            else:
                if dq.get("tuned"):
                    autotune.apply(dq["tuned"])
                ops.join_groupby(dq["cols"], dq["probes"], out=res[o:o + w], **dq["kw"])

        from fastlanesgpu_b200 import autotune
        if tune_joins:
            # the library's autotuner picks each join's variants (late or
            # staged measures, group sums per CTA or per row, shared-memory
            # budget of the hash tables) by timing them,
            # before the timed region; the step applies each query's choice
            for name, dq, o, w in suite:
                if dq["kind"] == "join":
                    best = autotune.tune(f"ssb-{name}", lambda: run_query(dq, o, w), space=autotune.JOIN_SPACE,
                                         iters=10, use_cache=False, prefer=autotune.JOIN_DEFAULT, margin=0.02,
                                         retime=3)
                    dq["tuned"] = best["config"]
            autotune.reset()

        def step():
            for _, dq, o, w in suite:
                run_query(dq, o, w)
            return res
        what = ("SSB suite: Q1.1-Q4.3 (crystal-opt src/ssb q11..q43 shapes) over one lineorder table, 13 fused "
                "decode+query launches per step")
        if a.workload == "ssb-real":
            what += (f"; the Star Schema Benchmark's own data (dbgen, {a.rows} lineorder rows, the reference loader's "
                     "encoding), FastLanes FOR columns at the smallest bit widths")
        workload = {"workload": what,
                    "rows_per_gpu": a.rows, "rows_scanned_per_step": 13 * a.rows,
                    "columns": ", ".join(f"{k[3:]} {c.bw}b" for k, c in zip(names, hcols)),
                    "dimensions": dims,
                    "join_variants": {name: dq.get("tuned", "defaults") for name, dq, _, _ in suite
                                      if dq["kind"] == "join"}}
        metric_key = a.workload
    else:
        from fastlanesgpu_b200 import LAYOUT_TRANSPOSED, SCHEME_DELTA, SCHEME_RLE
        if a.decode_scheme == "for" and a.decode_width != 32:
            vals, hcols = None, []  # built below
        elif a.decode_scheme == "for":
            vals = datagen.uniform_bits(a.rows, a.decode_bw, seed=seed)
            hcols = [EncodedColumn.uniform(vals, bw=a.decode_bw)]
            what, key = f"bit-pack + FOR, bw {a.decode_bw} (uniform column)", f"for_bw{a.decode_bw}"
        elif a.decode_scheme == "delta":
            vals = datagen.sorted_geometric(a.rows, p=0.3, seed=seed)
            hcols = [EncodedColumn.encode(vals, SCHEME_DELTA, layout=LAYOUT_TRANSPOSED)]
            what, key = "delta over sorted keys with geometric gaps (p=0.3), per-vector bw", "delta"
        elif a.decode_scheme == "rfor":
            from fastlanesgpu_b200.column import RforColumn
            vals = datagen.geometric_runs(a.rows, mean_run=16.0, value_bits=16, seed=seed)
            hcols = [RforColumn.encode(vals)]
            what, key = "tile-based RLE (RFOR), geometric runs (mean 16) of values in [0,2^16)", "rfor"
        elif a.decode_scheme == "rle":
            vals = datagen.geometric_runs(a.rows, mean_run=16.0, value_bits=16, seed=seed)
            hcols = [EncodedColumn.encode(vals, SCHEME_RLE, layout=LAYOUT_TRANSPOSED)]
            what, key = "RLE, geometric runs (mean 16) of values in [0,2^16)", "rle"
        else:
            from fastlanesgpu_b200 import SCHEME_DICT
            vals = datagen.zipf_device(a.rows, s=1.1, domain=1 << 20, seed=seed, device=dev).cpu().numpy()
            hcols = [EncodedColumn.encode(vals, SCHEME_DICT, layout=LAYOUT_TRANSPOSED)]
            what, key = "dictionary, Zipf 1.1 over [0,2^20)", "dict"
        del vals
        dcols = [c.to_device(dev) for c in hcols]
        if a.decode_scheme == "for" and a.decode_width != 32:
            # the same decode over lanes of another width: values uniform in
            # [0, 2^bw), bw capped at the width
            bits, bw_w = a.decode_width, min(a.decode_bw, a.decode_width)
            dt = {8: np.uint8, 16: np.uint16, 64: np.uint64}[bits]
            raw = np.random.default_rng(seed).integers(0, 2**64 - 1, a.rows, dtype=np.uint64, endpoint=True)
            if bw_w < 64:
                raw &= np.uint64((1 << bw_w) - 1)
            packed = ops.pack_column_width(raw.astype(dt), bw_w, 0)
            del raw
            n_vec_w = (a.rows + 1023) // 1024

            class _Packed:  # host column for the end-to-end copies
                words, meta, nbytes = packed.view(np.uint32), None, n_vec_w * 128 * bw_w

            class _DevPacked:
                data = torch.from_numpy(packed.view(np.int32)).to(dev)
                n_vec = n_vec_w
            hcols, dcols = [_Packed], [_DevPacked]
            tdt = {8: torch.uint8, 16: torch.int16, 64: torch.int64}[bits]
            if a.decode_out == "sum":
                res = torch.zeros(1, dtype=torch.int64, device=dev)

                def step():
                    ops.decode_width_into(_DevPacked.data, a.rows, bits, bw_w, 0, None, res)
                    return res
            else:
                res = torch.empty(n_vec_w * 1024, dtype=tdt, device=dev)

                def step():
                    ops.decode_width_into(_DevPacked.data, a.rows, bits, bw_w, 0, res, None)
                    return res
            out_bytes = (bits // 8) * n_vec_w * 1024 if a.decode_out == "hbm" else 0
            what = f"bit-pack {bits}-bit lanes, bw {bw_w} (uniform column, fls_decode_u{bits})"
            key = f"u{bits}_bw{bw_w}"
        elif a.decode_scheme == "rfor":
            if a.decode_out == "sum":
                res = torch.zeros(1, dtype=torch.int64, device=dev)

                def step():
                    ops.rfor_decode_sum(dcols[0], out=res)
                    return res
            else:
                res = torch.empty(a.rows, dtype=torch.int32, device=dev)

                def step():
                    ops.rfor_decode(dcols[0], out=res)
                    return res
            out_bytes = 4 * a.rows if a.decode_out == "hbm" else 0
        elif a.decode_out == "sum":
            res = torch.zeros(1, dtype=torch.int64, device=dev)

            def step():
                ops.query_aggregate(dcols[0], out=res)
                return res
        else:
            res = torch.empty(dcols[0].n_vec * 1024, dtype=torch.int32, device=dev)

            def step():
                ops.unpack_global(dcols[0], out=res)
                return res
        if not (a.decode_scheme == "for" and a.decode_width != 32) and a.decode_scheme != "rfor":
            out_bytes = 4 * dcols[0].n_vec * 1024 if a.decode_out == "hbm" else 0
        workload = {"workload": f"decode {'to HBM' if a.decode_out == 'hbm' else 'fused with uint64 sum'}: {what}",
                    "rows_per_gpu": a.rows}
        metric_key = f"decode_{a.decode_out}_{key}"
    if a.workload in ("q21", "q31", "q41") and tune_joins:
        # the library's autotuner picks the join variants (late or staged
        # measures, group sums per CTA or per row, shared-memory budget of
        # the hash tables) by timing them, before the timed region
        from fastlanesgpu_b200 import autotune
        best = autotune.tune(f"{a.workload}-{a.rows}", step, space=autotune.JOIN_SPACE, iters=20, use_cache=False,
                             prefer=autotune.JOIN_DEFAULT, margin=0.02, retime=3)
        workload["join_variants"] = best["config"]
    comp_bytes = sum(c.nbytes for c in hcols)
    algo_bytes = comp_bytes + (out_bytes if a.workload == "decode" else 0)
    if a.workload in ("ssb", "ssb-real"):
        algo_bytes = suite_bytes  # every query reads its own columns

    def collective():
        # the one exchange of the sharded query: combine the ranks' partial aggregates
        if not dist.pg:
            return
        if a.workload in ("ssb", "ssb-real"):
            for _, dq, o, w in suite:
                if dq["kind"] == "filter":
                    allreduce_sum(res[o:o + 2].view(torch.int64))
                else:
                    kw = dq["kw"]
                    combine_group_records(res[o:o + w], kw["res_stride"], kw["sum_slot"], kw["sum_bits"])
        elif a.workload in ("q21", "q31", "q41"):
            stride, sum_slot = (4, 2) if a.workload == "q21" else (jkw["res_stride"], jkw["sum_slot"])
            combine_group_records(res, stride, sum_slot)
        elif a.workload == "decode" and a.decode_out == "hbm":
            return  # each rank's decoded shard is its final output: nothing to exchange
        else:
            allreduce_sum(res)  # the int64 partial sum (filter-aggregate, decode fused with a sum)

    # -------------------------------------------------- device-resident timing
    clocks = ClockSampler(dist.local)
    clocks.start()
    for _ in range(a.warmup):
        step()
        collective()
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    l0 = ops.kernel_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    e0.record(stream)
    for _ in range(a.steps):
        step()
        collective()
    e1.record(stream)
    torch.cuda.synchronize()
    w1 = time.time()
    dist.barrier()
    launches = ops.kernel_launch_count() - l0
    clocks.mark(w0, w1)
    ms_local = e0.elapsed_time(e1)
    ms = dist.max(ms_local)
    ops.check_device_error()

    # ------------------------------------------- end-to-end through the C ABI
    # every encoded buffer of every column: packed words and, for per-vector
    # columns, the vector metadata
    copies = []
    if a.workload == "decode" and a.decode_scheme == "rfor":
        hc, dc = hcols[0], dcols[0]
        for dst, src in ((dc.values, hc.values), (dc.run_lengths, hc.run_lengths), (dc.val_offsets, hc.val_offsets),
                         (dc.rl_offsets, hc.rl_offsets)):
            copies.append((dst, torch.from_numpy(src.view("int32")).pin_memory()))
    else:
        for c, dc in zip(hcols, dcols):
            copies.append((dc.data, torch.from_numpy(c.words.view("int32")).pin_memory()))
            if c.meta is not None:
                copies.append((dc.meta, torch.from_numpy(c.meta.view(np.uint8)).pin_memory()))
    h2d = sum(hp.numel() * hp.element_size() for _, hp in copies)
    d2h = res.numel() * res.element_size()
    host_res = torch.empty_like(res, device="cpu").pin_memory()
    n_e2e = max(3, min(a.e2e_steps, a.steps))
    torch.cuda.synchronize()
    dist.barrier()
    x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    for _ in range(n_e2e):
        for dst, hp in copies:
            dst.copy_(hp.view(dst.dtype).view(dst.shape), non_blocking=True)
        step()
        collective()
        host_res.copy_(res, non_blocking=True)
    x1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = dist.max(x0.elapsed_time(x1)) / n_e2e
    clk = clocks.stop()
    per_query = None
    if a.workload in ("ssb", "ssb-real"):
        # each query alone (outside the timed region), CUDA events, 20 runs
        per_query = {}
        for name, dq, o, w in suite:
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            run_query(dq, o, w)
            q0.record(stream)
            for _ in range(20):
                run_query(dq, o, w)
            q1.record(stream)
            torch.cuda.synchronize()
            qb = sum(c.nbytes for c in dq["cols"])
            qms = q0.elapsed_time(q1) / 20
            per_query[name] = {"ms": round(qms, 4), "hbm_frac": round(qb / (qms / 1e3) / 1e9 / measured_peak_gbs()[0],
                                                                       3)}

    answers = ssb_real_answers(a.rows, suite, res) if a.workload == "ssb-real" else None
    if a.workload == "decode" and a.decode_out == "hbm":
        exchange = "no exchange (each rank keeps its decoded shard)"
    elif a.workload in ("q21", "q31", "q41", "ssb", "ssb-real"):
        exchange = "group records combined per step (all-reduce MAX of the key words, SUM of the group sums)"
    else:
        exchange = "one int64 all-reduce per step"
    rows_total = a.rows * dist.world * (13 if a.workload in ("ssb", "ssb-real") else 1)
    value = rows_total * a.steps / (ms / 1e3)
    ms_step = ms / a.steps
    peak, peak_src = measured_peak_gbs()
    achieved = algo_bytes / (ms_local / a.steps / 1e3) / 1e9
    # profiled traffic is per launch at the default size; it grows with the
    # vectors processed
    traffic = profiled_traffic(metric_key)
    if traffic is not None:
        traffic = int(traffic * a.rows / ((1 << 28) if a.workload == "decode" else (1 << 27)))
    out = {
        "metric": "fused decode+query rows/s", "value": value, "unit": "rows/s", "n_gpus": dist.world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32->int64", "data": "synthetic (seeded)",
        "config": {**workload, "rows_total": rows_total, "compressed_bytes_per_gpu": comp_bytes,
                   "l2": "inputs larger than L2 (126 MB), no flush",
                   "parallelism": (f"row shards x{dist.world}, " + exchange) if dist.world > 1 else "1 GPU"},
        "e2e": {"value": rows_total / (e2e_ms / 1e3), "unit": "rows/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "path": "pinned host encoded columns -> H2D -> fused kernel (C ABI) -> D2H result"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured"
                     else "fallback 6650 GB/s",
                     "traffic": traffic, "algorithmic_bytes_per_launch": algo_bytes},
        "gpu_launches": int(launches),
        "launch_config": dict(zip(["warps", "stages", "ctas_per_sm", "tile_bytes"], ops.get_launch_config()),
                              sparse_rows=ops.get_tuning(0), jit=ops.get_tuning(1), group_smem=ops.get_tuning(2),
                              late_measure=ops.get_tuning(3), table_kb=ops.get_tuning(4),
                              half_vectors=ops.get_tuning(5),
                              jit_launches=int(ops.jit_stats()["launches"])),
        "clocks": clk,
    }
    if answers is not None:
        out["reference_answers"] = answers
    if per_query is not None:
        out["per_query"] = per_query
        out["roofline"]["algorithmic_bytes_per_launch"] = algo_bytes
        out["roofline"]["note"] = "a step is 13 query launches; bytes and time are the whole step's"
    ctx = {"workload": a.workload, "hcols": hcols, "res": res,
           "tabs": {k: v.cpu().numpy() for k, v in tabs.items()} if a.workload in ("q21", "q31", "q41") else None}
    return out, ctx


M64 = (1 << 64) - 1


def ssb_real_answers(rows: int, suite, res) -> dict:
    """The SSB results on dbgen's data against the answers the reference holds
    (fastlanes/src/include/ssb_utils.h:178-183 and data/result_of_queries,
    committed as tests/golden/ssb_answers.json): Q1.1 at scale factors 0.1, 1
    and 10, Q1.2 and Q1.3 at 1, every group of Q2.1, Q3.1 and Q4.1 at 10."""
    import numpy as np
    with open(os.path.join(ROOT, "tests", "golden", "ssb_answers.json")) as f:
        ans = json.load(f)
    sf = {600597: "0.1", 6001171: "1", 59986214: "10"}.get(rows)
    got = {name: (dq, o, w) for name, dq, o, w in suite}
    checked, equal = [], True
    for name, by_sf in ans["scalar"].items():
        if sf in by_sf:
            dq, o, w = got[name]
            v = int(res[o:o + 2].view(__import__("torch").int64).cpu()[0])
            checked.append(name)
            equal = equal and v == by_sf[sf]
    if sf == "10":
        for name, key_words in (("q21", 2), ("q31", 3), ("q41", 2)):
            dq, o, w = got[name]
            kw = dq["kw"]
            rec = res[o:o + w].cpu().numpy().reshape(-1, kw["res_stride"])
            sums = rec[:, kw["sum_slot"]:kw["sum_slot"] + 2].copy().view(np.int64)[:, 0]
            rows_ = sorted([int(x) for x in r[:key_words]] + [int(s_)] for r, s_ in zip(rec, sums) if s_ != 0)
            checked.append(name)
            equal = equal and rows_ == sorted(ans["groups_sf10"][name])
    return {"scale_factor": sf, "checked": checked, "equal": bool(equal and checked)}

REF_HOW = {
    "q11": "the reference's unpack (unpack_fused.cuh, host-compiled from its sources) + the fls_q11.cu loop",
    "q21": "the reference's unpack (host-compiled from its sources) + the fls_q21.cu probe_v1 loop",
    "q31": "the reference's unpack (host-compiled from its sources) + the fls_q31.cu probe_v1 loop",
    "q41": "the reference's unpack (host-compiled from its sources) + the fls_q41.cu probe_v1 loop",
    "decode": "the reference's unpack (unpack.cuh, host-compiled from its sources) + uint64 sum",
}


def cpu_info() -> dict:
    """The host CPU: model name (/proc/cpuinfo) and the cores this process may use."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except Exception:
        usable = os.cpu_count() or 1
    return {"model": model, "logical_cpus": os.cpu_count(), "usable_cpus": usable}


def _time_cpu(fn, args, budget_s: float, min_reps: int = 3, max_reps: int = 100000):
    """fn(*args) once untimed, then at least min_reps timed runs and more
    until budget_s is spent: (median seconds, runs, last result)."""
    res = fn(*args)
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < min_reps or (time.perf_counter() < t_end and len(times) < max_reps):
        t0 = time.perf_counter()
        res = fn(*args)
        times.append(time.perf_counter() - t0)
    return statistics.median(times), len(times), res


def reference_call(R, workload: str, words, bws, n_rows: int, tabs, threads: int, decode_bw: int = 0):
    """(function, arguments) of the reference's CPU implementation of a
    workload over packed words (uniform FOR columns in the reference's
    format) and, for the joins, the perfect hash tables."""
    from fastlanesgpu_b200 import datagen
    if workload == "q11":
        f = datagen.Q11_FILTER
        return R.q11_sum, (words, bws, n_rows, *f["date"], *f["discount"], f["quantity"][1] + 1, threads)
    if workload == "q21":
        return R.q21_groupby, (words, bws, n_rows, tabs["ht_s"], tabs["ht_p"], tabs["ht_d"], 0, threads)
    if workload == "q31":
        return R.q31_groupby, (words, bws, n_rows, tabs["ht_s"], tabs["ht_c"], tabs["ht_d"], 0, threads)
    if workload == "q41":
        return R.q41_groupby, (words, bws, n_rows, tabs["ht_s"], tabs["ht_c"], tabs["ht_p"], tabs["ht_d"], 0,
                               threads)
    return R.decode_sum, (words[0], decode_bw, (n_rows + 1023) // 1024, threads)


def _same_result(workload: str, ref, res) -> bool:
    """The reference's result equals the GPU's (device tensor `res`)."""
    import numpy as np
    if workload in ("q21", "q31", "q41"):
        return bool(np.array_equal(np.asarray(ref), res.cpu().numpy()))
    got = int(res.cpu()[0])
    return (got & M64) == (int(ref) & M64)


def cpu_baseline(a, ctx, budget_s: float) -> dict:
    """The reference's CPU implementation of the benched workload (its own
    unpack compiled from its sources + its scalar query loop), timed on the
    host cores over the WHOLE benched table with all usable threads, and on a
    prefix with one thread; its result on the whole table is compared with
    the GPU's result (the bench line fails on a mismatch)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as orc
    R = orc.Reference()
    info = cpu_info()
    threads = info["usable_cpus"]
    w = ctx["workload"]
    words = [np.ascontiguousarray(c.words).view(np.uint32) for c in ctx["hcols"]]
    bws = [c.bw for c in ctx["hcols"]]
    fn, args = reference_call(R, w, words, bws, a.rows, ctx["tabs"], threads, a.decode_bw)
    med, reps, ref = _time_cpu(fn, args, budget_s)
    n1 = min(a.rows, 1 << 22)
    fn1, args1 = reference_call(R, w, words, bws, n1, ctx["tabs"], 1, a.decode_bw)
    med1, reps1, _ = _time_cpu(fn1, args1, budget_s / 4, min_reps=1)
    return {"value": a.rows / med, "unit": "rows/s", "cores": threads, "kind": "reference", "cpu": info,
            "sample": f"the whole benched table ({a.rows} rows), {reps} runs after one untimed, median; "
                      f"{REF_HOW[w]}, OpenMP {threads} threads",
            "single_thread": {"value": n1 / med1, "unit": "rows/s", "cores": 1,
                              "sample": f"first {n1} rows of the table, {reps1} runs, median, 1 thread"},
            "result_equal": _same_result(w, ref, ctx["res"])}


def _pad_vectors(v):
    """A column padded to whole vectors with its last value (as the encoder pads)."""
    import numpy as np
    r = (-v.size) % 1024
    return v if r == 0 else np.concatenate([v, np.full(r, v[-1], v.dtype)])


def run_mixed(a, dist: Dist):
    """Learned encoding + batched mixed workload: the MLP is trained on the GPU
    on exhaustively labelled vectors; 64 columns of uneven length and
    distribution are encoded with the learned picks and with the exhaustive
    encoder; 256 seeded filter-aggregate queries run as one CUDA-graph replay of
    the batch executor and as one launch per query."""
    import numpy as np
    import torch

    from fastlanesgpu_b200 import LAYOUT_TRANSPOSED, ORDER_ORIGINAL, EncodedColumn, datagen, ops
    from fastlanesgpu_b200.batch import Batch, graph_of
    from fastlanesgpu_b200.column import encode_column_gpu, encode_column_learned_gpu
    from fastlanesgpu_b200.selector import LearnedSelector, corpus_device, decode_aware_labels, gpu_features
    dev = torch.device("cuda", dist.local)
    stream = torch.cuda.current_stream()
    ops.set_tuning(1, a.jit)
    threads = os.cpu_count() or 1

    def now():
        torch.cuda.synchronize()
        return time.perf_counter()

    # ------------------------------------------------ train the selector
    t0 = now()
    train_dev = corpus_device(a.train_vectors, seed=7, device=dev)
    train_host = train_dev.cpu().numpy()
    t1 = now()
    tr_sizes, _ = ops.encode_exhaustive(train_host)
    labels = decode_aware_labels(tr_sizes, a.decode_kappa)
    t2 = now()
    sel = LearnedSelector(device=dev, seed=1)
    feats = gpu_features(train_dev)
    losses = sel.train(feats, torch.from_numpy(labels).to(dev), epochs=a.train_epochs, batch=4096, lr=3e-3)
    t3 = now()
    del train_dev, train_host, feats
    training = {"vectors": a.train_vectors, "epochs": a.train_epochs, "batch": 4096, "decode_kappa": a.decode_kappa,
                "corpus_gen_s": t1 - t0, "exhaustive_label_s": t2 - t1, "gpu_train_s": t3 - t2,
                "loss_first_epoch": losses[0], "loss_last_epoch": losses[-1]}

    # --------------------------------------------------- the 64 columns
    cols = datagen.mixed_columns(a.mixed_columns, 16, a.mixed_max_log, seed=64, device=dev)
    host = [_pad_vectors(v.cpu().numpy()) for _, v in cols]
    lens = [int(v.numel()) for _, v in cols]
    n_vec = [h.size // 1024 for h in host]
    rows_all = sum(lens)
    # exhaustive: exact size of every scheme of every vector, argmin, encode
    t0 = time.perf_counter()
    ex = [ops.encode_exhaustive(h, threads) for h in host]
    t1 = time.perf_counter()
    enc_ex = [EncodedColumn.encode(h[:n], best, layout=LAYOUT_TRANSPOSED) for h, n, (_, best) in zip(host, lens, ex)]
    t2 = time.perf_counter()
    ex_select_s, ex_encode_s = t1 - t0, t2 - t1
    # learned, on the GPU: upload the raw columns, statistics + MLP, the
    # exhaustive encoder only for low-confidence vectors, GPU encode.  Both
    # arms start from the raw columns in pinned host memory.
    cat_t = torch.empty(sum(h.size for h in host), dtype=torch.int32, pin_memory=True)
    cat = cat_t.numpy()
    np.concatenate(host, out=cat)
    vstart = np.concatenate([[0], np.cumsum(n_vec)])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    cat_dev = cat_t.to(dev, non_blocking=True)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    schemes_dev, info = sel.select_device(cat_dev, cat, threshold=a.threshold, kappa=a.decode_kappa)
    t2 = time.perf_counter()
    dcols = [encode_column_gpu(cat_dev[vstart[i] * 1024: vstart[i] * 1024 + lens[i]],
                               schemes_dev[vstart[i]: vstart[i + 1]].contiguous(), layout=LAYOUT_TRANSPOSED)
             for i in range(len(cols))]
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    ln_upload_s, ln_select_s, ln_encode_s = t1 - t0, t2 - t1, t3 - t2
    # the exhaustive picks encoded on the GPU as well (selection is then the
    # only difference between the arms)
    t0 = time.perf_counter()
    best_dev = torch.from_numpy(np.concatenate([b for _, b in ex])).to(dev)
    ex_gpu = [encode_column_gpu(cat_dev[vstart[i] * 1024: vstart[i] * 1024 + lens[i]],
                                best_dev[vstart[i]: vstart[i + 1]].contiguous(), layout=LAYOUT_TRANSPOSED)
              for i in range(len(cols))]
    torch.cuda.synchronize()
    ex_gpu_encode_s = time.perf_counter() - t0 + ln_upload_s
    # the whole learned encoder as one device call per column
    # (fls_encode_learned_gpu: statistics, MLP, exhaustive choice on the device
    # for low-confidence vectors, encode), and the same call with every vector
    # sent to the device's exhaustive choice
    enc_streams = [torch.cuda.Stream() for _ in range(4)]

    def one_call(threshold):
        # every column's call enqueued back to back, round robin over four
        # streams so that small columns run beside large ones; the encoders'
        # info words are read once all have run (no host round trip per column)
        torch.cuda.synchronize()
        t0_ = time.perf_counter()
        pend = []
        for i in range(len(cols)):
            with torch.cuda.stream(enc_streams[i % len(enc_streams)]):
                pend.append(encode_column_learned_gpu(cat_dev[vstart[i] * 1024: vstart[i] * 1024 + lens[i]],
                                                      sel.params, threshold=threshold, kappa=a.decode_kappa,
                                                      layout=LAYOUT_TRANSPOSED, compact=False, defer=True))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0_
        return [p.finish() for p in pend], dt
    one_call(a.threshold)  # first use of the select kernel on this device
    # median of three timed passes of each (a single host-timed pass is
    # noisy); the first pass's columns are kept
    def timed3(threshold):
        cols_, t_ = one_call(threshold)
        ts = [t_] + [one_call(threshold)[1] for _ in range(2)]
        return cols_, float(np.median(ts))
    ln1, ln1_s = timed3(a.threshold)
    exd, exd_s = timed3(2.0)
    one_call_same = bool(torch.equal(torch.cat([sc for _, sc, _ in ln1]), schemes_dev))
    size_ln1 = sum(c.nbytes for c, _, _ in ln1)
    size_exd = sum(c.nbytes for c, _, _ in exd)
    del ln1, exd
    size_ex = sum(c.nbytes for c in enc_ex)
    size_ex_gpu = sum(c.nbytes for c in ex_gpu)
    size_ln = sum(c.nbytes for c in dcols)
    size_for = sum(int(sz[:, 0].astype(np.int64).sum()) for sz, _ in ex)  # bit-packing only
    schemes_ln = schemes_dev.cpu().numpy()
    del cat, cat_t, cat_dev, best_dev

    # lossless: decode every learned column on the GPU and compare
    lossless = all(torch.equal(ops.unpack_global(dc, order=ORDER_ORIGINAL)[:n], v)
                   for dc, n, (_, v) in zip(dcols, lens, cols))

    # ----------------------------------------------- 256 seeded queries
    g = np.random.default_rng(256)
    queries = []
    for q in range(a.queries):
        c = q % len(cols)
        smp = host[c][: lens[c]: 97] if lens[c] > 97 * 64 else host[c][: lens[c]]
        lo_q, hi_q = np.sort(g.random(2))
        lo, hi = (int(x) for x in np.quantile(smp, [lo_q, hi_q]))
        queries.append((c, lo, hi, c))
    want = []
    for c, lo, hi, _ in queries:  # plain torch on the raw columns
        v = cols[c][1].to(torch.int64)
        m = (v >= lo) & (v <= hi)
        want.append((int(v[m].sum()), int(m.sum())))
    batch = Batch(dcols, queries)
    graph = graph_of(batch.run)
    res = batch.results.view(-1, 2)

    def per_query():
        return [ops.query_filter_agg([dcols[c]], [(0, lo, hi)], agg_a=0) for c, lo, hi, _ in queries]

    pq = [int(x.cpu()[0]) for x in per_query()]
    graph.replay()
    torch.cuda.synchronize()
    got = [(int(s_), int(n_)) for s_, n_ in res.cpu().tolist()]
    exact = got == want and pq == [w[0] for w in want]

    def timed(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    # kernels per batch: what one fls_batch_run enqueues (the graph replays it)
    l0 = ops.kernel_launch_count()
    batch.run()
    per_run = ops.kernel_launch_count() - l0
    clocks = ClockSampler(dist.local)
    clocks.start()
    w0 = time.time()
    batch_ms = timed(graph.replay, a.steps)
    w1 = time.time()
    launches = per_run * a.steps
    clocks.mark(w0, w1)
    per_query_ms = timed(per_query, max(3, a.steps // 10))
    # the same queries over the exhaustive encoder's columns (decode cost of
    # the two encodings)
    batch_ex = Batch(ex_gpu, queries)
    graph_ex = graph_of(batch_ex.run)
    graph_ex.replay()
    torch.cuda.synchronize()
    exact = exact and [(int(s_), int(n_)) for s_, n_ in batch_ex.results.view(-1, 2).cpu().tolist()] == want
    batch_ex_ms = timed(graph_ex.replay, max(3, a.steps // 5))
    del graph_ex, batch_ex
    # end to end: encoded columns H2D, the batch, results D2H
    copies = []
    for dc in dcols:
        copies.append((dc.data, dc.data.cpu().pin_memory()))
        copies.append((dc.meta, dc.meta.cpu().pin_memory()))
    host_res = torch.empty(res.numel(), dtype=torch.int64).pin_memory()

    def e2e():
        for dst, hp in copies:
            dst.copy_(hp.view(dst.dtype).view(dst.shape), non_blocking=True)
        graph.replay()
        host_res.copy_(batch.results, non_blocking=True)
    e2e_ms = timed(e2e, 3)
    clk = clocks.stop()

    q_rows = sum(lens[c] for c, _, _, _ in queries)
    q_bytes = sum(dcols[c].nbytes for c, _, _, _ in queries)
    peak, peak_src = measured_peak_gbs()
    achieved = q_bytes / (batch_ms / 1e3) / 1e9
    return {
        "metric": "fused decode+query rows/s", "value": q_rows / (batch_ms / 1e3), "unit": "rows/s",
        "n_gpus": dist.world, "steps": a.steps, "warmup": 3, "ms_per_step": batch_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32->int64", "data": "synthetic (seeded)",
        "config": {"workload": f"mixed: {len(cols)} columns (lengths 2^16..2^{a.mixed_max_log}; uniform, Zipf 1.1, "
                               f"sorted gaps, geometric runs), learned encoding, {len(queries)} filter-aggregate "
                               "queries in one CUDA-graph batch launch",
                   "rows_in_columns": rows_all, "rows_scanned_per_step": q_rows,
                   "l2": "columns larger than L2 (126 MB) in total, no flush", "parallelism": "1 GPU"},
        "learned_encoding": {
            "bytes_exhaustive": size_ex, "bytes_learned": size_ln, "bytes_bitpack_only": size_for,
            "bytes_exhaustive_gpu_encoder": size_ex_gpu,
            "regret": size_ln / size_ex - 1.0,
            "scheme_counts_learned": np.bincount(schemes_ln, minlength=5).tolist(),
            "scheme_counts_exhaustive": np.bincount(np.concatenate([b for _, b in ex]), minlength=5).tolist(),
            "exhaustive": {"where": f"host, {threads} threads", "select_s": ex_select_s, "encode_s": ex_encode_s,
                           "total_s": ex_select_s + ex_encode_s},
            "learned": {"where": "GPU (upload, statistics, MLP, encode) + host exhaustive fallback",
                        "upload_s": ln_upload_s, "select_s": ln_select_s, "encode_s": ln_encode_s,
                        "total_s": ln_upload_s + ln_select_s + ln_encode_s,
                        "parts_s": {k: v for k, v in info.items() if k.endswith("_s")}},
            "exhaustive_select_then_gpu_encode_s": ex_select_s + ex_gpu_encode_s,
            "device_one_call": {"where": "fls_encode_learned_gpu per column, columns already on the GPU, "
                                         "round robin over 4 streams",
                                "learned_s": ln1_s, "bytes_learned": size_ln1,
                                "same_schemes_as_select_device": one_call_same,
                                "exhaustive_on_device_s": exd_s, "bytes_exhaustive_on_device": size_exd},
            "encode_speedup": (ex_select_s + ex_encode_s) / (ln_upload_s + ln_select_s + ln_encode_s),
            "select_speedup": ex_select_s / (ln_upload_s + ln_select_s),
            "fallback_vectors": info["fallback_vectors"], "vectors": info["vectors"], "threshold": a.threshold,
            "lossless": bool(lossless), "training": training},
        "batched": {"ms_batch_graph": batch_ms, "ms_per_query_launches": per_query_ms,
                    "ms_batch_graph_exhaustive_encoding": batch_ex_ms,
                    "speedup": per_query_ms / batch_ms, "queries": len(queries), "work_items": batch.n_items,
                    "results_equal": bool(exact)},
        "e2e": {"value": q_rows / (e2e_ms / 1e3), "unit": "rows/s",
                "h2d_bytes_per_step": sum(hp.numel() * hp.element_size() for _, hp in copies),
                "d2h_bytes_per_step": host_res.numel() * 8, "ms_per_step": e2e_ms,
                "path": "pinned host encoded columns -> H2D -> batch graph (C ABI) -> D2H results"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured"
                     else "fallback 6650 GB/s", "traffic": None, "algorithmic_bytes_per_launch": q_bytes},
        "gpu_launches": int(launches),
        "clocks": clk,
    }


def run_reference(a, dist: Dist):
    """--impl reference: the reference's own CPU implementation of the path
    (its unpack compiled from its sources, its fls_q11.cu / fls_q21.cu /
    fls_q31.cu / fls_q41.cu scalar loops) on the host cores, with every usable
    thread, over the same workload at full size: --warmup untimed and --steps
    timed passes over the whole table (the timed passes stop early only if
    they would exceed about two minutes; `steps` then says how many ran)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from fastlanesgpu_b200 import datagen
    from fastlanesgpu_b200.shard import shard_seed
    R = orc.Reference()
    info = cpu_info()
    threads = info["usable_cpus"]
    if a.workload in ("mixed", "ssb", "ssb-real") or (a.workload == "decode" and (a.decode_scheme != "for" or
                                                                        a.decode_width != 32)):
        return {"impl": "reference", "unavailable": "the reference has no CPU implementation of this workload "
                "(learned selection, batching, per-vector DELTA/RLE/DICT columns, 8/16/64-bit lanes (it only "
                "packs them), or the SSB queries other than its fls_q11/q21/q31/q41 loops)"}
    n = a.rows
    seed = shard_seed(1000, 0)  # the table the GPU arm benches on rank 0
    tabs, bws, decode_bw = None, None, a.decode_bw
    if a.workload == "q11":
        t = datagen.lineorder_q11(n, seed=seed)
        names, bits = ["date", "discount", "quantity", "price"], datagen.Q11_BITS
        what = "fused decode + filter-aggregate (Q1.1 shape)"
    elif a.workload in ("q21", "q31", "q41"):
        O = orc.Oracle()
        if a.workload == "q21":
            t = datagen.q21_tables(n, seed=seed)
            tabs = {"ht_s": O.pht1_build(t["s_region"], 1, t["s_suppkey"], t["s_suppkey"].size),
                    "ht_p": O.pht2_build(t["p_category"], 1, t["p_partkey"], t["p_brand1"], t["p_partkey"].size),
                    "ht_d": O.pht2_build(None, 0, t["d_datekey"], t["d_year"], datagen.N_DAYS)}
            names, bits = ["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"], datagen.Q21_BITS
            what = "fused decode + 3-way perfect-hash probe + 7000-group int64 group-by (Q2.1 shape)"
        elif a.workload == "q31":
            t = datagen.q31_tables(n, seed=seed)
            tabs = {"ht_s": O.pht2_build(t["s_region"], 1, t["s_suppkey"], t["s_nation"], t["s_suppkey"].size),
                    "ht_c": O.pht2_build(t["c_region"], 1, t["c_custkey"], t["c_nation"], t["c_custkey"].size),
                    "ht_d": O.pht2_build(t["d_in_range"], 1, t["d_datekey"], t["d_year"], datagen.N_DAYS)}
            names, bits = ["lo_suppkey", "lo_custkey", "lo_orderdate", "lo_revenue"], datagen.Q31_BITS
            what = "fused decode + perfect-hash probes + int64 group-by (Q3.1 shape)"
        else:
            t = datagen.q41_tables(n, seed=seed)
            tabs = {"ht_s": O.pht1_build(t["s_region"], 1, t["s_suppkey"], t["s_suppkey"].size),
                    "ht_c": O.pht2_build(t["c_region"], 1, t["c_custkey"], t["c_nation"], t["c_custkey"].size),
                    "ht_p": O.pht1_build(t["p_mfgr_low"], 1, t["p_partkey"], t["p_partkey"].size),
                    "ht_d": O.pht2_build(None, 0, t["d_datekey"], t["d_year"], datagen.N_DAYS)}
            names = ["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue", "lo_supplycost"]
            bits = datagen.Q41_BITS
            what = "fused decode + perfect-hash probes + int64 group-by (Q4.1 shape)"
    else:
        t = {"v": datagen.uniform_bits(n, a.decode_bw, seed=seed)}
        names, bits = ["v"], {"v": a.decode_bw}
        what = f"decode fused with uint64 sum: bit-pack + FOR, bw {a.decode_bw}"
    # the reference's own packer (pack.cpp) encodes the columns
    words = [R.pack_column(t[k], bits[k], threads) for k in names]
    bws = [bits[k] for k in names]
    del t
    fn, args = reference_call(R, a.workload, words, bws, n, tabs, threads, decode_bw)
    for _ in range(a.warmup):
        fn(*args)
    times = []
    budget = 120.0
    for i in range(a.steps):
        t0 = time.perf_counter()
        fn(*args)
        times.append(time.perf_counter() - t0)
        if sum(times) / (i + 1) * a.steps > budget and sum(times) > budget:
            break
    ms = 1e3 * sum(times) / len(times)
    value = n / (ms / 1e3)
    n1 = min(n, 1 << 22)
    fn1, args1 = reference_call(R, a.workload, words, bws, n1, tabs, 1, decode_bw)
    med1, reps1, _ = _time_cpu(fn1, args1, 3.0, min_reps=1)
    return {
        "impl": "reference", "metric": "fused decode+query rows/s", "value": value, "unit": "rows/s",
        "n_gpus": a.gpus, "steps": len(times), "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32->int64", "data": "synthetic (seeded)",
        "config": {"workload": what, "rows_per_gpu": n, "rows_per_step": n},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "reference", "cpu": info,
                         "sample": f"the whole table ({n} rows) per step, {len(times)} timed steps after "
                                   f"{a.warmup} untimed, mean; {REF_HOW[a.workload]}, OpenMP {threads} threads",
                         "single_thread": {"value": n1 / med1, "unit": "rows/s", "cores": 1,
                                           "sample": f"first {n1} rows, {reps1} runs, median, 1 thread"}},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def _time_gpu(fn, steps: int, warmup: int = 3) -> float:
    """Milliseconds per call of fn: CUDA events on the current stream around
    `steps` calls, after `warmup` untimed ones (inputs larger than L2)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def secondary_joins(a, dist, steps: int) -> dict:
    """Q2.1, Q3.1 and Q4.1 (2^27 rows each) through the same path as the
    headline, each checked against the reference's CPU implementation on the
    whole table, with the median SM clock of its timed region."""
    import argparse as _ap

    import torch
    out = {}
    for w in ("q21", "q31", "q41"):
        b = _ap.Namespace(**vars(a))
        b.workload, b.steps, b.e2e_steps, b.rows = w, steps, 3, a.rows
        line, ctx = run_ours(b, dist)
        cb = cpu_baseline(b, ctx, 2.0)
        clk = line["clocks"]
        ms = line["ms_per_step"]
        ent = {"workload": line["config"]["workload"], "rows": b.rows, "steps": steps, "ms_per_step": ms,
               "rows_per_s": line["value"],
               "roofline": {k: line["roofline"][k] for k in ("achieved", "frac", "algorithmic_bytes_per_launch",
                                                             "traffic")},
               "clocks": clk, "join_variants": line["config"].get("join_variants"),
               "e2e_rows_per_s": line["e2e"]["value"],
               "cpu_baseline": {k: cb[k] for k in ("value", "cores", "single_thread")},
               "result_equal": cb["result_equal"]}
        if clk.get("sm_mhz") and clk.get("sm_max_mhz"):
            ent["ms_x_sm_mhz"] = ms * clk["sm_mhz"]
            ent["ms_at_max_sm_clock"] = ms * clk["sm_mhz"] / clk["sm_max_mhz"]
        out[w] = ent
        del ctx, line
        torch.cuda.empty_cache()
    return out


def decode_sweep(a, dist, steps: int) -> dict:
    """Uniform FOR bit-packed columns of 2^28 values at every bit width 1..32,
    decoded to HBM and fused with a uint64 sum.  Values uniform in [0, 2^bw)
    pack to uniformly random words (every bit of a packed vector belongs to
    exactly one value), so the packed words are drawn directly on the device.
    Checks per width: the fused sum equals the sum of the decoded array and the
    reference's own unpack + sum over the whole column on the host (which is
    also timed, all threads), and three vectors decode element-wise as the
    reference's unpack decodes them."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as orc
    import torch

    from fastlanesgpu_b200 import ops
    from fastlanesgpu_b200.column import DeviceUniformColumn
    R = orc.Reference()
    threads = cpu_info()["usable_cpus"]
    dev = torch.device("cuda", dist.local)
    n = 1 << 28
    n_vec = n // 1024
    peak = measured_peak_gbs()[0]
    g = torch.Generator(device=dev)
    g.manual_seed(2800)
    dec = torch.empty(n, dtype=torch.int32, device=dev)
    s = torch.zeros(1, dtype=torch.int64, device=dev)
    clocks = ClockSampler(dist.local)
    clocks.start()
    w0 = time.time()
    per_bw, ok = {}, True
    for bw in range(1, 33):
        words = torch.randint(0, 256, (4 * n_vec * 32 * bw,), dtype=torch.uint8, device=dev,
                              generator=g).view(torch.int32)
        col = DeviceUniformColumn(words, n, bw)
        ms_sum = _time_gpu(lambda: ops.query_aggregate(col, out=s), steps, max(3, a.warmup))
        ms_hbm = _time_gpu(lambda: ops.unpack_global(col, out=dec), steps, max(3, a.warmup))
        got_sum = int(s.cpu()[0]) & M64
        dec_sum = int((dec.to(torch.int64) & 0xFFFFFFFF).sum()) & M64
        host = words.cpu().numpy().view(np.uint32)
        t0 = time.perf_counter()
        ref_sum = R.decode_sum(host, bw, n_vec, threads) & M64
        ref_s = time.perf_counter() - t0
        vec_ok = all(np.array_equal(dec[v * 1024:(v + 1) * 1024].cpu().numpy().view(np.uint32),
                                    R.unpack(host[v * 32 * bw:(v + 1) * 32 * bw], bw).view(np.uint32))
                     for v in (0, n_vec // 2, n_vec - 1))
        equal = got_sum == dec_sum == ref_sum and vec_ok
        ok = ok and equal
        b_in = n_vec * 128 * bw
        per_bw[bw] = {"sum_ms": ms_sum, "sum_frac": b_in / (ms_sum / 1e3) / 1e9 / peak,
                      "sum_values_per_s": n / (ms_sum / 1e3),
                      "hbm_ms": ms_hbm, "hbm_frac": (b_in + 4 * n) / (ms_hbm / 1e3) / 1e9 / peak,
                      "cpu_reference_values_per_s": n / ref_s, "result_equal": equal}
        del words, col, host
    clocks.mark(w0, time.time())
    clk = clocks.stop()
    del dec
    torch.cuda.empty_cache()
    return {"workload": "decode of a uniform FOR bit-packed column of 2^28 values at bit widths 1..32, to HBM "
                        "(algorithmic bytes 128*bw per vector + 4 B per value written) and fused with a uint64 sum "
                        "(128*bw per vector)", "steps": steps, "peak_gbs": peak, "clocks": clk,
            "cpu_reference": f"{REF_HOW['decode']}, OpenMP {threads} threads, one pass over the whole column",
            "all_equal": ok, "per_bw": per_bw}


def decode_schemes(a, dist, steps: int) -> dict:
    """DELTA (sorted keys, geometric gaps p=0.3), RLE (geometric runs of mean
    16, values in [0, 2^16)) and DICT (Zipf 1.1 over [0, 2^20)) columns of 2^28
    values, generated and encoded on the GPU (per-vector metadata), and the
    same runs in the reference's tile-based RLE format (RFOR, host-encoded),
    decoded to HBM (stored order) and fused with a uint64 sum; checked by
    decoding in original order against the input values and by the input's
    sum."""
    import torch

    from fastlanesgpu_b200 import LAYOUT_TRANSPOSED, ORDER_ORIGINAL, SCHEME_DELTA, SCHEME_DICT, SCHEME_RLE, datagen, ops
    from fastlanesgpu_b200.column import encode_column_gpu
    dev = torch.device("cuda", dist.local)
    n = 1 << 28
    peak = measured_peak_gbs()[0]
    out = {}
    from fastlanesgpu_b200.column import RforColumn
    for name, scheme, gen in (
            ("delta", SCHEME_DELTA, lambda: datagen.sorted_geometric_device(n, 0.3, seed=2801, device=dev)),
            ("rle", SCHEME_RLE, lambda: datagen.geometric_runs_device(n, 16.0, 16, seed=2802, device=dev)),
            ("dict", SCHEME_DICT, lambda: datagen.zipf_device(n, s=1.1, domain=1 << 20, seed=2803, device=dev)),
            ("rfor", None, lambda: datagen.geometric_runs_device(n, 16.0, 16, seed=2804, device=dev))):
        vals = gen()
        s = torch.zeros(1, dtype=torch.int64, device=dev)
        if scheme is None:
            # the reference's tile-based RLE (tile_based/src/rlebinpack.cpp), encoded on the host
            col = RforColumn.encode(vals.cpu().numpy()).to_device(dev)
            dec = torch.empty(n, dtype=torch.int32, device=dev)
            sum_fn, hbm_fn = (lambda: ops.rfor_decode_sum(col, out=s)), (lambda: ops.rfor_decode(col, out=dec))
        else:
            col = encode_column_gpu(vals, scheme, layout=LAYOUT_TRANSPOSED)
            dec = torch.empty(col.n_vec * 1024, dtype=torch.int32, device=dev)
            sum_fn, hbm_fn = (lambda: ops.query_aggregate(col, out=s)), (lambda: ops.unpack_global(col, out=dec))
        ms_sum = _time_gpu(sum_fn, steps, max(3, a.warmup))
        ms_hbm = _time_gpu(hbm_fn, steps, max(3, a.warmup))
        want = int((vals.to(torch.int64) & 0xFFFFFFFF).sum()) & M64
        equal = (int(s.cpu()[0]) & M64) == want
        if scheme is None:
            ops.rfor_decode(col, out=dec)
        else:
            ops.unpack_global(col, order=ORDER_ORIGINAL, out=dec)
        equal = equal and bool(torch.equal(dec[:n], vals))
        ops.check_device_error()
        b = col.nbytes
        out[name] = {"encoded_bytes": b, "bits_per_value": 8 * b / n, "sum_ms": ms_sum,
                     "sum_frac": b / (ms_sum / 1e3) / 1e9 / peak, "sum_values_per_s": n / (ms_sum / 1e3),
                     "hbm_ms": ms_hbm, "hbm_frac": (b + 4 * n) / (ms_hbm / 1e3) / 1e9 / peak,
                     "result_equal": equal}
        del vals, col, dec
        torch.cuda.empty_cache()
    return out


def mixed_summary(a, dist) -> dict:
    """The learned-encoding + batched workload (64 mixed columns, MLP trained on
    the GPU, 256 batched filter-aggregate queries), condensed."""
    import argparse as _ap
    b = _ap.Namespace(**vars(a))
    b.steps = max(20, min(a.steps, 200))
    m = run_mixed(b, dist)
    le, bt = m["learned_encoding"], m["batched"]
    dc = le["device_one_call"]
    return {"workload": m["config"]["workload"], "rows_scanned_per_step": m["config"]["rows_scanned_per_step"],
            "batch_rows_per_s": m["value"], "batch_roofline_frac": m["roofline"]["frac"],
            "bytes_exhaustive": le["bytes_exhaustive"], "bytes_learned": le["bytes_learned"], "regret": le["regret"],
            "host_exhaustive_s": le["exhaustive"]["total_s"], "host_exhaustive_where": le["exhaustive"]["where"],
            "learned_gpu_pipeline_s": le["learned"]["total_s"],
            "learned_vs_host_exhaustive": le["encode_speedup"],
            "device_learned_s": dc["learned_s"], "device_exhaustive_s": dc["exhaustive_on_device_s"],
            "learned_vs_device_exhaustive": dc["exhaustive_on_device_s"] / dc["learned_s"],
            "bytes_device_learned": dc["bytes_learned"], "bytes_device_exhaustive": dc["bytes_exhaustive_on_device"],
            "fallback_vectors": le["fallback_vectors"], "vectors": le["vectors"], "lossless": le["lossless"],
            "batch_ms": bt["ms_batch_graph"], "per_query_launches_ms": bt["ms_per_query_launches"],
            "batch_speedup": bt["speedup"], "results_equal": bt["results_equal"], "clocks": m["clocks"]}


def main():
    a = parse_args()
    dist = Dist()
    if a.impl == "reference":
        if dist.rank == 0:
            print(json.dumps(run_reference(a, dist)), flush=True)
        return
    dist.init()
    failed = False
    try:
        if a.workload in ("mixed", "ssb-real") and dist.world > 1:
            raise SystemExit(f"--workload {a.workload} runs on one GPU")
        if a.workload == "mixed":
            print(json.dumps(run_mixed(a, dist)), flush=True)
            return
        out, ctx = run_ours(a, dist)
        checkable = a.workload in ("q11", "q21", "q31", "q41") or (
            a.workload == "decode" and a.decode_scheme == "for" and a.decode_width == 32 and a.decode_out == "sum")
        if dist.rank == 0 and dist.world == 1 and checkable and not a.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(a, ctx, a.cpu_seconds)
            out["result_check"] = {"against": "the reference's CPU implementation on the whole benched table "
                                              "(cpu_baseline leg)", "equal": out["cpu_baseline"]["result_equal"]}
            failed = not out["result_check"]["equal"]
        if "reference_answers" in out:
            failed = failed or not out["reference_answers"]["equal"]
        del ctx
        if dist.world == 1 and a.workload == "q11" and a.secondary == "all" and not failed:
            sec = {"note": "other configurations, each timed with CUDA events after warm-up; inputs larger than L2"}
            sec_steps = max(a.steps, 200)
            sec.update(secondary_joins(a, dist, max(a.steps, 1000)))
            sec["decode_for_2p28"] = decode_sweep(a, dist, sec_steps)
            sec["decode_schemes_2p28"] = decode_schemes(a, dist, sec_steps)
            sec["mixed"] = mixed_summary(a, dist)
            out["secondary"] = sec
            failed = not (all(sec[w]["result_equal"] for w in ("q21", "q31", "q41")) and
                          sec["decode_for_2p28"]["all_equal"] and
                          all(v["result_equal"] for v in sec["decode_schemes_2p28"].values()) and
                          sec["mixed"]["results_equal"] and sec["mixed"]["lossless"])
        if dist.rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        dist.close()
    if failed:
        raise SystemExit("bench: a result differs from the reference's (see result_check / secondary)")


if __name__ == "__main__":
    main()
