"""Seeded synthetic inputs with the shapes, sizes and value distributions of the
workloads the reference measures, and the Star Schema Benchmark queries on
them and on SSB's own data (dbgen's tables, loaded in the reference loader's
integer encoding).  All generators use numpy's PCG64 with an explicit seed.
"""
from __future__ import annotations

import os

import numpy as np

# Day ids 0..2555 cover 1992-01-01 .. 1998-12-30 (the SSB date dimension);
# first day id of each year 1992..1998 and one past the end.
YEAR_START = np.array([0, 366, 731, 1096, 1461, 1827, 2192, 2556], dtype=np.int32)
N_DAYS = 2556


def year_of_day(day: np.ndarray) -> np.ndarray:
    return (1992 + np.searchsorted(YEAR_START, day, side="right") - 1).astype(np.int32)


def rng(seed: int) -> np.random.Generator:
    return np.random.default_rng(seed)


def for_bitpack_mixed(n: int, seed: int = 1, widths=(3, 7, 11, 16, 21)) -> np.ndarray:
    """Per 1024-value vector a seeded width w from `widths`, base U[0,2^20),
    values base + U[0,2^w)."""
    g = rng(seed)
    nv = (n + 1023) // 1024
    w = g.choice(np.asarray(widths), size=nv)
    base = g.integers(0, 1 << 20, size=nv)
    off = (g.integers(0, 1 << 32, size=(nv, 1024), dtype=np.uint64) & ((np.uint64(1) << w.astype(np.uint64)[:, None])
                                                                       - np.uint64(1))).astype(np.int64)
    return (base[:, None] + off).reshape(-1)[:n].astype(np.int32)


def uniform_bits(n: int, bw: int, seed: int = 2) -> np.ndarray:
    """Uniform values in [0, 2^bw) (bw 32 uses the full uint32 range)."""
    g = rng(seed)
    x = g.integers(0, 1 << 32, size=n, dtype=np.uint64)
    if bw < 32:
        x &= np.uint64((1 << bw) - 1)
    return x.astype(np.uint32).view(np.int32)


def sorted_geometric(n: int, p: float = 0.3, seed: int = 3) -> np.ndarray:
    """Sorted keys with geometric(p) gaps (delta workload)."""
    g = rng(seed)
    return np.cumsum(g.geometric(p, size=n), dtype=np.int64).astype(np.int32)


def geometric_runs(n: int, mean_run: float = 16.0, value_bits: int = 16, seed: int = 4) -> np.ndarray:
    """Runs with geometric lengths (mean `mean_run`) of uniform values in [0, 2^value_bits)."""
    g = rng(seed)
    n_runs = int(n / mean_run * 1.2) + 16
    lens = g.geometric(1.0 / mean_run, size=n_runs)
    while lens.sum() < n:
        lens = np.concatenate([lens, g.geometric(1.0 / mean_run, size=n_runs)])
    vals = g.integers(0, 1 << value_bits, size=lens.size)
    return np.repeat(vals, lens)[:n].astype(np.int32)


def zipf_values(n: int, s: float = 1.1, domain: int = 1 << 20, seed: int = 5) -> np.ndarray:
    """Zipf(s) ranks folded into [0, domain)."""
    g = rng(seed)
    z = g.zipf(s, size=n)
    return ((z - 1) % domain).astype(np.int32)


def lineorder_q11(n: int, seed: int = 11) -> dict:
    """Fact table of the filter-aggregate workload: date day id U[0,2556)
    (12 bit), discount U[0,10] (4 bit), quantity U[1,50] (6 bit), price
    U[90000,10.5M] (24 bit)."""
    g = rng(seed)
    return {
        "date": g.integers(0, N_DAYS, size=n).astype(np.int32),
        "discount": g.integers(0, 11, size=n).astype(np.int32),
        "quantity": g.integers(1, 51, size=n).astype(np.int32),
        "price": g.integers(90000, 10_500_001, size=n).astype(np.int32),
    }


# Q1.1-shape predicate on the synthetic table: year 1993, discount in [1,3],
# quantity < 25 (fls_q11.cu:20-26 on SSB), ~1/7 * 3/11 * 24/50 = 1.87 %.
Q11_FILTER = {"date": (int(YEAR_START[1]), int(YEAR_START[2]) - 1), "discount": (1, 3), "quantity": (-2**31, 24)}
Q11_BITS = {"date": 12, "discount": 4, "quantity": 6, "price": 24}


def q21_tables(n: int, seed: int = 21, part_ids: int = 1 << 19, supp_ids: int = 1 << 17) -> dict:
    """Join workload: fact foreign keys (part 19 bit, supplier 17 bit, date
    12 bit, revenue 24 bit) and uniform dimension attributes; part filter
    category == 1 of 5, supplier filter region == 1 of 25, brand in [0,1000)."""
    g = rng(seed)
    return {
        "lo_partkey": g.integers(0, part_ids, size=n).astype(np.int32),
        "lo_suppkey": g.integers(0, supp_ids, size=n).astype(np.int32),
        "lo_orderdate": g.integers(0, N_DAYS, size=n).astype(np.int32),
        "lo_revenue": g.integers(90000, 10_500_001, size=n).astype(np.int32),
        "p_partkey": np.arange(part_ids, dtype=np.int32),
        "p_category": g.integers(0, 5, size=part_ids).astype(np.int32),
        "p_brand1": g.integers(0, 1000, size=part_ids).astype(np.int32),
        "s_suppkey": np.arange(supp_ids, dtype=np.int32),
        "s_region": g.integers(0, 25, size=supp_ids).astype(np.int32),
        "d_datekey": np.arange(N_DAYS, dtype=np.int32),
        "d_year": year_of_day(np.arange(N_DAYS)),
    }


Q21_BITS = {"lo_suppkey": 17, "lo_partkey": 19, "lo_orderdate": 12, "lo_revenue": 24}


def q31_tables(n: int, seed: int = 31, cust_ids: int = 1 << 18, supp_ids: int = 1 << 17) -> dict:
    """Q3.1-shape join workload: fact foreign keys customer (18 bit), supplier
    (17 bit), date (12 bit) and revenue (24 bit); dimension nations U[0,25)
    with region = nation // 5; customer and supplier filtered on region 1
    (1/5 each), dates on years 1992..1997."""
    g = rng(seed)
    c_nation = g.integers(0, 25, size=cust_ids).astype(np.int32)
    s_nation = g.integers(0, 25, size=supp_ids).astype(np.int32)
    d_year = year_of_day(np.arange(N_DAYS))
    return {
        "lo_custkey": g.integers(0, cust_ids, size=n).astype(np.int32),
        "lo_suppkey": g.integers(0, supp_ids, size=n).astype(np.int32),
        "lo_orderdate": g.integers(0, N_DAYS, size=n).astype(np.int32),
        "lo_revenue": g.integers(90000, 10_500_001, size=n).astype(np.int32),
        "c_custkey": np.arange(cust_ids, dtype=np.int32), "c_nation": c_nation,
        "c_region": (c_nation // 5).astype(np.int32),
        "s_suppkey": np.arange(supp_ids, dtype=np.int32), "s_nation": s_nation,
        "s_region": (s_nation // 5).astype(np.int32),
        "d_datekey": np.arange(N_DAYS, dtype=np.int32), "d_year": d_year,
        "d_in_range": ((d_year >= 1992) & (d_year <= 1997)).astype(np.int32),
    }


Q31_BITS = {"lo_suppkey": 17, "lo_custkey": 18, "lo_orderdate": 12, "lo_revenue": 24}
Q31_GROUPS = 7 * 25 * 25


def q41_tables(n: int, seed: int = 41, cust_ids: int = 1 << 18, supp_ids: int = 1 << 17,
               part_ids: int = 1 << 19) -> dict:
    """Q4.1-shape join workload: fact foreign keys supplier, customer, part
    (19 bit), date; revenue (24 bit) and supply cost U[50000, 150000) (18 bit);
    supplier and customer on region 1, part manufacturer in {0, 1} of 5 (2/5),
    every date."""
    g = rng(seed)
    c_nation = g.integers(0, 25, size=cust_ids).astype(np.int32)
    s_nation = g.integers(0, 25, size=supp_ids).astype(np.int32)
    p_mfgr = g.integers(0, 5, size=part_ids).astype(np.int32)
    return {
        "lo_suppkey": g.integers(0, supp_ids, size=n).astype(np.int32),
        "lo_custkey": g.integers(0, cust_ids, size=n).astype(np.int32),
        "lo_partkey": g.integers(0, part_ids, size=n).astype(np.int32),
        "lo_orderdate": g.integers(0, N_DAYS, size=n).astype(np.int32),
        "lo_revenue": g.integers(90000, 10_500_001, size=n).astype(np.int32),
        "lo_supplycost": g.integers(50000, 150000, size=n).astype(np.int32),
        "c_custkey": np.arange(cust_ids, dtype=np.int32), "c_nation": c_nation,
        "c_region": (c_nation // 5).astype(np.int32),
        "s_suppkey": np.arange(supp_ids, dtype=np.int32), "s_region": (s_nation // 5).astype(np.int32),
        "p_partkey": np.arange(part_ids, dtype=np.int32), "p_mfgr_low": (p_mfgr < 2).astype(np.int32),
        "d_datekey": np.arange(N_DAYS, dtype=np.int32), "d_year": year_of_day(np.arange(N_DAYS)),
    }


Q41_BITS = {"lo_suppkey": 17, "lo_custkey": 18, "lo_partkey": 19, "lo_orderdate": 12, "lo_revenue": 24,
            "lo_supplycost": 18}
Q41_GROUPS = 7 * 25
N_GROUPS = (1998 - 1992 + 1) * (5 * 5 * 40)


MIXED_FAMILIES = ("uniform", "zipf", "sorted_gaps", "geometric_runs")


def zipf_device(n: int, s: float = 1.1, domain: int = 1 << 20, seed: int = 5, device="cpu"):
    """Zipf(s) ranks truncated to [1, domain], minus 1 (values in [0, domain)),
    drawn by inverse CDF with torch on `device` (int32 tensor)."""
    import torch
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    cdf = torch.cumsum(torch.arange(1, domain + 1, dtype=torch.float64, device=dev) ** -s, 0)
    cdf /= cdf[-1].clone()
    v = torch.searchsorted(cdf, torch.rand(n, generator=g, device=dev, dtype=torch.float64))
    return torch.clamp(v, max=domain - 1).to(torch.int32)


def mixed_columns(n_cols: int = 64, lo_log: int = 16, hi_log: int = 26, seed: int = 64, device="cpu"):
    """Columns of the mixed workload, generated with torch on `device`:
    lengths log-uniform in [2^lo_log, 2^hi_log]; family i % 4 of
    MIXED_FAMILIES: uniform in [0, 2^w) with w in {8, 12, 16, 20}; Zipf s=1.1
    over [0, 2^20) (ranks truncated to 2^20, rank 1 -> 0); sorted keys with
    geometric gaps (p=0.3); runs of geometric length (mean 16) of values in
    [0, 2^16).  Returns [(family, int32 tensor)]."""
    import torch
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    lens = rng(seed)
    k = torch.arange(1, (1 << 20) + 1, dtype=torch.float64, device=dev) ** -1.1
    zcdf = torch.cumsum(k, 0)
    zcdf /= zcdf[-1].clone()
    cols = []
    for i in range(n_cols):
        n = int(2 ** lens.uniform(lo_log, hi_log))
        fam = MIXED_FAMILIES[i % 4]
        if fam == "uniform":
            w = int(lens.choice([8, 12, 16, 20]))
            v = torch.randint(0, 1 << w, (n,), generator=g, device=dev, dtype=torch.int64)
        elif fam == "zipf":
            v = torch.searchsorted(zcdf, torch.rand(n, generator=g, device=dev, dtype=torch.float64))
            v = torch.clamp(v, max=(1 << 20) - 1)
        elif fam == "sorted_gaps":
            u = torch.rand(n, generator=g, device=dev, dtype=torch.float64)
            gaps = torch.floor(torch.log1p(-u) / torch.log1p(torch.tensor(-0.3, dtype=torch.float64))) + 1
            v = torch.cumsum(gaps.to(torch.int64), 0)
        else:
            starts = torch.rand(n, generator=g, device=dev) < 1.0 / 16.0
            starts[0] = True
            run = torch.cumsum(starts.to(torch.int64), 0) - 1
            vals = torch.randint(0, 1 << 16, (int(run[-1]) + 1,), generator=g, device=dev, dtype=torch.int64)
            v = vals[run]
        cols.append((fam, v.to(torch.int32)))
    return cols


def sorted_geometric_device(n: int, p: float = 0.3, seed: int = 3, device="cuda"):
    """Sorted keys with geometric(p) gaps (>= 1), drawn with torch on `device`
    (int32 tensor; the distribution of sorted_geometric)."""
    import torch
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    u = torch.rand(n, generator=g, device=dev, dtype=torch.float64)
    gaps = torch.floor(torch.log1p(-u) / torch.log1p(torch.tensor(-p, dtype=torch.float64, device=dev))) + 1
    return torch.cumsum(gaps.to(torch.int64), 0).to(torch.int32)


def geometric_runs_device(n: int, mean_run: float = 16.0, value_bits: int = 16, seed: int = 4, device="cuda"):
    """Runs of geometric length (mean `mean_run`: a run starts at each row with
    probability 1/mean_run) of uniform values in [0, 2^value_bits), drawn with
    torch on `device` (int32 tensor; the distribution of geometric_runs)."""
    import torch
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    starts = torch.rand(n, generator=g, device=dev) < 1.0 / mean_run
    starts[0] = True
    run = torch.cumsum(starts.to(torch.int64), 0) - 1
    vals = torch.randint(0, 1 << value_bits, (int(run[-1]) + 1,), generator=g, device=dev, dtype=torch.int64)
    return vals[run].to(torch.int32)


def ssb_join(query: str, n: int, seed: int, device="cuda"):
    """Device columns, hash tables and the join + group-by arguments of the
    Q3.1 / Q4.1 shapes (fls_q31.cu / fls_q41.cu): (tables, hash tables, host
    encoded columns, device columns, probes, join_groupby keyword arguments)."""
    import torch

    from . import ops
    from .column import EncodedColumn
    if query == "q31":
        t = q31_tables(n, seed=seed)
        names, bits = ["lo_suppkey", "lo_custkey", "lo_orderdate", "lo_revenue"], Q31_BITS
    else:
        t = q41_tables(n, seed=seed)
        names = ["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue", "lo_supplycost"]
        bits = Q41_BITS
    dev = {k: torch.from_numpy(v).to(device) for k, v in t.items() if not k.startswith("lo_")}
    hcols = [EncodedColumn.uniform(t[k], bw=bits[k]) for k in names]
    dcols = [c.to_device(device) for c in hcols]
    if query == "q31":
        ht_s = ops.build_pht(dev["s_suppkey"], dev["s_suppkey"].numel(), vals=dev["s_nation"], filt=dev["s_region"])
        ht_c = ops.build_pht(dev["c_custkey"], dev["c_custkey"].numel(), vals=dev["c_nation"], filt=dev["c_region"])
        ht_d = ops.build_pht(dev["d_datekey"], N_DAYS, vals=dev["d_year"], filt=dev["d_in_range"])
        tables = {"ht_s": ht_s, "ht_c": ht_c, "ht_d": ht_d}
        probes = [(0, ht_s, ht_s.numel() // 2, 0, 2), (1, ht_c, ht_c.numel() // 2, 0, 2),
                  (2, ht_d, ht_d.numel() // 2, 0, 2)]
        kw = dict(agg_col=3, keys=[(0, 175, 2), (1, 7, 1), (2, 1, 0)], group_sub=1992, n_groups=Q31_GROUPS,
                  res_stride=6, sum_slot=4)
    else:
        ht_s = ops.build_pht(dev["s_suppkey"], dev["s_suppkey"].numel(), filt=dev["s_region"])
        ht_c = ops.build_pht(dev["c_custkey"], dev["c_custkey"].numel(), vals=dev["c_nation"], filt=dev["c_region"])
        ht_p = ops.build_pht(dev["p_partkey"], dev["p_partkey"].numel(), filt=dev["p_mfgr_low"])
        ht_d = ops.build_pht(dev["d_datekey"], N_DAYS, vals=dev["d_year"])
        tables = {"ht_s": ht_s, "ht_c": ht_c, "ht_p": ht_p, "ht_d": ht_d}
        probes = [(0, ht_s, ht_s.numel(), 0, 1), (1, ht_c, ht_c.numel() // 2, 0, 2), (2, ht_p, ht_p.numel(), 0, 1),
                  (3, ht_d, ht_d.numel() // 2, 0, 2)]
        kw = dict(agg_col=4, keys=[(1, 7, 1), (3, 1, 0)], group_sub=1992, n_groups=Q41_GROUPS, res_stride=4,
                  sum_slot=2, agg_sub_col=5)
    return t, tables, hcols, dcols, probes, kw


# ------------------------------------------------------------- SSB suite
# All thirteen SSB queries on one seeded SSB-shaped schema (SSB data is not
# available): cities U[0,250) with nation = city // 10 and region = nation // 5
# (dbgen's hierarchy), brands U[0,1000) with category = brand // 40 and
# manufacturer = category // 5, day ids 0..2555 with year and yyyymm.  The
# predicate constants and group formulas are those of crystal-opt src/ssb
# (q11.cu .. q43.cu); date keys are day ids instead of yyyymmdd, so date
# ranges become day-id ranges and the date table is indexed from 0.

SSB_SUPP, SSB_CUST, SSB_PART = 1 << 17, 1 << 18, 1 << 19
SSB_BITS = {"lo_orderdate": 12, "lo_suppkey": 17, "lo_custkey": 18, "lo_partkey": 19, "lo_quantity": 6,
            "lo_discount": 4, "lo_extendedprice": 24, "lo_revenue": 24, "lo_supplycost": 18}


def day_id(y: int, m: int, d: int) -> int:
    return int((np.datetime64(f"{y:04d}-{m:02d}-{d:02d}") - np.datetime64("1992-01-01")).astype(int))


def ssb_tables(n: int, seed: int = 13) -> dict:
    """Fact columns of n rows and the four dimension tables."""
    g = rng(seed)
    days = np.arange(N_DAYS)
    dates = np.datetime64("1992-01-01") + days
    ym = dates.astype("datetime64[M]").astype(int)
    s_city = g.integers(0, 250, size=SSB_SUPP).astype(np.int32)
    c_city = g.integers(0, 250, size=SSB_CUST).astype(np.int32)
    brand = g.integers(0, 1000, size=SSB_PART).astype(np.int32)
    t = {
        "lo_orderdate": g.integers(0, N_DAYS, size=n).astype(np.int32),
        "lo_suppkey": g.integers(0, SSB_SUPP, size=n).astype(np.int32),
        "lo_custkey": g.integers(0, SSB_CUST, size=n).astype(np.int32),
        "lo_partkey": g.integers(0, SSB_PART, size=n).astype(np.int32),
        "lo_quantity": g.integers(1, 51, size=n).astype(np.int32),
        "lo_discount": g.integers(0, 11, size=n).astype(np.int32),
        "lo_extendedprice": g.integers(90000, 10_500_001, size=n).astype(np.int32),
        "lo_revenue": g.integers(90000, 10_500_001, size=n).astype(np.int32),
        "lo_supplycost": g.integers(50000, 150000, size=n).astype(np.int32),
        "d_datekey": days.astype(np.int32), "d_year": year_of_day(days),
        "d_yearmonthnum": ((1970 + ym // 12) * 100 + ym % 12 + 1).astype(np.int32),
        "s_suppkey": np.arange(SSB_SUPP, dtype=np.int32), "s_city": s_city,
        "s_nation": (s_city // 10).astype(np.int32), "s_region": (s_city // 50).astype(np.int32),
        "c_custkey": np.arange(SSB_CUST, dtype=np.int32), "c_city": c_city,
        "c_nation": (c_city // 10).astype(np.int32), "c_region": (c_city // 50).astype(np.int32),
        "p_partkey": np.arange(SSB_PART, dtype=np.int32), "p_brand1": brand,
        "p_category": (brand // 40).astype(np.int32), "p_mfgr": (brand // 200).astype(np.int32),
    }
    return t


_I32_MIN = -(1 << 31)
_YEARS_92_97 = [(1992, 1997)]
_YEARS_97_98 = [(1997, 1998)]


def _dim(name):
    return {"d": ("d_datekey", N_DAYS), "s": ("s_suppkey", SSB_SUPP), "c": ("c_custkey", SSB_CUST),
            "p": ("p_partkey", SSB_PART)}[name]


# filter queries: (fact columns, [(column index, lo, hi)], agg_a, agg_b) with
# sum(cols[agg_a] * cols[agg_b]); join queries: fact columns, probes
# [(fact column index, dimension, payload column or None, filter column or
# None, [(lo, hi)] ranges)], group keys [(probe, multiplier, record word)],
# group_sub, n_groups, record stride, sum word, sum bits, measure column and
# subtracted column (or None).
SSB_QUERIES = {
    "q11": dict(kind="filter", cols=["lo_orderdate", "lo_discount", "lo_quantity", "lo_extendedprice"],
                filters=[(0, day_id(1993, 1, 1), day_id(1993, 12, 31)), (1, 1, 3), (2, _I32_MIN, 24)]),
    "q12": dict(kind="filter", cols=["lo_orderdate", "lo_discount", "lo_quantity", "lo_extendedprice"],
                filters=[(0, day_id(1994, 1, 1), day_id(1994, 1, 31)), (1, 4, 6), (2, 26, 35)]),
    "q13": dict(kind="filter", cols=["lo_orderdate", "lo_discount", "lo_quantity", "lo_extendedprice"],
                filters=[(0, day_id(1994, 2, 4), day_id(1994, 2, 10)), (1, 5, 7), (2, 26, 35)]),
    "q21": dict(kind="join", cols=["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"],
                probes=[(0, "s", None, "s_region", [(1, 1)]), (1, "p", "p_brand1", "p_category", [(1, 1)]),
                        (2, "d", "d_year", None, None)],
                keys=[(1, 7, 1), (2, 1, 0)], sub=1992, groups=7 * 1000, stride=4, sum_slot=2, sum_bits=64,
                agg=3, agg_sub=None),
    "q22": dict(kind="join", cols=["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"],
                probes=[(0, "s", None, "s_region", [(2, 2)]), (1, "p", "p_brand1", "p_brand1", [(260, 267)]),
                        (2, "d", "d_year", None, None)],
                keys=[(1, 7, 1), (2, 1, 0)], sub=1992, groups=7 * 1000, stride=4, sum_slot=2, sum_bits=64,
                agg=3, agg_sub=None),
    "q23": dict(kind="join", cols=["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"],
                probes=[(0, "s", None, "s_region", [(3, 3)]), (1, "p", "p_brand1", "p_brand1", [(260, 260)]),
                        (2, "d", "d_year", None, None)],
                keys=[(1, 7, 1), (2, 1, 0)], sub=1992, groups=7 * 1000, stride=4, sum_slot=2, sum_bits=64,
                agg=3, agg_sub=None),
    "q31": dict(kind="join", cols=["lo_suppkey", "lo_custkey", "lo_orderdate", "lo_revenue"],
                probes=[(0, "s", "s_nation", "s_region", [(2, 2)]), (1, "c", "c_nation", "c_region", [(2, 2)]),
                        (2, "d", "d_year", "d_year", _YEARS_92_97)],
                keys=[(0, 25 * 7, 2), (1, 7, 1), (2, 1, 0)], sub=1992, groups=7 * 25 * 25, stride=6, sum_slot=4,
                sum_bits=64, agg=3, agg_sub=None),
    "q32": dict(kind="join", cols=["lo_suppkey", "lo_custkey", "lo_orderdate", "lo_revenue"],
                probes=[(0, "s", "s_city", "s_nation", [(24, 24)]), (1, "c", "c_city", "c_nation", [(24, 24)]),
                        (2, "d", "d_year", "d_year", _YEARS_92_97)],
                keys=[(0, 250 * 7, 2), (1, 7, 1), (2, 1, 0)], sub=1992, groups=7 * 250 * 250, stride=4, sum_slot=3,
                sum_bits=32, agg=3, agg_sub=None),
    "q33": dict(kind="join", cols=["lo_suppkey", "lo_custkey", "lo_orderdate", "lo_revenue"],
                probes=[(0, "s", "s_city", "s_city", [(231, 231), (235, 235)]),
                        (1, "c", "c_city", "c_city", [(231, 231), (235, 235)]),
                        (2, "d", "d_year", "d_year", _YEARS_92_97)],
                keys=[(0, 250 * 7, 2), (1, 7, 1), (2, 1, 0)], sub=1992, groups=7 * 250 * 250, stride=4, sum_slot=3,
                sum_bits=32, agg=3, agg_sub=None),
    "q34": dict(kind="join", cols=["lo_suppkey", "lo_custkey", "lo_orderdate", "lo_revenue"],
                probes=[(0, "s", "s_city", "s_city", [(231, 231), (235, 235)]),
                        (1, "c", "c_city", "c_city", [(231, 231), (235, 235)]),
                        (2, "d", "d_year", "d_yearmonthnum", [(199712, 199712)])],
                keys=[(0, 250 * 7, 2), (1, 7, 1), (2, 1, 0)], sub=1992, groups=7 * 250 * 250, stride=4, sum_slot=3,
                sum_bits=32, agg=3, agg_sub=None),
    "q41": dict(kind="join", cols=["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue",
                                   "lo_supplycost"],
                probes=[(0, "s", None, "s_region", [(1, 1)]), (1, "c", "c_nation", "c_region", [(1, 1)]),
                        (2, "p", None, "p_mfgr", [(0, 1)]), (3, "d", "d_year", None, None)],
                keys=[(1, 7, 1), (3, 1, 0)], sub=1992, groups=7 * 25, stride=4, sum_slot=2, sum_bits=64,
                agg=4, agg_sub=5),
    "q42": dict(kind="join", cols=["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue",
                                   "lo_supplycost"],
                probes=[(0, "s", "s_nation", "s_region", [(1, 1)]), (1, "c", None, "c_region", [(1, 1)]),
                        (2, "p", "p_category", "p_mfgr", [(0, 0), (1, 1)]),
                        (3, "d", "d_year", "d_year", _YEARS_97_98)],
                keys=[(3, 25 * 25, 0), (0, 25, 1), (2, 1, 2)], sub=1992 * 25 * 25, groups=7 * 25 * 25, stride=6,
                sum_slot=4, sum_bits=64, agg=4, agg_sub=5),
    "q43": dict(kind="join", cols=["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue",
                                   "lo_supplycost"],
                probes=[(0, "s", "s_city", "s_nation", [(24, 24)]), (1, "c", None, "c_region", [(1, 1)]),
                        (2, "p", "p_brand1", "p_category", [(3, 3)]), (3, "d", "d_year", "d_year", _YEARS_97_98)],
                keys=[(3, 250 * 1000, 0), (0, 1000, 1), (2, 1, 2)], sub=1992 * 250 * 1000, groups=7 * 250 * 1000,
                stride=4, sum_slot=3, sum_bits=32, agg=4, agg_sub=5),
}


def ssb_device_query(name: str, t: dict, dcols: dict, device="cuda"):
    """Device hash tables and operator arguments of SSB query `name` over the
    tables `t` and the device columns `dcols` (fact column name -> device
    column).  Filter queries: {"kind", "cols", "filters", "agg_a", "agg_b"};
    join queries: {"kind", "cols", "tables", "probes", "kw"} with probes in the
    join_groupby form and kw its keyword arguments."""
    import torch

    from . import ops
    q = SSB_QUERIES[name]
    cols = [dcols[c] for c in q["cols"]]
    if q["kind"] == "filter":
        return dict(kind="filter", cols=cols, filters=q["filters"], agg_a=3, agg_b=1)
    tables, probes = [], []
    for col, dim, payload, filt, ranges in q["probes"]:
        key_col, length = _dim(dim)
        to = lambda k: torch.from_numpy(t[k]).to(device)  # noqa: E731
        ht = ops.build_pht(to(key_col), length, vals=None if payload is None else to(payload),
                           filt=None if filt is None else to(filt), ranges=ranges)
        tables.append(ht)
        probes.append((col, ht, length, 0, 1 if payload is None else 2))
    kw = dict(agg_col=q["agg"], keys=q["keys"], group_sub=q["sub"], n_groups=q["groups"], res_stride=q["stride"],
              sum_slot=q["sum_slot"], sum_bits=q["sum_bits"], agg_sub_col=-1 if q["agg_sub"] is None else q["agg_sub"])
    return dict(kind="join", cols=cols, tables=tables, probes=probes, kw=kw)


# ------------------------------------------------ SSB on dbgen's tables
# The same thirteen queries on the tables of SSB's own generator (dbgen), in
# the reference loader's integer encoding: dates are yyyymmdd day keys, the
# dimension keys run from 1 to the table's row count, and the hash tables are
# those of crystal-opt src/ssb and fastlanes/src/ssb: a supplier, customer or
# part table has one slot per dimension row, slot = key % rows
# (HASH(key, len, 0), crystal-opt/join.cuh:26), and the date table has
# 19981230 - 19920101 + 1 slots from key 19920101 (fls_q21.cu:290,309).

SSB_DATE_MIN = 19920101
SSB_DATE_SLOTS = 19981230 - 19920101 + 1

# Q1.x date predicates on yyyymmdd keys (crystal-opt src/ssb/q11.cu: year
# 1993; q12.cu: January 1994; q13.cu: week 6 of 1994 = 4-10 February).
SSB_DBGEN_DATE_FILTER = {"q11": (19930101, 19931231), "q12": (19940101, 19940131), "q13": (19940204, 19940210)}


def ssb_dbgen_dims(t: dict) -> dict:
    """(key column, hash table slots, keys_min) of each dimension."""
    return {"d": ("d_datekey", SSB_DATE_SLOTS, SSB_DATE_MIN), "s": ("s_suppkey", int(t["s_suppkey"].size), 0),
            "c": ("c_custkey", int(t["c_custkey"].size), 0), "p": ("p_partkey", int(t["p_partkey"].size), 0)}


def ssb_dbgen_columns(t: dict, names=None) -> dict:
    """Fact columns encoded as the reference encodes them: uniform FOR with the
    column minimum as base (fls_q21.cu:373-375 subtracts lo_orderdate's) and
    the smallest bit width that holds max - min."""
    from .column import EncodedColumn
    out = {}
    for k in names or SSB_BITS:
        v = t[k]
        out[k] = EncodedColumn.uniform(v, base=int(v.min()))
    return out


def ssb_dbgen_query(name: str, t: dict, dcols: dict, device="cuda"):
    """ssb_device_query for dbgen's tables (see ssb_dbgen_dims and
    SSB_DBGEN_DATE_FILTER): the same predicates, group formulas and record
    layouts."""
    import torch

    from . import ops
    q = SSB_QUERIES[name]
    cols = [dcols[c] for c in q["cols"]]
    if q["kind"] == "filter":
        lo, hi = SSB_DBGEN_DATE_FILTER[name]
        filters = [(0, lo, hi)] + list(q["filters"][1:])
        return dict(kind="filter", cols=cols, filters=filters, agg_a=3, agg_b=1)
    dims = ssb_dbgen_dims(t)
    tables, probes = [], []
    for col, dim, payload, filt, ranges in q["probes"]:
        key_col, length, kmin = dims[dim]
        to = lambda k: torch.from_numpy(t[k]).to(device)  # noqa: E731
        ht = ops.build_pht(to(key_col), length, vals=None if payload is None else to(payload),
                           filt=None if filt is None else to(filt), ranges=ranges, keys_min=kmin)
        tables.append(ht)
        probes.append((col, ht, length, kmin, 1 if payload is None else 2))
    kw = dict(agg_col=q["agg"], keys=q["keys"], group_sub=q["sub"], n_groups=q["groups"], res_stride=q["stride"],
              sum_slot=q["sum_slot"], sum_bits=q["sum_bits"], agg_sub_col=-1 if q["agg_sub"] is None else q["agg_sub"])
    return dict(kind="join", cols=cols, tables=tables, probes=probes, kw=kw)


SSB_DBGEN_COLUMNS = ["lo_custkey", "lo_partkey", "lo_suppkey", "lo_orderdate", "lo_quantity", "lo_extendedprice",
                     "lo_discount", "lo_revenue", "lo_supplycost", "s_suppkey", "s_city", "s_nation", "s_region",
                     "c_custkey", "c_city", "c_nation", "c_region", "p_partkey", "p_mfgr", "p_category", "p_brand1",
                     "d_datekey", "d_year", "d_yearmonthnum", "d_weeknuminyear"]


def ssb_dbgen_default_dir(sf: float) -> str:
    import tempfile
    base = os.environ.get("FLS_SSB_DIR") or os.path.join(tempfile.gettempdir(), "fls_ssb")
    return os.path.join(base, f"sf{sf:g}")


def ssb_dbgen_load(path: str) -> dict:
    """SSB columns loaded from dbgen's tables: <path>/<column>.i32, raw int32
    in the reference loader's encoding (written by the loader next to the
    oracle, oracle/ssb_load.c)."""
    if not os.path.exists(os.path.join(path, "complete")):
        raise FileNotFoundError(f"no loaded SSB tables in {path} (generate them with python oracle/ssb_data.py)")
    return {k: np.fromfile(os.path.join(path, k + ".i32"), dtype=np.int32) for k in SSB_DBGEN_COLUMNS}
