"""Writes tests/golden/ssb_answers.json: the Star Schema Benchmark answers the
reference holds, read as text from its files (nothing is computed here).

    python tests/golden/make_ssb_answers.py [REFERENCE_ROOT]

  * Q1.1 at scale factors 0.1, 1 and 10, Q1.2 and Q1.3 at 1:
    fastlanes/src/include/ssb_utils.h:178-183 (`SSBQuery1 ssb_qXY_SF {result, ssb_SF}`).
  * Q2.1, Q3.1 and Q4.1 at scale factor 10 (their magnitudes and the Q1.1
    file, which holds the SF 10 answer of ssb_utils.h, say so):
    data/result_of_queries/q21 ("year brand sum" per group), q31 ("year
    c_nation s_nation sum"), q41 ("year c_nation sum"); each file ends with
    a "Res Count: n" line, checked against the rows read.
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main() -> None:
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    hdr = open(os.path.join(ref, "fastlanes/src/include/ssb_utils.h")).read()
    scalar = {}
    for q, sf, value in re.findall(r"SSBQuery1\s+ssb_(q\d\d)_(\w+)\s*\{(\d+),\s*ssb_\w+\}", hdr):
        scalar.setdefault(q, {})[sf.replace("_", ".")] = int(value)
    groups = {}
    for q in ("q21", "q31", "q41"):
        rows = []
        for line in open(os.path.join(ref, "data/result_of_queries", q)):
            parts = line.split()
            if parts and all(x.lstrip("-").isdigit() for x in parts):  # the last line is "Res Count: n"
                rows.append([int(x) for x in parts])
        count = [int(x) for x in open(os.path.join(ref, "data/result_of_queries", q)).read().split("Res Count:")[1].split()[:1]]
        assert count == [len(rows)], (q, count, len(rows))
        groups[q] = rows
    q11_file = open(os.path.join(ref, "data/result_of_queries/q11")).read().split()
    out = {"source": "reference files: fastlanes/src/include/ssb_utils.h:178-183, data/result_of_queries/q11,q21,q31,q41",
           "scalar": scalar, "q11_file": int(q11_file[0]) if q11_file else None,
           "groups_sf10": groups}
    # one group per line
    text = json.dumps({k: v for k, v in out.items() if k != "groups_sf10"}, indent=1)[:-2]
    text += ',\n "groups_sf10": {\n'
    text += ",\n".join(f'  "{q}": [\n' + ",\n".join("   " + json.dumps(r) for r in rows) + "\n  ]"
                       for q, rows in groups.items())
    text += "\n }\n}\n"
    assert json.loads(text) == out
    with open(os.path.join(HERE, "ssb_answers.json"), "w") as f:
        f.write(text)
    print({k: len(v) for k, v in groups.items()}, scalar)


if __name__ == "__main__":
    main()
