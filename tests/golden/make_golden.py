"""Generate tests/golden/q1_golden.json from the reference's OWN CPU kernels.

Run in a container where the reference sources exist (oracle/Makefile builds them into
oracle/_ref/libq1ref.so):  python tests/golden/make_golden.py

Each case regenerates its input with the seeded generator (tests/gen_np.py), records a SHA-256 of
the input columns (so a test can tell that it rebuilt the same input), and stores the per-group
aggregates computed by KernelHyPer<true> (cpu/kernel_hyper.hpp) and by
KernelX100<kMagic,true,kNoAvx512> (cpu/kernel_x100.hpp). Nothing from any benchmark suite is
stored: the inputs are synthetic and only the 6x6 aggregate table per case is kept.
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import gen_np  # noqa: E402
from oracle import py_oracle as O  # noqa: E402

CASES = [
    # name, seed, first_row, rows, cutoff_day
    ("config0_6M", 20260101, 0, 6_000_000, 729999),
    ("small_default", 11, 0, 100_000, 729999),
    ("offset_rows", 12, 123_456, 50_000, 729999),
    ("cutoff_1998_06_01", 13, 0, 40_000, 729906),
    ("cutoff_all_pass", 14, 0, 10_000, 730089),
    ("cutoff_none_pass", 15, 0, 10_000, 727000),
    ("cutoff_1995_06_17", 16, 0, 30_000, 728826),
    ("ragged_4097", 17, 0, 4097, 729999),
    ("ragged_33", 18, 0, 33, 729999),
    ("one_row", 19, 0, 1, 729999),
]


def input_digest(cols):
    h = hashlib.sha256()
    for k in ["shipdate", "discount", "extendedprice", "tax", "quantity", "returnflag", "linestatus"]:
        h.update(cols[k].tobytes())
    return h.hexdigest()


def as_lists(t):
    return [[int(v) for v in row] for row in t]


def main():
    out = {"aggregates": ["count", "sum_qty", "sum_base_price", "sum_disc", "sum_disc_price", "sum_charge"],
           "groups": ["AF", "AO", "NF", "NO", "RF", "RO"],
           "source": "reference cpu/kernel_hyper.hpp KernelHyPer<true> and cpu/kernel_x100.hpp "
                     "KernelX100<kMagic,true,kNoAvx512>, built by oracle/Makefile",
           "cases": []}
    for name, seed, first, rows, cutoff in CASES:
        cols = gen_np.generate(seed, first, rows)
        t = O.RefTable(cols, cutoff)
        hyper, flag = t.hyper()
        x100, rc = t.x100()
        t.close()
        assert flag == 0, name
        case = {"name": name, "seed": seed, "first_row": first, "rows": rows, "cutoff_day": cutoff,
                "input_sha256": input_digest(cols), "hyper": as_lists(hyper),
                "x100": as_lists(x100) if rc == 0 else None}
        out["cases"].append(case)
        print(name, "ok", "x100" if rc == 0 else "x100 n/a")
    with open(os.path.join(HERE, "q1_golden.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
