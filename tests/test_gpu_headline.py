"""Parity at the headline sizes, against the reference's own CPU kernels.

* 600 M rows, compressed (pair codes), HBM-resident: every placement, filter pushdown off and on,
  against the reference's KernelX100 (cpu/kernel_x100.hpp:140-402, built from the reference
  sources into oracle/_ref) over the same generated rows, in chunks of its compact copy.
  At this size the N/O group's sum_charge is about 2^62 and the 128-bit sums carry across
  CTAs' partials.
* 6 M rows, uncompressed reference types, in_registers placement (the CPU-runnable workload):
  through q1_run against the golden table the reference's KernelHyPer produced
  (tests/golden/q1_golden.json, case config0_6M).
Tolerance 0: every aggregate is an exact integer."""
import json
import os

import numpy as np
import pytest

import gen_np
import tpchq01_gpu_b200 as q
from oracle import py_oracle as O

pytestmark = pytest.mark.gpu

PLACEMENTS = ["in_registers", "in_registers_per_thread", "local_mem", "shared_mem_per_thread", "global"]
HEADLINE_ROWS = 600_000_000
HEADLINE_SEED = 20260102
GOLDEN = {c["name"]: c for c in json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                                            "q1_golden.json")))["cases"]}


@pytest.fixture(scope="module")
def reference_600m():
    """KernelX100's table over the 600 M generated rows (the inputs built by the oracle)."""
    chunks = O.RefChunks(HEADLINE_SEED, 0, HEADLINE_ROWS, chunk_rows=1 << 25)
    try:
        table, rc = chunks.run()
    finally:
        chunks.close()
    assert rc == 0
    return table


@pytest.fixture(scope="module")
def ctx_600m(cuda):
    c = q.Q1Context()
    c.generate(HEADLINE_SEED, HEADLINE_ROWS, layout="compressed", packing="pair", residency="hbm")
    yield c
    c.close()


@pytest.mark.parametrize("pushdown", [False, True])
@pytest.mark.parametrize("placement", PLACEMENTS)
def test_600m_rows_bit_exact_against_reference_x100(ctx_600m, reference_600m, placement, pushdown):
    res = ctx_600m.run(hash_table_placement=placement, apply_compression=True, use_filter_pushdown=pushdown,
                       num_query_execution_runs=1)
    got = res.table()
    assert np.array_equal(got, reference_600m)
    assert sum(int(got[g, 0]) for g in range(6)) > 0.98 * HEADLINE_ROWS
    # the largest group's sum_charge is past 2^62: its 128-bit partials carry between words
    assert max(int(got[g, 5]) for g in range(6)) > 1 << 62


@pytest.mark.parametrize("placement", ["in_registers", "in_registers_per_thread"])
@pytest.mark.parametrize("residency", ["hbm", "pinned"])
def test_config0_6m_golden_on_gpu(cuda, placement, residency):
    case = GOLDEN["config0_6M"]
    cols = gen_np.generate(case["seed"], case["first_row"], case["rows"])
    with q.Q1Context() as c:
        c.load_columns(cols, "uncompressed", "pair", residency)
        res = c.run(hash_table_placement=placement, apply_compression=False, cutoff_day=case["cutoff_day"],
                    num_query_execution_runs=2)
    assert [[int(v) for v in row] for row in res.table()] == case["hyper"]
