"""The oracle (oracle/q1_oracle.c) against golden aggregates produced by the reference's own CPU
kernels (tests/golden/q1_golden.json, written by tests/golden/make_golden.py)."""
import hashlib
import json
import os

import numpy as np
import pytest

import gen_np
from oracle import py_oracle as O

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "q1_golden.json")))
CASES = {c["name"]: c for c in GOLDEN["cases"]}


def digest(cols):
    h = hashlib.sha256()
    for k in ["shipdate", "discount", "extendedprice", "tax", "quantity", "returnflag", "linestatus"]:
        h.update(cols[k].tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_golden(name):
    c = CASES[name]
    cols = gen_np.generate(c["seed"], c["first_row"], c["rows"])
    assert digest(cols) == c["input_sha256"], "generator no longer reproduces the golden input"
    got, flag = O.q1_uncompressed(cols, c["cutoff_day"])
    assert flag == 0
    assert [[int(v) for v in row] for row in got] == c["hyper"]
    if c["x100"] is not None:
        assert c["x100"] == c["hyper"]


@pytest.mark.parametrize("name", ["small_default", "cutoff_1998_06_01", "ragged_4097", "one_row"])
@pytest.mark.parametrize("packing", ["pair", "sep"])
def test_compressed_oracle_matches_golden(name, packing):
    """The compressed-input restatement (src/main.cu:773-803 layout) gives the same table,
    with and without the precomputed filter bitmap (src/main.cu:362-389)."""
    c = CASES[name]
    cols = gen_np.generate(c["seed"], c["first_row"], c["rows"])
    comp = gen_np.compress(cols, packing)
    got, _ = O.q1_compressed(comp, c["cutoff_day"])
    assert [[int(v) for v in row] for row in got] == c["hyper"]
    comp["filter"] = O.precompute_filter(comp["shipdate"], c["cutoff_day"])
    assert np.array_equal(comp["filter"], gen_np.filter_bitmap(comp["shipdate"], c["cutoff_day"]))
    got_f, _ = O.q1_compressed(comp, c["cutoff_day"], use_filter=True)
    assert [[int(v) for v in row] for row in got_f] == c["hyper"]


def test_oracle_empty_input():
    cols = gen_np.generate(1, 0, 0)
    got, flag = O.q1_uncompressed(cols)
    assert flag == 0 and all(int(v) == 0 for v in got.flat)


def test_oracle_detects_int64_overflow():
    """HyPer's handle_overflow path (cpu/kernel_hyper.hpp:65-91): a product beyond int64."""
    cols = gen_np.generate(3, 0, 4)
    cols["extendedprice"][0] = 1 << 62
    _, flag = O.q1_uncompressed(cols)
    assert flag == 1


def test_oracle_catches_a_planted_mistake():
    """A mistake planted in the oracle's input (one row's discount changed) changes its answer."""
    c = CASES["small_default"]
    cols = gen_np.generate(c["seed"], c["first_row"], c["rows"])
    i = int(np.argmax(cols["shipdate"] <= c["cutoff_day"]))
    cols["discount"][i] = (cols["discount"][i] + 1) % 11
    got, _ = O.q1_uncompressed(cols, c["cutoff_day"])
    assert [[int(v) for v in row] for row in got] != c["hyper"]


@pytest.mark.parametrize("seed,first,rows,threads", [(20260101, 0, 200_003, 4), (9, 1 << 40, 1000, 3), (5, 17, 1, 8)])
def test_oracle_generator_equals_numpy_restatement(seed, first, rows, threads):
    """oracle/gen_rows.h (the generator the reference arm and the headline parity use) gives the
    numpy restatement's columns bit for bit."""
    a = O.generate(seed, first, rows, threads)
    b = gen_np.generate(seed, first, rows)
    for k in b:
        assert np.array_equal(a[k], b[k]), k
