"""Binary column cache in the reference's on-disk format (src/file_access.hpp, src/main.cu:405-474):
raw per-column arrays shipdate.bin (int32), returnflag.bin / linestatus.bin (char), discount.bin,
tax.bin, extendedprice.bin, quantity.bin (int64). Host-side tests; loading into a context and
running the query is covered by the gpu-marked test at the end."""
import ctypes
import os

import numpy as np
import pytest

import gen_np
import tpchq01_gpu_b200 as q
from tpchq01_gpu_b200 import _lib

FILES = {"shipdate": ("shipdate.bin", np.int32), "returnflag": ("returnflag.bin", "S1"),
         "linestatus": ("linestatus.bin", "S1"), "discount": ("discount.bin", np.int64), "tax": ("tax.bin", np.int64),
         "extendedprice": ("extendedprice.bin", np.int64), "quantity": ("quantity.bin", np.int64)}


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def write(dirpath, cols):
    keep = {k: np.ascontiguousarray(v) for k, v in cols.items()}
    c = _lib.Columns(ptr(keep["shipdate"]), ptr(keep["discount"]), ptr(keep["extendedprice"]), ptr(keep["tax"]),
                     ptr(keep["quantity"]), ptr(keep["returnflag"]), ptr(keep["linestatus"]))
    _lib.check(q.lib().q1_cache_write(str(dirpath).encode(), ctypes.byref(c), len(keep["shipdate"])))


def rows_of(dirpath):
    n = ctypes.c_uint64()
    st = q.lib().q1_cache_rows(str(dirpath).encode(), ctypes.byref(n))
    return st, n.value


@pytest.mark.parametrize("rows", [0, 1, 31, 100_003])
def test_write_matches_reference_format_and_reads_back(tmp_path, rows):
    cols = gen_np.generate(11, 0, rows)
    write(tmp_path, cols)
    for k, (name, dt) in FILES.items():
        raw = np.fromfile(tmp_path / name, dtype=dt)
        assert raw.shape[0] == rows and np.array_equal(raw, cols[k]), name
    st, n = rows_of(tmp_path)
    assert st == 0 and n == rows
    out = {k: np.zeros(rows, dtype=dt) for k, (name, dt) in FILES.items()}
    o = _lib.ColumnsOut(*[ptr(out[k]) for k in ["shipdate", "returnflag", "linestatus", "discount", "tax",
                                                  "extendedprice", "quantity"]])
    _lib.check(q.lib().q1_cache_read(str(tmp_path).encode(), rows, ctypes.byref(o)))
    for k in FILES:
        assert np.array_equal(out[k], cols[k]), k


def test_missing_and_mis_sized_files_are_rejected(tmp_path):
    st, _ = rows_of(tmp_path)
    assert st == 1
    write(tmp_path, gen_np.generate(12, 0, 1000))
    with open(tmp_path / "tax.bin", "ab") as f:
        f.write(b"\0" * 8)                      # one element too many
    st, _ = rows_of(tmp_path)
    assert st == 1 and "tax.bin" in q.lib().q1_last_error().decode()
    write(tmp_path, gen_np.generate(12, 0, 1000))
    os.remove(tmp_path / "quantity.bin")
    st, _ = rows_of(tmp_path)
    assert st == 1 and "quantity.bin" in q.lib().q1_last_error().decode()


def test_sf1_sized_cache_is_not_rescaled(tmp_path):
    """The reference multiplies an SF-1-sized cache's cardinality by the scale factor and then
    fails to read it (src/main.cu:412-414); the row count here is the file's."""
    rows = 6001215 // 1000   # small stand-in: the count comes from the file size alone
    write(tmp_path, gen_np.generate(13, 0, rows))
    st, n = rows_of(tmp_path)
    assert st == 0 and n == rows


@pytest.mark.gpu
def test_cache_load_runs_like_generated_table(cuda, tmp_path):
    rows = 300_011
    cols = gen_np.generate(14, 0, rows)
    write(tmp_path, cols)
    n = ctypes.c_uint64()
    with q.Q1Context() as a, q.Q1Context() as b:
        _lib.check(q.lib().q1_cache_load(a._h, str(tmp_path).encode(), 1, 0, 0, ctypes.byref(n)))
        assert n.value == rows
        b.load_columns(cols, layout="compressed", packing="pair", residency="hbm")
        ra = a.run(apply_compression=True, num_query_execution_runs=1)
        rb = b.run(apply_compression=True, num_query_execution_runs=1)
        assert np.array_equal(ra.table(), rb.table())
