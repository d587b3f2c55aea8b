"""lineitem .tbl ingestion on the GPU (q1_tbl_parse_device, q1_tbl_read_file, q1_tbl_load) against
the oracle's parse restatement (itself pinned to the reference's Decimal/Char/Date types in
tests/test_tbl.py): row counts, every column bit for bit, lines across 64 KB tile boundaries,
unaligned text, a missing final newline, malformed lines (count and first offset), too-small
outputs, chunked file reads, and a loaded table answering Q1 like the generated one."""
import ctypes
import os

import numpy as np
import pytest
import torch

import tpchq01_gpu_b200 as q
from oracle import py_oracle as O
from tpchq01_gpu_b200 import _lib

pytestmark = pytest.mark.gpu

COLS = ["shipdate", "quantity", "extendedprice", "discount", "tax", "returnflag", "linestatus"]


def gpu_parse(text, offset=0, capacity=None):
    """Parses `text` placed `offset` bytes into a device buffer; returns (columns, rows, status, message)."""
    L = q.lib()
    dev = torch.zeros(len(text) + offset + 16, dtype=torch.uint8, device="cuda")
    if text:
        dev[offset: offset + len(text)] = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    base = dev.data_ptr() + offset
    n = ctypes.c_uint64(0)
    _lib.check(L.q1_tbl_count_device(ctypes.c_void_p(base), len(text), ctypes.byref(n), None))
    rows = n.value if capacity is None else capacity
    out = {"shipdate": torch.zeros(rows + 1, dtype=torch.int32, device="cuda"),
           "quantity": torch.zeros(rows + 1, dtype=torch.int64, device="cuda"),
           "extendedprice": torch.zeros(rows + 1, dtype=torch.int64, device="cuda"),
           "discount": torch.zeros(rows + 1, dtype=torch.int64, device="cuda"),
           "tax": torch.zeros(rows + 1, dtype=torch.int64, device="cuda"),
           "returnflag": torch.zeros(rows + 1, dtype=torch.uint8, device="cuda"),
           "linestatus": torch.zeros(rows + 1, dtype=torch.uint8, device="cuda")}
    o = _lib.ColumnsOut(*[out[k].data_ptr() for k in ["shipdate", "returnflag", "linestatus", "discount", "tax",
                                                       "extendedprice", "quantity"]])
    got = ctypes.c_uint64(0)
    st = L.q1_tbl_parse_device(ctypes.c_void_p(base), len(text), ctypes.byref(o), rows, ctypes.byref(got), None)
    msg = L.q1_last_error().decode() if st else ""
    torch.cuda.synchronize()
    r = min(got.value, rows)
    cols = {k: v[:r].cpu().numpy() for k, v in out.items()}
    cols["returnflag"] = cols["returnflag"].view("S1")
    cols["linestatus"] = cols["linestatus"].view("S1")
    return cols, got.value, st, msg


def check_same(got, want):
    for k in COLS:
        assert np.array_equal(got[k], want[k]), k


@pytest.mark.parametrize("rows", [0, 1, 7, 1000, 40_000, 200_003])
def test_parse_matches_oracle(cuda, rows):
    text = q.tbl_format(q.generate_host(41, 0, rows)) if rows else b""
    want, wrows, bad, _ = O.parse_tbl(text)
    got, grows, st, msg = gpu_parse(text)
    assert st == 0, msg
    assert grows == wrows == rows and bad == 0
    check_same(got, want)


@pytest.mark.parametrize("offset", [1, 3, 8, 15])
def test_unaligned_text_and_no_final_newline(cuda, offset):
    text = q.tbl_format(q.generate_host(42, 5, 3000))[:-1]     # drop the final '\n'
    want, wrows, bad, _ = O.parse_tbl(text)
    got, grows, st, msg = gpu_parse(text, offset=offset)
    assert st == 0, msg
    assert grows == wrows == 3000 and bad == 0
    check_same(got, want)


def test_lines_across_tile_boundaries(cuda):
    """Lines of every length around the 64 KB tiles: each tile's first line starts in the tile
    before it."""
    cols = q.generate_host(43, 0, 20_000)
    base = q.tbl_format(cols).split(b"\n")[:-1]
    pads = [b"|" + b"z" * (k % 97) for k in range(len(base))]   # longer trailing fields
    text = b"\n".join(line + pad for line, pad in zip(base, pads)) + b"\n"
    assert len(text) > 4 * 65536
    want, wrows, bad, _ = O.parse_tbl(text)
    got, grows, st, msg = gpu_parse(text)
    assert st == 0 and bad == 0, msg
    check_same(got, want)
    check_same(got, cols)


def test_quirks_match_oracle(cuda):
    text = (b"1|2|3|4|17.5|100|-0.04|+3|R|F|1992-02-29|x|y|z|\n"
            b"1|2|3|4|17|12345.67|0.1|0.08|N|O|2000-02-29|\n"
            b"9|9|9|9|-1.05|0.00|0.10|0.00|A|F|1998-12-31|tail\n"
            b"1|2|3|4|50.00|104949.50|0.10|0.08|N|O|1995-06-17|no newline at the end")
    want, _, bad, _ = O.parse_tbl(text)
    got, rows, st, msg = gpu_parse(text)
    assert st == 0 and rows == 4 and bad == 0, msg
    check_same(got, want)


def test_malformed_lines_are_reported(cuda):
    lines = q.tbl_format(q.generate_host(44, 0, 5000)).split(b"\n")[:-1]
    lines[10] = b"1|2|3|4|x|1.00|0.01|0.02|R|F|1994-01-01|"
    lines[2000] = b"1|2|3|4|1.00|1.00|0.01|0.02|RR|F|1994-01-01|"
    lines[4999] = b"1|2|3|4|1|1|0|0|A|F|1994-02-30|"
    text = b"\n".join(lines) + b"\n\n"
    want, wrows, wbad, wfirst = O.parse_tbl(text)
    got, rows, st, msg = gpu_parse(text)
    assert st == 1 and rows == wrows == 5001
    assert f"{wbad} malformed line(s); the first starts at byte {wfirst}" in msg
    check_same(got, want)


def test_capacity_too_small_is_reported(cuda):
    text = q.tbl_format(q.generate_host(45, 0, 100))
    got, rows, st, msg = gpu_parse(text, capacity=60)
    assert st == 1 and rows == 100 and "holds 100 rows" in msg


@pytest.mark.parametrize("chunk", [1 << 20, 256 << 20])
def test_read_file_in_chunks(cuda, tmp_path, monkeypatch, chunk):
    monkeypatch.setenv("Q1_TBL_CHUNK_BYTES", str(chunk))
    cols = q.generate_host(46, 0, 60_000)
    path = tmp_path / "lineitem.tbl"
    path.write_bytes(q.tbl_format(cols))
    got = q.tbl_read_file(str(path))
    check_same(got, cols)


@pytest.mark.parametrize("layout", ["compressed", "uncompressed"])
def test_loaded_table_answers_like_the_generated_one(cuda, tmp_path, layout):
    rows = 300_007
    path = tmp_path / "lineitem.tbl"
    path.write_bytes(q.tbl_format(q.generate_host(47, 0, rows)))
    with q.Q1Context() as a, q.Q1Context() as b:
        assert a.load_tbl(str(path), layout=layout) == rows
        b.generate(47, rows, layout=layout)
        kw = dict(apply_compression=layout == "compressed", num_query_execution_runs=1)
        assert np.array_equal(a.run(**kw).table(), b.run(**kw).table())


def test_missing_file(cuda, tmp_path):
    with pytest.raises(q.Q1Error) as e:
        q.tbl_read_file(str(tmp_path / "absent.tbl"))
    assert e.value.status == 1 and "cannot open" in str(e.value)
