"""lineitem .tbl text: the product's writer (q1_tbl_format) and the oracle's parse restatement,
pinned against the reference's own value types (Decimal<15,2>, Char, Date from
cpu/tpch_kit.hpp / cpu/tpch_kit.cpp, built from the reference sources into oracle/_ref). No GPU."""
import datetime

import numpy as np
import pytest

import tpchq01_gpu_b200 as q
from oracle import py_oracle as O

COLS = ["shipdate", "quantity", "extendedprice", "discount", "tax", "returnflag", "linestatus"]


def same(a, b):
    return all(np.array_equal(a[k], b[k]) for k in COLS)


def test_format_parse_round_trip():
    cols = q.generate_host(31, 0, 50_000)
    text = q.tbl_format(cols)
    assert text.count(b"\n") == 50_000 and text.endswith(b"|\n")
    parsed, rows, bad, _ = O.parse_tbl(text)
    assert rows == 50_000 and bad == 0
    assert same(parsed, cols)


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent")
def test_restatement_matches_reference_value_types():
    cols = q.generate_host(32, 1000, 20_000)
    text = q.tbl_format(cols, first_row=1000)
    mine, rows, bad, _ = O.parse_tbl(text)
    ref, rrows = O.ref_parse_tbl(text)
    assert rows == rrows == 20_000 and bad == 0
    assert same(mine, ref)


QUIRKS = (b"1|2|3|4|17.5|100|-0.04|+3|R|F|1992-02-29|x|y|z|\n"
          b"1|2|3|4|17|12345.67|0.1|0.08|N|O|2000-02-29|\n"
          b"9|9|9|9|-1.05|0.00|0.10|0.00|A|F|1998-12-31|tail\n"
          b"1|2|3|4|50.00|104949.50|0.10|0.08|N|O|1995-06-17|no newline at the end")


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent")
def test_value_quirks_match_reference():
    """The fraction's digits are an integer ("17.5" is 1705, as in the reference), signs and
    missing fractions are accepted, fields after the eleventh are ignored, the last line may lack
    its newline."""
    mine, rows, bad, _ = O.parse_tbl(QUIRKS)
    ref, rrows = O.ref_parse_tbl(QUIRKS)
    assert rows == rrows == 4 and bad == 0
    assert same(mine, ref)
    assert list(mine["quantity"]) == [1705, 1700, -95, 5000]


def test_dates_match_calendar():
    """Day numbers: MonetDB's count, i.e. Python's proleptic ordinal + 365 (1992-01-01 = 727563)."""
    days = [datetime.date(1992, 1, 1), datetime.date(1992, 2, 29), datetime.date(1900, 3, 1),
            datetime.date(2000, 2, 29), datetime.date(1998, 9, 2), datetime.date(1, 1, 1), datetime.date(9999, 12, 31)]
    n = len(days)
    cols = {"shipdate": np.array([d.toordinal() + 365 for d in days], np.int32),
            "quantity": np.full(n, 100, np.int64), "extendedprice": np.full(n, 100, np.int64),
            "discount": np.zeros(n, np.int64), "tax": np.zeros(n, np.int64),
            "returnflag": np.full(n, b"A", "S1"), "linestatus": np.full(n, b"F", "S1")}
    text = q.tbl_format(cols)
    lines = text.decode().splitlines()
    assert [ln.split("|")[10] for ln in lines] == [d.isoformat() for d in days]
    parsed, rows, bad, _ = O.parse_tbl(text)
    assert bad == 0 and np.array_equal(parsed["shipdate"], cols["shipdate"])
    assert cols["shipdate"][0] == 727563 and cols["shipdate"][4] == 729999


def test_oracle_flags_malformed_lines():
    good = q.tbl_format(q.generate_host(33, 0, 10))
    lines = good.split(b"\n")[:-1]
    lines[3] = b"1|2|3|4|x|1.00|0.01|0.02|R|F|1994-01-01|"       # bad decimal
    lines[7] = b"1|2|3|4|1.00|1.00|0.01|0.02|RR|F|1994-01-01|"   # two-character flag
    text = b"\n".join(lines) + b"\n" + b"\n" + b"1|2|3|4|1|1|0|0|A|F|1994-02-30|\n"   # empty line, 30 February
    cols, rows, bad, first = O.parse_tbl(text)
    assert rows == 12 and bad == 4
    assert first == len(b"\n".join(lines[:3])) + 1
    assert cols["quantity"][3] == 0 and cols["returnflag"][7] == b""
