"""Host-side mirror of the reference's Q1 operator surface, over the C ABI (include/q1.h).

Names follow the reference's q1_params_t (src/main.cu:205-240) and its command line
(src/main.cu:255-360): hash_table_placement, apply_compression, use_filter_pushdown,
use_coprocessing, cpu_processing_fraction, num_gpu_streams, num_threads_per_block,
num_tuples_per_thread, num_tuples_per_kernel_launch, num_query_execution_runs.
Invalid combinations raise Q1Error with the reference's messages.

Numbers are exact: every sum is a Python int (decoded from 128-bit two's complement).
"""
import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import Q1Error, check, lib

AGG_NAMES = ["count", "sum_qty", "sum_base_price", "sum_disc", "sum_disc_price", "sum_charge"]
LAYOUTS = {"uncompressed": _lib.LAYOUT_UNCOMPRESSED, "compressed": _lib.LAYOUT_COMPRESSED}
PACKINGS = {"pair": _lib.FLAGS_PAIR_2BIT, "separate": _lib.FLAGS_SEPARATE}
RESIDENCIES = {"hbm": _lib.RESIDENCY_HBM, "pinned": _lib.RESIDENCY_PINNED_HOST}


def placement_id(name):
    """Placement number from either spelling (src/main.cu:166-191 or README.md:47-58)."""
    if isinstance(name, int):
        return name
    out = ctypes.c_int(0)
    check(lib().q1_placement_from_name(name.encode(), ctypes.byref(out)))
    return out.value


@dataclass
class Q1Params:
    hash_table_placement: str = "in_registers_per_thread"
    apply_compression: bool = False
    use_filter_pushdown: bool = False
    use_coprocessing: bool = False
    cpu_processing_fraction: float = 0.5
    num_gpu_streams: int = 4
    num_threads_per_block: int = 0          # 0: tuned default
    num_tuples_per_thread: int = 0          # 0: tuned default
    num_tuples_per_kernel_launch: int = 1 << 21
    num_query_execution_runs: int = 5
    cutoff_day: int = 729999                # l_shipdate <= 1998-09-02

    def to_c(self):
        p = _lib.Params()
        lib().q1_params_default(ctypes.byref(p))
        p.placement = placement_id(self.hash_table_placement)
        p.apply_compression = int(bool(self.apply_compression))
        p.use_filter_pushdown = int(bool(self.use_filter_pushdown))
        p.use_coprocessing = int(bool(self.use_coprocessing))
        p.cpu_fraction = float(self.cpu_processing_fraction)
        p.streams = int(self.num_gpu_streams)
        p.threads_per_block = int(self.num_threads_per_block)
        p.tuples_per_thread = int(self.num_tuples_per_thread)
        p.tuples_per_launch = int(self.num_tuples_per_kernel_launch)
        p.runs = int(self.num_query_execution_runs)
        p.cutoff_day = int(self.cutoff_day)
        return p

    def validate(self):
        p = self.to_c()
        check(lib().q1_params_validate(ctypes.byref(p)))


class Q1Result:
    """Per-group exact aggregates of one run (the table print_results shows, src/main.cu:92-164)."""

    def __init__(self, c_result):
        self.raw = c_result
        self.groups = []
        for g in range(c_result.num_groups):
            r = c_result.groups[g]
            self.groups.append({
                "group": r.group, "returnflag": r.returnflag.decode(), "linestatus": r.linestatus.decode(),
                "count": int(r.count), "sum_qty": r.sum_qty.value(), "sum_base_price": r.sum_base_price.value(),
                "sum_disc": r.sum_disc.value(), "sum_disc_price": r.sum_disc_price.value(),
                "sum_charge": r.sum_charge.value(), "avg_qty_e4": int(r.avg_qty_e4),
                "avg_price_e4": int(r.avg_price_e4), "avg_disc_e4": int(r.avg_disc_e4)})
        self.rows_total = int(c_result.rows_total)
        self.rows_gpu = int(c_result.rows_gpu)
        self.rows_cpu = int(c_result.rows_cpu)
        self.ms_last_run = float(c_result.ms_last_run)
        self.ms_gpu_last_run = float(c_result.ms_gpu_last_run)

    def table(self):
        """[6 groups][6 aggregates] of Python ints (count, qty, base_price, disc, disc_price, charge)."""
        t = np.empty((len(self.groups), 6), dtype=object)
        for g, r in enumerate(self.groups):
            for a, name in enumerate(AGG_NAMES):
                t[g, a] = r[name]
        return t

    def format(self):
        def dec(v, scale=100):
            sign = "-" if v < 0 else ""
            v = abs(v)
            return f"{sign}{v // scale}.{v % scale:02d}"
        lines = ["|  RF | LS |  sum_quantity        |  sum_base_price      |  sum_disc_price      |"
                 "  sum_charge          | count      |"]
        for r in self.groups:
            if r["count"] == 0:
                continue
            lines.append(f"| # {r['returnflag']} | {r['linestatus']}  | {dec(r['sum_qty']):>20} | "
                         f"{dec(r['sum_base_price']):>20} | {dec(r['sum_disc_price'], 10000):>20} | "
                         f"{dec(r['sum_charge'], 1000000):>20} | {r['count']:>10} |")
        return "\n".join(lines)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Q1Context:
    """One GPU, one loaded lineitem table (q1_open / q1_load_columns / q1_run / q1_close)."""

    def __init__(self, device=0, cpu_threads=0):
        self._h = ctypes.c_void_p()
        opts = _lib.DeviceOpts(device, cpu_threads)
        check(lib().q1_open(ctypes.byref(self._h), ctypes.byref(opts)))

    def close(self):
        if self._h:
            lib().q1_close(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_columns(self, cols, layout="compressed", packing="pair", residency="hbm"):
        """cols: dict of reference-typed numpy columns (int32 shipdate, int64 hundredths, S1 flags)."""
        keep = {k: np.ascontiguousarray(v) for k, v in cols.items()}
        n = len(keep["shipdate"])
        c = _lib.Columns(_ptr(keep["shipdate"]), _ptr(keep["discount"]), _ptr(keep["extendedprice"]),
                         _ptr(keep["tax"]), _ptr(keep["quantity"]), _ptr(keep["returnflag"]),
                         _ptr(keep["linestatus"]))
        check(lib().q1_load_columns(self._h, ctypes.byref(c), n, LAYOUTS[layout], PACKINGS[packing],
                                    RESIDENCIES[residency]))

    def generate(self, seed, rows, first_row=0, layout="compressed", packing="pair", residency="hbm"):
        """Seeded synthetic table; compressed tables are generated on the device."""
        check(lib().q1_generate_table(self._h, seed, first_row, rows, LAYOUTS[layout], PACKINGS[packing],
                                      RESIDENCIES[residency]))

    def load_tbl(self, path, layout="compressed", packing="pair", residency="hbm"):
        """A lineitem .tbl file, parsed on the GPU; returns the row count."""
        n = ctypes.c_uint64(0)
        check(lib().q1_tbl_load(self._h, os.fsencode(path), LAYOUTS[layout], PACKINGS[packing],
                                RESIDENCIES[residency], ctypes.byref(n)))
        return n.value

    def run(self, params=None, **kw):
        params = params or Q1Params(**kw)
        p = params.to_c()
        res = _lib.Result()
        check(lib().q1_run(self._h, ctypes.byref(p), ctypes.byref(res)))
        return Q1Result(res)

    def run_times(self):
        n = ctypes.c_int32(0)
        check(lib().q1_run_times(self._h, None, None, 0, ctypes.byref(n)))
        wall = (ctypes.c_double * max(n.value, 1))()
        gpu = (ctypes.c_double * max(n.value, 1))()
        check(lib().q1_run_times(self._h, wall, gpu, n.value, ctypes.byref(n)))
        return list(wall[: n.value]), list(gpu[: n.value])

    def stats(self):
        s = _lib.ColumnStats()
        check(lib().q1_table_stats(self._h, ctypes.byref(s)))
        return s

    def table_columns(self):
        """(compressed CompressedColumns | None, uncompressed Columns | None, rows, layout, residency)."""
        comp = _lib.CompressedColumns()
        unc = _lib.Columns()
        rows = ctypes.c_uint64(0)
        layout = ctypes.c_int(0)
        res = ctypes.c_int(0)
        check(lib().q1_table_columns(self._h, ctypes.byref(comp), ctypes.byref(unc), ctypes.byref(rows),
                                     ctypes.byref(layout), ctypes.byref(res)))
        if layout.value == _lib.LAYOUT_COMPRESSED:
            return comp, None, rows.value, layout.value, res.value
        return None, unc, rows.value, layout.value, res.value


def launch_compressed(placement, dev_cols, rows, cutoff_day, use_filter, dev_aggregates, stream=0, config=None):
    """Kernel-level entry (q1_launch_compressed): dev_cols is a CompressedColumns of device pointers,
    dev_aggregates a device pointer to 6*6 zeroed int128; asynchronous on `stream`."""
    cfg = config or _lib.LaunchConfig(0, 0, 0)
    check(lib().q1_launch_compressed(placement_id(placement), ctypes.byref(dev_cols), rows, cutoff_day,
                                     int(bool(use_filter)), ctypes.byref(cfg), ctypes.c_void_p(dev_aggregates),
                                     ctypes.c_void_p(stream)))


def launch_uncompressed(placement, dev_cols, rows, cutoff_day, dev_aggregates, stream=0, config=None):
    cfg = config or _lib.LaunchConfig(0, 0, 0)
    check(lib().q1_launch_uncompressed(placement_id(placement), ctypes.byref(dev_cols), rows, cutoff_day,
                                       ctypes.byref(cfg), ctypes.c_void_p(dev_aggregates), ctypes.c_void_p(stream)))


def sync_check(stream=0):
    check(lib().q1_sync_check(ctypes.c_void_p(stream)))


def precompute_filter(dev_shipdate, rows, cutoff_day, dev_bitmap, stream=0):
    check(lib().q1_precompute_filter(ctypes.c_void_p(dev_shipdate), rows, cutoff_day, ctypes.c_void_p(dev_bitmap),
                                     ctypes.c_void_p(stream)))


def decode_aggregates(words, groups=6):
    """uint64 array [groups*6*2] (lo, hi) -> [groups][6] Python ints."""
    w = np.asarray(words, dtype=np.uint64).reshape(groups, 6, 2)
    out = np.empty((groups, 6), dtype=object)
    for g in range(groups):
        for a in range(6):
            v = int(w[g, a, 0]) | (int(w[g, a, 1]) << 64)
            out[g, a] = v - (1 << 128) if v >= (1 << 127) else v
    return out


def generate_host(seed, first_row, rows):
    """Reference-typed columns from the seeded generator (host, multi-threaded C++)."""
    cols = {
        "shipdate": np.empty(rows, np.int32), "discount": np.empty(rows, np.int64),
        "extendedprice": np.empty(rows, np.int64), "tax": np.empty(rows, np.int64),
        "quantity": np.empty(rows, np.int64), "returnflag": np.empty(rows, "S1"), "linestatus": np.empty(rows, "S1"),
    }
    c = _lib.Columns(_ptr(cols["shipdate"]), _ptr(cols["discount"]), _ptr(cols["extendedprice"]), _ptr(cols["tax"]),
                     _ptr(cols["quantity"]), _ptr(cols["returnflag"]), _ptr(cols["linestatus"]))
    check(lib().q1_generate_host(seed, first_row, rows, ctypes.byref(c)))
    return cols


def tbl_format(cols, first_row=0):
    """Reference-typed host columns as lineitem .tbl text (bytes)."""
    n = len(cols["shipdate"])
    c = _lib.Columns(_ptr(cols["shipdate"]), _ptr(cols["discount"]), _ptr(cols["extendedprice"]), _ptr(cols["tax"]),
                     _ptr(cols["quantity"]), _ptr(cols["returnflag"]), _ptr(cols["linestatus"]))
    size = ctypes.c_uint64(0)
    check(lib().q1_tbl_format(ctypes.byref(c), first_row, n, None, 0, ctypes.byref(size)))
    buf = np.empty(max(size.value, 1), np.uint8)
    check(lib().q1_tbl_format(ctypes.byref(c), first_row, n, _ptr(buf), size.value, ctypes.byref(size)))
    return buf[: size.value].tobytes()


def tbl_read_file(path):
    """Reference-typed host columns of a .tbl file, parsed on the current GPU."""
    n = ctypes.c_uint64(0)
    check(lib().q1_tbl_read_file(os.fsencode(path), None, 0, ctypes.byref(n)))
    rows = n.value
    cols = {
        "shipdate": np.empty(rows, np.int32), "discount": np.empty(rows, np.int64),
        "extendedprice": np.empty(rows, np.int64), "tax": np.empty(rows, np.int64),
        "quantity": np.empty(rows, np.int64), "returnflag": np.empty(rows, "S1"), "linestatus": np.empty(rows, "S1"),
    }
    o = _lib.ColumnsOut(_ptr(cols["shipdate"]), _ptr(cols["returnflag"]), _ptr(cols["linestatus"]),
                        _ptr(cols["discount"]), _ptr(cols["tax"]), _ptr(cols["extendedprice"]), _ptr(cols["quantity"]))
    check(lib().q1_tbl_read_file(os.fsencode(path), ctypes.byref(o), rows, ctypes.byref(n)))
    return cols


def compress_host(cols, packing="pair"):
    """Compressed columns (numpy) + stats from the product's host compressor."""
    n = len(cols["shipdate"])
    out = {
        "shipdate": np.zeros(n, np.uint16), "discount": np.zeros(n, np.uint8), "extendedprice": np.zeros(n, np.uint32),
        "tax": np.zeros(n, np.uint8), "quantity": np.zeros(n, np.uint8),
    }
    o = _lib.CompressedHostOut(_ptr(out["shipdate"]), _ptr(out["discount"]), _ptr(out["extendedprice"]),
                               _ptr(out["tax"]), _ptr(out["quantity"]), None, None, None)
    if packing == "pair":
        out["flags"] = np.zeros((n + 15) // 16, np.uint32)
        o.flags = _ptr(out["flags"])
    else:
        out["returnflag"] = np.zeros((n + 15) // 16, np.uint32)
        out["linestatus"] = np.zeros((n + 31) // 32, np.uint32)
        o.returnflag = _ptr(out["returnflag"])
        o.linestatus = _ptr(out["linestatus"])
    keep = {k: np.ascontiguousarray(v) for k, v in cols.items()}
    c = _lib.Columns(_ptr(keep["shipdate"]), _ptr(keep["discount"]), _ptr(keep["extendedprice"]), _ptr(keep["tax"]),
                     _ptr(keep["quantity"]), _ptr(keep["returnflag"]), _ptr(keep["linestatus"]))
    st = _lib.ColumnStats()
    check(lib().q1_compress_host(ctypes.byref(c), n, PACKINGS[packing], ctypes.byref(o), ctypes.byref(st)))
    if packing == "pair":
        out["pair_group"] = np.array(list(st.pair_group), dtype=np.uint8)
        out["num_pair_codes"] = int(st.num_pair_codes)
    return out, st


def precompute_filter_host(c_shipdate, cutoff_day):
    n = len(c_shipdate)
    out = np.zeros((n + 31) // 32, np.uint32)
    s = np.ascontiguousarray(c_shipdate, dtype=np.uint16)
    check(lib().q1_precompute_filter_host(_ptr(s), n, cutoff_day, _ptr(out)))
    return out


__all__ = ["Q1Context", "Q1Params", "Q1Result", "Q1Error", "launch_compressed", "launch_uncompressed", "sync_check",
           "precompute_filter", "decode_aggregates", "generate_host", "compress_host", "precompute_filter_host",
           "placement_id", "AGG_NAMES"]
