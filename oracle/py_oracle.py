"""ctypes access to the oracle (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs import this
module; the product never does.

  liboracle.so       plain-C restatement of the reference's algorithm (oracle/q1_oracle.c)
  _ref/libq1ref.so   the reference's own CPU kernels (KernelHyPer, KernelX100), compiled from the
                     reference sources by oracle/Makefile
Results are numpy arrays of shape (groups, 6) holding Python ints (exact 128-bit values), in the
aggregate order count, sum_qty (hundredths), sum_base_price, sum_disc, sum_disc_price, sum_charge.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NG, NA = 6, 6

_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} (run make -C oracle)")
        _lib = ctypes.CDLL(path)
    return _lib


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libq1ref.so"))


def ref():
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libq1ref.so")
        if not os.path.exists(path):
            raise RuntimeError(f"reference oracle not built: {path}")
        r = ctypes.CDLL(path)
        r.q1ref_table_new.restype = ctypes.c_void_p
        r.q1ref_table_new.argtypes = [ctypes.c_uint64]
        r.q1ref_table_free.argtypes = [ctypes.c_void_p]
        r.q1ref_table_push.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 7 + [ctypes.c_uint64, ctypes.c_int32]
        r.q1ref_table_rows.restype = ctypes.c_uint64
        r.q1ref_table_rows.argtypes = [ctypes.c_void_p]
        r.q1ref_hyper.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        r.q1ref_x100.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p]
        r.q1ref_pool_new.restype = ctypes.c_void_p
        r.q1ref_pool_new.argtypes = [ctypes.c_void_p, ctypes.c_int]
        r.q1ref_pool_run.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p]
        r.q1ref_pool_threads.argtypes = [ctypes.c_void_p]
        r.q1ref_pool_free.argtypes = [ctypes.c_void_p]
        r.q1ref_table_generate.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                           ctypes.c_int32]
        r.q1ref_chunks_new.restype = ctypes.c_void_p
        r.q1ref_chunks_new.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                       ctypes.c_int32, ctypes.c_int]
        r.q1ref_chunks_run.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        r.q1ref_chunks_threads.argtypes = [ctypes.c_void_p]
        r.q1ref_chunks_count.restype = ctypes.c_uint64
        r.q1ref_chunks_count.argtypes = [ctypes.c_void_p]
        r.q1ref_chunks_free.argtypes = [ctypes.c_void_p]
        _ref = r
    return _ref


def ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def i128_to_ints(buf, groups):
    """Decode a little-endian int128 buffer of shape (groups*6*2) uint64 into Python ints."""
    u = buf.reshape(groups, NA, 2)
    out = np.empty((groups, NA), dtype=object)
    for g in range(groups):
        for a in range(NA):
            v = int(u[g, a, 0]) | (int(u[g, a, 1]) << 64)
            if v >= 1 << 127:
                v -= 1 << 128
            out[g, a] = v
    return out


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def generate(seed, first_row, rows, threads=None):
    """Reference-typed columns of the seeded generator (oracle/gen_rows.h), built by the oracle
    itself: int32 day numbers, int64 hundredths / cents, one-byte flags."""
    threads = threads or os.cpu_count() or 1
    c = {"shipdate": np.empty(rows, np.int32), "quantity": np.empty(rows, np.int64),
         "extendedprice": np.empty(rows, np.int64), "discount": np.empty(rows, np.int64),
         "tax": np.empty(rows, np.int64), "returnflag": np.empty(rows, "S1"), "linestatus": np.empty(rows, "S1")}
    L = lib()
    L.oracle_generate.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int] + [ctypes.c_void_p] * 7
    L.oracle_generate(seed, first_row, rows, threads, *[ptr(c[k]) for k in ["shipdate", "quantity", "extendedprice",
                                                                            "discount", "tax", "returnflag",
                                                                            "linestatus"]])
    return c


def q1_uncompressed(cols, cutoff_day=729999):
    n = len(cols["shipdate"])
    buf = np.zeros(NG * NA * 2, dtype=np.uint64)
    L = lib()
    L.oracle_q1_uncompressed.argtypes = [ctypes.c_void_p] * 7 + [ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p]
    keep = [_c(cols["shipdate"], np.int32), _c(cols["discount"], np.int64), _c(cols["extendedprice"], np.int64),
            _c(cols["tax"], np.int64), _c(cols["quantity"], np.int64),
            _c(cols["returnflag"].view(np.uint8), np.uint8), _c(cols["linestatus"].view(np.uint8), np.uint8)]
    flag = L.oracle_q1_uncompressed(*[ptr(k) for k in keep], n, cutoff_day, ptr(buf))
    return i128_to_ints(buf, NG), flag


def q1_compressed(c, cutoff_day=729999, use_filter=False):
    n = len(c["shipdate"])
    buf = np.zeros(NG * NA * 2, dtype=np.uint64)
    L = lib()
    L.oracle_q1_compressed.argtypes = ([ctypes.c_void_p] * 5 + [ctypes.c_int] + [ctypes.c_void_p] * 5 +
                                       [ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p])
    pair = "flags" in c
    filt = c.get("filter") if use_filter else None
    keep = [_c(c["shipdate"], np.uint16), _c(c["discount"], np.uint8), _c(c["extendedprice"], np.uint32),
            _c(c["tax"], np.uint8), _c(c["quantity"], np.uint8)]
    flags = _c(c["flags"], np.uint32) if pair else None
    pg = _c(c["pair_group"], np.uint8) if pair else None
    rf = None if pair else _c(c["returnflag"], np.uint32)
    ls = None if pair else _c(c["linestatus"], np.uint32)
    fl = None if filt is None else _c(filt, np.uint32)
    flag = L.oracle_q1_compressed(*[ptr(k) for k in keep], 0 if pair else 1, ptr(flags), ptr(pg), ptr(rf), ptr(ls),
                                  ptr(fl), n, cutoff_day, ptr(buf))
    return i128_to_ints(buf, NG), flag


def q1_groupkey(c, keys, num_groups, cutoff_day=729999):
    n = len(c["shipdate"])
    buf = np.zeros(num_groups * NA * 2, dtype=np.uint64)
    L = lib()
    L.oracle_q1_groupkey.argtypes = ([ctypes.c_void_p] * 6 + [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32,
                                                              ctypes.c_void_p])
    keep = [_c(c["shipdate"], np.uint16), _c(c["discount"], np.uint8), _c(c["extendedprice"], np.uint32),
            _c(c["tax"], np.uint8), _c(c["quantity"], np.uint8), _c(keys, np.uint32)]
    flag = L.oracle_q1_groupkey(*[ptr(k) for k in keep], num_groups, n, cutoff_day, ptr(buf))
    return buf.view(np.uint64), flag


def groupkey_ints(buf, num_groups):
    return i128_to_ints(buf, num_groups)


def precompute_filter(c_shipdate, cutoff_day):
    n = len(c_shipdate)
    out = np.zeros((n + 31) // 32, dtype=np.uint32)
    L = lib()
    L.oracle_precompute_filter.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p]
    s = _c(c_shipdate, np.uint16)
    L.oracle_precompute_filter(ptr(s), n, cutoff_day, ptr(out))
    return out


# KernelHyPerCompact compares the compact ship date (ship - 727563 under -DGPU) with the int16
# truncation of the cutoff day (729999 -> 9103): pushing the table with cutoff_day - 6667 makes it
# evaluate ship <= cutoff_day.
HYPER_COMPACT_SHIFT = 6667


class RefTable:
    """The reference's lineitem (cpu/tpch_kit.hpp:135-149) filled through Column::Push."""

    def __init__(self, cols, cutoff_day=729999):
        r = ref()
        n = len(cols["shipdate"])
        self.n = n
        self.h = r.q1ref_table_new(n + 1)
        self.pool = None
        if n == 0:
            return
        keep = [_c(cols["shipdate"], np.int32), _c(cols["discount"], np.int64), _c(cols["extendedprice"], np.int64),
                _c(cols["tax"], np.int64), _c(cols["quantity"], np.int64),
                _c(cols["returnflag"].view(np.uint8), np.uint8), _c(cols["linestatus"].view(np.uint8), np.uint8)]
        r.q1ref_table_push(self.h, *[ptr(k) for k in keep], n, cutoff_day)

    @classmethod
    def generated(cls, seed, first_row, rows, cutoff_day=729999):
        """A table of generator rows pushed by the reference bridge itself (no numpy copy)."""
        t = cls.__new__(cls)
        t.n = rows
        t.pool = None
        t.h = ref().q1ref_table_new(rows + 1)
        ref().q1ref_table_generate(t.h, seed, first_row, rows, cutoff_day)
        return t

    def hyper(self):
        buf = np.zeros(NG * NA * 2, dtype=np.uint64)
        flag = ref().q1ref_hyper(self.h, ptr(buf))
        return i128_to_ints(buf, NG), flag

    def hyper_compact(self):
        """KernelHyPerCompact<true>; the table must have been pushed with HYPER_COMPACT_SHIFT
        subtracted from the cutoff day (see q1ref_hyper_compact)."""
        r = ref()
        r.q1ref_hyper_compact.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        buf = np.zeros(NG * NA * 2, dtype=np.uint64)
        flag = r.q1ref_hyper_compact(self.h, ptr(buf))
        return i128_to_ints(buf, NG), flag

    def x100(self, offset=0, num=None):
        num = self.n - offset if num is None else num
        buf = np.zeros(NG * NA * 2, dtype=np.uint64)
        rc = ref().q1ref_x100(self.h, offset, num, ptr(buf))
        return i128_to_ints(buf, NG), rc

    def x100_parallel(self, threads, offset=0, num=None, morsel=1 << 16):
        num = self.n - offset if num is None else num
        if self.pool is None:
            self.pool = ref().q1ref_pool_new(self.h, threads)
        buf = np.zeros(NG * NA * 2, dtype=np.uint64)
        rc = ref().q1ref_pool_run(self.pool, offset, num, morsel, ptr(buf))
        return i128_to_ints(buf, NG), rc

    def threads(self):
        return ref().q1ref_pool_threads(self.pool) if self.pool else 0

    def close(self):
        if self.pool is not None:
            ref().q1ref_pool_free(self.pool)
            self.pool = None
        if self.h:
            ref().q1ref_table_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefChunks:
    """The reference's KernelX100 over rows [first_row, first_row + rows) of the generator, held
    as chunks of compact copies (12 B/row; see q1ref_chunks_new) and run on `threads` threads."""

    def __init__(self, seed, first_row, rows, chunk_rows=1 << 25, cutoff_day=729999, threads=None):
        threads = threads or os.cpu_count() or 1
        self.rows = rows
        self.h = ref().q1ref_chunks_new(seed, first_row, rows, chunk_rows, cutoff_day, threads)
        if not self.h:
            raise ValueError("RefChunks needs at least one row")

    def run(self, morsel=1 << 16):
        buf = np.zeros(NG * NA * 2, dtype=np.uint64)
        rc = ref().q1ref_chunks_run(self.h, morsel, ptr(buf))
        return i128_to_ints(buf, NG), rc

    def threads(self):
        return ref().q1ref_chunks_threads(self.h)

    def chunks(self):
        return int(ref().q1ref_chunks_count(self.h))

    def close(self):
        if self.h:
            ref().q1ref_chunks_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _tbl_cols(rows):
    return {"shipdate": np.zeros(rows, np.int32), "quantity": np.zeros(rows, np.int64),
            "extendedprice": np.zeros(rows, np.int64), "discount": np.zeros(rows, np.int64),
            "tax": np.zeros(rows, np.int64), "returnflag": np.zeros(rows, "S1"), "linestatus": np.zeros(rows, "S1")}


def _tbl_ptrs(c):
    return [ptr(c[k]) for k in ["shipdate", "quantity", "extendedprice", "discount", "tax", "returnflag", "linestatus"]]


def parse_tbl(text, capacity=None):
    """The restatement's .tbl parse: (columns, rows, malformed lines, first malformed byte)."""
    L = lib()
    L.oracle_parse_tbl.restype = ctypes.c_uint64
    L.oracle_parse_tbl.argtypes = [ctypes.c_char_p, ctypes.c_uint64] + [ctypes.c_void_p] * 7 + [
        ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    if capacity is None:
        capacity = text.count(b"\n") + 1
    c = _tbl_cols(capacity)
    bad, first = ctypes.c_uint64(0), ctypes.c_uint64(0)
    rows = L.oracle_parse_tbl(text, len(text), *_tbl_ptrs(c), capacity, ctypes.byref(bad), ctypes.byref(first))
    n = min(rows, capacity)
    return {k: v[:n] for k, v in c.items()}, rows, bad.value, first.value


def ref_parse_tbl(text):
    """The reference's own value types (Decimal<15,2>, Char, Date) over well-formed .tbl text."""
    r = ref()
    r.q1ref_parse_tbl.restype = ctypes.c_uint64
    r.q1ref_parse_tbl.argtypes = [ctypes.c_char_p, ctypes.c_uint64] + [ctypes.c_void_p] * 7 + [ctypes.c_uint64]
    capacity = text.count(b"\n") + 1
    c = _tbl_cols(capacity)
    rows = r.q1ref_parse_tbl(text, len(text), *_tbl_ptrs(c), capacity)
    return {k: v[:rows] for k, v in c.items()}, rows
