"""Host logic of the product (no GPU compute): generator, compressor, filter bitmap, placement
names, parameter validation, result finalisation. Every check is against an independent
restatement (tests/gen_np.py) or the oracle."""
import ctypes

import numpy as np
import pytest

import gen_np
import tpchq01_gpu_b200 as q
from oracle import py_oracle as O
from tpchq01_gpu_b200 import _lib


@pytest.mark.parametrize("seed,first,rows", [(1, 0, 1), (7, 100, 100_000), (20260101, 5_000_000, 33_333)])
def test_host_generator_equals_numpy_restatement(seed, first, rows):
    a = q.generate_host(seed, first, rows)
    b = gen_np.generate(seed, first, rows)
    for k in b:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


def test_generator_distribution_matches_spec():
    c = gen_np.generate(99, 0, 200_000)
    ship = c["shipdate"]
    assert ship.min() >= 727563 + 1 and ship.max() <= 729968 + 121
    assert set(np.unique(c["discount"])) <= set(range(11))
    assert set(np.unique(c["tax"])) <= set(range(9))
    assert set(np.unique(c["quantity"] // 100)) == set(range(1, 51))
    pairs = set(zip(c["returnflag"].tolist(), c["linestatus"].tolist()))
    assert pairs == {(b"A", b"F"), (b"N", b"F"), (b"N", b"O"), (b"R", b"F")}


@pytest.mark.parametrize("packing", ["pair", "separate"])
def test_compressor_equals_restatement(packing):
    cols = gen_np.generate(5, 0, 50_001)
    got, st = q.compress_host(cols, packing)
    ref = gen_np.compress(cols, "pair" if packing == "pair" else "sep")
    for k, v in ref.items():
        if k == "num_pair_codes":
            assert got[k] == v
        else:
            assert np.array_equal(np.asarray(got[k]), np.asarray(v)), k
    assert st.rows == 50_001 and st.max_discount <= 10 and st.max_quantity <= 50
    if packing == "separate":
        # also equal to the oracle's restatement of src/main.cu:773-803
        n = 50_001
        bufs = dict(s=np.zeros(n, np.uint16), d=np.zeros(n, np.uint8), p=np.zeros(n, np.uint32),
                    t=np.zeros(n, np.uint8), q=np.zeros(n, np.uint8), rf=np.zeros((n + 15) // 16, np.uint32),
                    ls=np.zeros((n + 31) // 32, np.uint32))
        L = O.lib()
        L.oracle_compress_separate.argtypes = [ctypes.c_void_p] * 7 + [ctypes.c_uint64] + [ctypes.c_void_p] * 7
        keep = [cols["shipdate"], cols["discount"], cols["extendedprice"], cols["tax"], cols["quantity"],
                cols["returnflag"].view(np.uint8), cols["linestatus"].view(np.uint8)]
        bad = L.oracle_compress_separate(*[O.ptr(k) for k in keep], n, *[O.ptr(bufs[k]) for k in
                                                                          ["s", "d", "p", "t", "q", "rf", "ls"]])
        assert bad == 0
        assert np.array_equal(bufs["rf"], got["returnflag"]) and np.array_equal(bufs["ls"], got["linestatus"])


@pytest.mark.parametrize("field,value,msg", [
    ("discount", 101, "discount"), ("tax", 300, "tax"), ("quantity", 150, "quantity"),
    ("shipdate", 727000, "shipdate"), ("extendedprice", 1 << 33, "extendedprice"), ("returnflag", b"X", "returnflag")])
def test_compressor_rejects_out_of_domain(field, value, msg):
    cols = gen_np.generate(6, 0, 100)
    cols[field][42] = value
    with pytest.raises(q.Q1Error) as e:
        q.compress_host(cols, "pair")
    assert e.value.status == 6 and msg in e.value.message and "row 42" in e.value.message


def test_pair_packing_rejects_more_than_four_combinations():
    cols = gen_np.generate(6, 0, 100)
    cols["returnflag"][0], cols["linestatus"][0] = b"A", b"O"
    cols["returnflag"][1], cols["linestatus"][1] = b"R", b"O"
    with pytest.raises(q.Q1Error):
        q.compress_host(cols, "pair")
    q.compress_host(cols, "separate")


def test_filter_bitmap_host():
    cols = gen_np.generate(8, 0, 10_007)
    c = gen_np.compress(cols)
    for cut in [727000, 728826, 729999, 731000]:
        assert np.array_equal(q.precompute_filter_host(c["shipdate"], cut), gen_np.filter_bitmap(c["shipdate"], cut))


@pytest.mark.parametrize("name,idx", [("in_registers", 0), ("in-registers", 0), ("in_registers_per_thread", 1),
                                      ("local_mem", 2), ("local-mem", 2), ("shared_mem_per_thread", 3),
                                      ("per-thread-shared-mem", 3), ("global", 4)])
def test_placement_names_both_spellings(name, idx):
    assert q.placement_id(name) == idx


def test_unknown_placement_message():
    with pytest.raises(q.Q1Error) as e:
        q.placement_id("shared_mem")
    assert 'No kernel variant named "shared_mem"' in e.value.message


@pytest.mark.parametrize("kw,fragment", [
    (dict(use_filter_pushdown=True), "only currently supported when compression is applied"),
    (dict(num_threads_per_block=100), "multiples of the warp size"),
    (dict(num_query_execution_runs=0), "Number of runs must be positive"),
    (dict(cpu_processing_fraction=1.5), "range 0.0 - 1.0"),
    (dict(num_tuples_per_kernel_launch=1000), "multiple of 128"),
    (dict(num_gpu_streams=0), "streams"),
])
def test_params_validation_like_reference(kw, fragment):
    with pytest.raises(q.Q1Error) as e:
        q.Q1Params(**kw).validate()
    assert fragment in e.value.message


def test_params_defaults_are_reference_defaults():
    p = _lib.Params()
    q.lib().q1_params_default(ctypes.byref(p))
    assert p.placement == 1 and p.streams == 4 and p.tuples_per_launch == 1 << 21 and p.runs == 5
    assert p.cpu_fraction == 0.5 and p.cutoff_day == 729999
    q.Q1Params(apply_compression=True, use_filter_pushdown=True).validate()


def test_finalize_averages_truncate_toward_zero():
    aggs = (_lib.I128 * 36)()
    def put(g, a, v):
        v &= (1 << 128) - 1
        aggs[g * 6 + a].lo = v & ((1 << 64) - 1)
        aggs[g * 6 + a].hi = v >> 64
    put(0, 0, 3); put(0, 1, 1000); put(0, 2, -1000); put(0, 3, 7)
    put(1, 0, 0); put(1, 1, 5)
    out = (_lib.GroupResult * 6)()
    _lib.check(q.lib().q1_finalize_groups(aggs, 6, out))
    assert out[0].avg_qty_e4 == 33333 and out[0].avg_price_e4 == -33333 and out[0].avg_disc_e4 == 233
    assert out[1].avg_qty_e4 == 0 and out[0].returnflag == b"A" and out[3].linestatus == b"O"
    assert out[0].sum_base_price.value() == -1000


def _host_cols(c):
    """q1_compressed_columns over the numpy arrays of a compressed dict (host memory)."""
    cc = _lib.CompressedColumns()
    for k in ["shipdate", "discount", "extendedprice", "tax", "quantity"]:
        setattr(cc, k, c[k].ctypes.data)
    if "flags" in c:
        cc.flags = c["flags"].ctypes.data
        cc.flag_packing = 0
        cc.num_pair_codes = c["num_pair_codes"]
        for i in range(4):
            cc.pair_group[i] = int(c["pair_group"][i])
    else:
        cc.returnflag = c["returnflag"].ctypes.data
        cc.linestatus = c["linestatus"].ctypes.data
        cc.flag_packing = 1
    return cc


def _edge_rows(c, seed, frac=0.02):
    """Copy with a fraction of rows at the edges of the domain the CPU share accepts: discount
    11..100, tax 9..255, prices up to 2^32 - 1, quantity 51..255 (the host kernel's slow steps)."""
    out = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in c.items()}
    rng = np.random.default_rng(seed)
    idx = rng.choice(len(out["shipdate"]), max(1, int(frac * len(out["shipdate"]))), replace=False)
    out["discount"][idx] = rng.integers(0, 101, len(idx))
    out["tax"][idx] = rng.integers(0, 256, len(idx))
    out["extendedprice"][idx] = rng.integers(0, 2**32, len(idx), dtype=np.uint64).astype(np.uint32)
    out["quantity"][idx] = rng.integers(0, 256, len(idx))
    return out


@pytest.mark.parametrize("packing", ["pair", "separate"])
@pytest.mark.parametrize("edges", [False, True])
@pytest.mark.parametrize("cutoff", [727000, 728000, 729999, 731000, 800000])
def test_cpu_share_equals_oracle(packing, edges, cutoff):
    """The coprocessing CPU share (q1_run's host kernel, vectorised on hosts that offer it) over
    three unaligned row ranges adds up to the oracle's table over the whole table."""
    rows = 300_017
    c = gen_np.compress(gen_np.generate(41, 0, rows), packing)
    if edges:
        c = _edge_rows(c, 5 + cutoff)
    cc = _host_cols(c)
    buf = np.zeros(6 * 6 * 2, dtype=np.uint64)
    for b, e in [(0, 37), (37, 150_001), (150_001, rows)]:
        _lib.check(q.lib().q1_selftest_cpu_share(ctypes.byref(cc), b, e, cutoff, ctypes.c_void_p(buf.ctypes.data)))
    want, flag = O.q1_compressed(c, cutoff)
    assert flag == 0
    assert np.array_equal(O.i128_to_ints(buf, 6), want)


def test_cpu_share_reports_out_of_domain():
    c = gen_np.compress(gen_np.generate(42, 0, 10_000), "pair")
    c["discount"][5000] = 101
    cc = _host_cols(c)
    buf = np.zeros(6 * 6 * 2, dtype=np.uint64)
    st = q.lib().q1_selftest_cpu_share(ctypes.byref(cc), 0, 10_000, 729999, ctypes.c_void_p(buf.ctypes.data))
    assert st == 6   # Q1_ERR_DOMAIN


def test_cpu_share_rejects_bad_arguments():
    c = gen_np.compress(gen_np.generate(43, 0, 1_000), "pair")
    buf = np.zeros(6 * 6 * 2, dtype=np.uint64)
    out = ctypes.c_void_p(buf.ctypes.data)
    L = q.lib()
    cc = _host_cols(c)
    assert L.q1_selftest_cpu_share(None, 0, 10, 729999, out) == 1
    assert L.q1_selftest_cpu_share(ctypes.byref(cc), 10, 5, 729999, out) == 1
    assert L.q1_selftest_cpu_share(ctypes.byref(cc), 5, 5, 729999, out) == 0   # empty range
    bad = _host_cols(c)
    bad.num_pair_codes = 0
    assert L.q1_selftest_cpu_share(ctypes.byref(bad), 0, 1_000, 729999, out) == 1
    bad = _host_cols(c)
    bad.pair_group[0] = 6
    assert L.q1_selftest_cpu_share(ctypes.byref(bad), 0, 1_000, 729999, out) == 1
    bad = _host_cols(c)
    bad.flags = None
    assert L.q1_selftest_cpu_share(ctypes.byref(bad), 0, 1_000, 729999, out) == 1
    assert not buf.any()


@pytest.mark.parametrize("edges", [False, True])
@pytest.mark.parametrize("cutoff", [727000, 728000, 729999, 731000])
def test_cpu_share_uncompressed_equals_oracle(edges, cutoff):
    """The CPU share on reference-typed columns (vectorised on hosts that offer it) over three
    unaligned ranges adds up to the oracle's table; with edges, some rows carry values at the edges
    of the domain (discount 100, tax 255, prices and quantities up to 2^32 - 1)."""
    rows = 200_003
    cols = gen_np.generate(44, 0, rows)
    cols = {k: np.ascontiguousarray(v) for k, v in cols.items()}
    if edges:
        rng = np.random.default_rng(cutoff)
        idx = rng.choice(rows, rows // 50, replace=False)
        cols["discount"][idx] = rng.integers(0, 101, len(idx))
        cols["tax"][idx] = rng.integers(0, 256, len(idx))
        cols["extendedprice"][idx] = rng.integers(0, 2**32, len(idx))
        cols["quantity"][idx] = rng.integers(0, 2**32, len(idx))
    cc = _lib.Columns()
    for k in ["shipdate", "discount", "extendedprice", "tax", "quantity", "returnflag", "linestatus"]:
        setattr(cc, k, cols[k].ctypes.data)
    buf = np.zeros(6 * 6 * 2, dtype=np.uint64)
    for b, e in [(0, 13), (13, 100_001), (100_001, rows)]:
        _lib.check(q.lib().q1_selftest_cpu_share_uncompressed(ctypes.byref(cc), b, e, cutoff,
                                                               ctypes.c_void_p(buf.ctypes.data)))
    want, flag = O.q1_uncompressed(cols, cutoff)
    assert flag == 0
    assert np.array_equal(O.i128_to_ints(buf, 6), want)


def wide_rows(cols, seed, frac=0.03):
    """Replaces `frac` of the rows by reference-typed values beyond the fast domain that the
    reference's int64 arithmetic still takes without overflow: prices up to 2^40 and quantities up
    to 2^44 (both also negative), negative and above-100 discounts, taxes up to 1023 and negative
    ones; |(100 - d) p (100 + t)| stays below 2^63."""
    rng = np.random.default_rng(seed)
    n = len(cols["shipdate"])
    idx = rng.choice(n, int(frac * n), replace=False)
    k = len(idx)
    out = {key: np.ascontiguousarray(v).copy() for key, v in cols.items()}
    out["extendedprice"][idx] = rng.integers(-(1 << 40), 1 << 40, k)
    out["quantity"][idx] = rng.integers(-(1 << 40), 1 << 44, k)
    out["discount"][idx] = rng.integers(-4000, 4000, k)
    out["tax"][idx] = rng.integers(-1000, 1024, k)
    return out


def cpu_share_unc(cols, cutoff, ranges):
    cc = _lib.Columns()
    for k in ["shipdate", "discount", "extendedprice", "tax", "quantity", "returnflag", "linestatus"]:
        setattr(cc, k, cols[k].ctypes.data)
    buf = np.zeros(6 * 6 * 2, dtype=np.uint64)
    st = 0
    for b, e in ranges:
        st |= q.lib().q1_selftest_cpu_share_uncompressed(ctypes.byref(cc), b, e, cutoff, ctypes.c_void_p(buf.ctypes.data))
    return O.i128_to_ints(buf, 6), st


@pytest.mark.parametrize("cutoff", [728000, 729999])
def test_cpu_share_uncompressed_wide_values_equal_oracle(cutoff):
    """Reference-typed rows outside the kernels' fast domain are summed exactly (signed 128-bit),
    like the reference's KernelHyPer sums any int64 values whose products do not overflow."""
    rows = 100_003
    cols = wide_rows(gen_np.generate(45, 0, rows), cutoff)
    got, st = cpu_share_unc(cols, cutoff, [(0, 13), (13, 60_001), (60_001, rows)])
    want, flag = O.q1_uncompressed(cols, cutoff)
    assert flag == 0 and st == 0
    assert np.array_equal(got, want)
    assert min(int(want[g, 4]) for g in range(6)) < 0   # negative disc_price sums occur


def test_cpu_share_uncompressed_reports_int64_overflow():
    """A passing row whose charge overflows int64 (the reference's handle_overflow) is reported as
    Q1_ERR_DOMAIN, as the oracle flags it."""
    cols = {k: np.ascontiguousarray(v).copy() for k, v in gen_np.generate(46, 0, 1000).items()}
    i = int(np.argmax(cols["shipdate"] <= 729999))
    cols["extendedprice"][i] = 1 << 58
    got, st = cpu_share_unc(cols, 729999, [(0, 1000)])
    _, flag = O.q1_uncompressed(cols, 729999)
    assert flag == 1 and st == 6
