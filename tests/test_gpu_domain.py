"""The scan kernels over their whole declared value domain, against the oracle (tolerance 0).

The compressed kernels accept discount <= 100, tax <= 255, quantity <= 255 and prices < 2^32;
TPC-H data (and the generator) stays far inside that: prices < 2^24, tax <= 8, discount <= 10,
quantity <= 50. Here 5% of the generator's rows are replaced by rows from the whole domain, so
that the price's top byte plane (the warp vote's kTop branch in AccPerThread::add_quad) and the
wide tax / discount / quantity bytes run under test in every placement, both flag packings and
with filter pushdown off and on, plus the uncompressed (reference-typed) layout.

The exactness bound of the per-thread 32-bit partials (2^15 rows per consumer thread per launch,
which the host enforces by splitting launches at whole tiles) is pinned with one-CTA launches over
maximal bytes: 384 x 2^15 + 4099 rows give each consumer thread of the CTA (256, 320 or 384 of
them, by layout and placement) 2^15 rows in its first launch where the tile is 4096 rows, and
32,760 (the last whole tile below the bound) where it is 3840 or 4608 rows; further launches take
the ragged rest. A group's
sum_charge there passes 2^64, so the 128-bit carries of the warp, CTA and global reductions run
too."""
import numpy as np
import pytest
import torch

import gen_np
import tpchq01_gpu_b200 as q
from oracle import py_oracle as O
from tpchq01_gpu_b200 import _lib
from test_gpu_kernel_abi import aggs_buffer, dev, device_compressed, read

pytestmark = pytest.mark.gpu

PLACEMENTS = ["in_registers", "in_registers_per_thread", "local_mem", "shared_mem_per_thread", "global"]
ROWS = 400_003
CUTOFF = 729999


def edge_rows(cols, seed, frac=0.05):
    """Replaces `frac` of the rows' values by values from the whole compressed domain."""
    rng = np.random.default_rng(seed)
    n = len(cols["shipdate"])
    idx = rng.choice(n, int(frac * n), replace=False)
    k = len(idx)
    out = {key: v.copy() for key, v in cols.items()}
    out["extendedprice"][idx] = rng.integers(1 << 24, 1 << 32, k)
    out["tax"][idx] = rng.integers(9, 256, k)
    out["discount"][idx] = rng.integers(11, 101, k)
    out["quantity"][idx] = rng.integers(51, 256, k) * 100
    # a few rows at the exact corners
    c = idx[:8]
    out["extendedprice"][c] = (1 << 32) - 1
    out["tax"][c] = 255
    out["discount"][c[:4]] = 0
    out["discount"][c[4:]] = 100
    out["quantity"][c] = 25500
    return out


@pytest.fixture(scope="module")
def wide_cols():
    return edge_rows(gen_np.generate(606, 0, ROWS), 606)


def oracle_table(cols, cutoff=CUTOFF):
    t, flag = O.q1_uncompressed(cols, cutoff)
    assert flag == 0
    return t


@pytest.mark.parametrize("use_filter", [False, True])
@pytest.mark.parametrize("packing", ["pair", "sep"])
@pytest.mark.parametrize("placement", PLACEMENTS)
def test_compressed_whole_domain(cuda, wide_cols, placement, packing, use_filter):
    comp = gen_np.compress(wide_cols, packing)
    if use_filter:
        comp["filter"] = gen_np.filter_bitmap(comp["shipdate"], CUTOFF)
    c, keep = device_compressed(comp)
    buf = aggs_buffer()
    stream = torch.cuda.current_stream().cuda_stream
    q.launch_compressed(placement, c, ROWS, CUTOFF, use_filter, buf.data_ptr(), stream)
    q.sync_check(stream)
    want = oracle_table(wide_cols)
    assert np.array_equal(read(buf), want)
    assert max(int(want[g, 2]) for g in range(6)) > 1 << 40   # the wide prices were summed


@pytest.mark.parametrize("placement", PLACEMENTS)
def test_uncompressed_whole_domain(cuda, wide_cols, placement):
    keep = {k: dev(v) for k, v in wide_cols.items()}
    c = _lib.Columns(*[keep[k].data_ptr() for k in ["shipdate", "discount", "extendedprice", "tax", "quantity",
                                                    "returnflag", "linestatus"]])
    buf = aggs_buffer()
    stream = torch.cuda.current_stream().cuda_stream
    q.launch_uncompressed(placement, c, ROWS, CUTOFF, buf.data_ptr(), stream)
    q.sync_check(stream)
    assert np.array_equal(read(buf), oracle_table(wide_cols))


def maximal_rows(rows, seed):
    """Rows that all pass, with the largest bytes the domain allows: prices in [2^32 - 2^20, 2^32),
    quantity 255, tax 255 (ab's high byte at its largest with discount 0) and a sprinkling of
    discount-100 and other rows, over the generator's four (returnflag, linestatus) groups."""
    rng = np.random.default_rng(seed)
    cols = gen_np.generate(seed, 0, rows)
    cols["shipdate"][:] = 727600
    cols["extendedprice"] = rng.integers((1 << 32) - (1 << 20), 1 << 32, rows).astype(np.int64)
    cols["quantity"] = np.full(rows, 25500, np.int64)
    cols["tax"] = np.full(rows, 255, np.int64)
    disc = np.zeros(rows, np.int64)
    some = rng.random(rows) < 0.05
    disc[some] = rng.integers(0, 101, int(some.sum()))
    cols["discount"] = disc
    return cols


@pytest.fixture(scope="module")
def maximal():
    rows = 384 * (1 << 15) + 4099
    cols = maximal_rows(rows, 7)
    return cols, oracle_table(cols)


@pytest.mark.parametrize("placement", PLACEMENTS)
@pytest.mark.parametrize("packing", ["pair", "sep"])
def test_one_cta_at_the_per_thread_bound(cuda, maximal, placement, packing):
    cols, want = maximal
    rows = len(cols["shipdate"])
    # one group's sum_charge is past 2^64 (the CTA's 128-bit reductions carried into the high word)
    assert max(int(want[g, 5]) for g in range(6)) > 1 << 64
    comp = gen_np.compress(cols, packing)
    c, keep = device_compressed(comp)
    buf = aggs_buffer()
    stream = torch.cuda.current_stream().cuda_stream
    q.launch_compressed(placement, c, rows, CUTOFF, False, buf.data_ptr(), stream, config=_lib.LaunchConfig(0, 0, 1))
    q.sync_check(stream)
    assert np.array_equal(read(buf), want)


def test_default_grid_carries_past_2_64(cuda, maximal):
    """The same rows over the whole grid: the global 128-bit atomics carry between words."""
    cols, want = maximal
    comp = gen_np.compress(cols, "pair")
    c, keep = device_compressed(comp)
    buf = aggs_buffer()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(3):   # accumulating launches, no zeroing in between
        q.launch_compressed("in_registers_per_thread", c, len(cols["shipdate"]), CUTOFF, False, buf.data_ptr(), stream)
    q.sync_check(stream)
    assert np.array_equal(read(buf), 3 * want)


@pytest.fixture(scope="module")
def wide_unc():
    from test_host import wide_rows
    return wide_rows(gen_np.generate(607, 0, ROWS), 607)


@pytest.mark.parametrize("placement", PLACEMENTS)
def test_uncompressed_wide_values_summed_exactly(cuda, wide_unc, placement):
    """Reference-typed rows beyond the fast domain (negative or large int64 values whose products
    still fit int64) are summed exactly, as the reference's KernelHyPer sums them."""
    want, flag = O.q1_uncompressed(wide_unc, CUTOFF)
    assert flag == 0
    keep = {k: dev(v) for k, v in wide_unc.items()}
    c = _lib.Columns(*[keep[k].data_ptr() for k in ["shipdate", "discount", "extendedprice", "tax", "quantity",
                                                    "returnflag", "linestatus"]])
    buf = aggs_buffer()
    stream = torch.cuda.current_stream().cuda_stream
    q.launch_uncompressed(placement, c, ROWS, CUTOFF, buf.data_ptr(), stream)
    q.sync_check(stream)
    assert np.array_equal(read(buf), want)


@pytest.mark.parametrize("residency", ["hbm", "pinned"])
@pytest.mark.parametrize("fraction", [0.0, 0.4])
def test_uncompressed_wide_values_through_q1_run(cuda, wide_unc, fraction, residency):
    """The same rows through q1_run, HBM-resident and streamed from pinned host memory, GPU alone
    and with the CPU share of coprocessing."""
    want, _ = O.q1_uncompressed(wide_unc, CUTOFF)
    with q.Q1Context(cpu_threads=3) as ctx:
        ctx.load_columns(wide_unc, "uncompressed", "pair", residency)
        res = ctx.run(apply_compression=False, use_coprocessing=fraction > 0, cpu_processing_fraction=fraction,
                      num_tuples_per_kernel_launch=1 << 16, num_query_execution_runs=1)
    assert np.array_equal(res.table(), want)


def test_uncompressed_int64_overflow_is_reported(cuda):
    """A passing row whose charge overflows int64 (the reference's handle_overflow) is reported."""
    cols = {k: v.copy() for k, v in gen_np.generate(608, 0, 5000).items()}
    i = int(np.argmax(cols["shipdate"] <= CUTOFF))
    cols["extendedprice"][i] = 1 << 58
    assert O.q1_uncompressed(cols, CUTOFF)[1] == 1
    keep = {k: dev(v) for k, v in cols.items()}
    c = _lib.Columns(*[keep[k].data_ptr() for k in ["shipdate", "discount", "extendedprice", "tax", "quantity",
                                                    "returnflag", "linestatus"]])
    stream = torch.cuda.current_stream().cuda_stream
    q.launch_uncompressed("in_registers_per_thread", c, 5000, CUTOFF, aggs_buffer().data_ptr(), stream)
    with pytest.raises(q.Q1Error) as e:
        q.sync_check(stream)
    assert e.value.status == 6
