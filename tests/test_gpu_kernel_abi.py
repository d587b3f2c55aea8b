"""The kernel-level C ABI (q1_launch_compressed / q1_launch_uncompressed / q1_precompute_filter)
on caller-owned device memory (torch tensors), against the oracle. Like the reference kernels,
launches accumulate into a caller-zeroed aggregate buffer."""
import numpy as np
import pytest
import torch

import gen_np
import tpchq01_gpu_b200 as q
from oracle import py_oracle as O
from tpchq01_gpu_b200 import _lib

pytestmark = pytest.mark.gpu

PLACEMENTS = ["in_registers", "in_registers_per_thread", "local_mem", "shared_mem_per_thread", "global"]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()


def device_compressed(comp):
    keep = {k: dev(v) for k, v in comp.items() if isinstance(v, np.ndarray) and k != "pair_group"}
    c = _lib.CompressedColumns()
    for k in ["shipdate", "discount", "extendedprice", "tax", "quantity", "flags", "returnflag", "linestatus",
              "filter"]:
        if k in keep:
            setattr(c, k, keep[k].data_ptr())
    if "flags" in comp:
        c.flag_packing = 0
        c.num_pair_codes = comp["num_pair_codes"]
        for i in range(4):
            c.pair_group[i] = int(comp["pair_group"][i])
    else:
        c.flag_packing = 1
    return c, keep


def aggs_buffer(groups=6):
    return torch.zeros(groups * 6 * 2, dtype=torch.int64, device="cuda")


def read(buf, groups=6):
    torch.cuda.synchronize()
    return q.decode_aggregates(buf.cpu().numpy().view(np.uint64), groups)


@pytest.mark.parametrize("placement", PLACEMENTS)
@pytest.mark.parametrize("packing", ["pair", "sep"])
@pytest.mark.parametrize("use_filter", [False, True])
def test_launch_compressed(cuda, placement, packing, use_filter):
    cols = gen_np.generate(31, 0, 123_457)
    comp = gen_np.compress(cols, packing)
    cutoff = 729906
    if use_filter:
        comp["filter"] = gen_np.filter_bitmap(comp["shipdate"], cutoff)
    c, keep = device_compressed(comp)
    buf = aggs_buffer()
    stream = torch.cuda.current_stream().cuda_stream
    q.launch_compressed(placement, c, len(cols["shipdate"]), cutoff, use_filter, buf.data_ptr(), stream)
    q.sync_check(stream)
    assert np.array_equal(read(buf), O.q1_uncompressed(cols, cutoff)[0])


@pytest.mark.parametrize("placement", PLACEMENTS)
@pytest.mark.parametrize("packing", ["pair", "sep"])
@pytest.mark.parametrize("frac", [0.0005, 0.3])
@pytest.mark.parametrize("use_filter,wide", [(False, False), (True, False), (False, True)])
def test_all_six_flag_groups(cuda, placement, packing, frac, use_filter, wide):
    """Rows of the groups A/O and R/O (absent from TPC-H data) change some rows' line status to O:
    every placement must still sum all six (returnflag, linestatus) groups exactly, with filter
    pushdown too, and with a tenth of the rows carrying bytes from the whole compressed domain
    (prices up to 2^32 - 1, tax up to 255, discount up to 100, quantity up to 255)."""
    cols = gen_np.generate(32, 0, 200_003)
    rng = np.random.default_rng(int(frac * 1e4))
    if wide:
        n = len(cols["shipdate"])
        idx = rng.choice(n, n // 10, replace=False)
        cols["extendedprice"] = cols["extendedprice"].copy()
        cols["extendedprice"][idx] = rng.integers(1 << 24, 1 << 32, len(idx))
        for k, hi in [("tax", 256), ("discount", 101)]:
            cols[k] = cols[k].copy()
            cols[k][idx] = rng.integers(0, hi, len(idx))
        cols["quantity"] = cols["quantity"].copy()
        cols["quantity"][idx] = rng.integers(0, 256, len(idx)) * 100
    rf = cols["returnflag"].view(np.uint8)
    ls = cols["linestatus"].view(np.uint8).copy()
    idx = np.flatnonzero(rf != ord("N"))
    pick = rng.choice(idx, max(1, int(frac * len(idx))), replace=False)
    ls[pick] = ord("O")
    cols["linestatus"] = ls.view("S1")
    if packing == "pair":
        # the pair dictionary holds at most 4 combinations: keep A/F, N/F, N/O, A/O (drop R rows)
        keep = cols["returnflag"].view(np.uint8) != ord("R")
        cols = {k: v[keep] for k, v in cols.items()}
    comp = gen_np.compress(cols, packing)
    cutoff = 729999
    if use_filter:
        comp["filter"] = gen_np.filter_bitmap(comp["shipdate"], cutoff)
    c, keep_ = device_compressed(comp)
    buf = aggs_buffer()
    stream = torch.cuda.current_stream().cuda_stream
    q.launch_compressed(placement, c, len(cols["shipdate"]), cutoff, use_filter, buf.data_ptr(), stream)
    q.sync_check(stream)
    want, flag = O.q1_compressed(comp, cutoff)
    assert flag == 0
    assert np.array_equal(read(buf), want)
    g = read(buf)
    assert g[1][0] > 0   # A/O rows counted


@pytest.mark.parametrize("placement", PLACEMENTS)
def test_launch_uncompressed_accumulates_like_reference(cuda, placement):
    cols = gen_np.generate(32, 0, 54_321)
    keep = {k: dev(v) for k, v in cols.items()}
    c = _lib.Columns(*[keep[k].data_ptr() for k in ["shipdate", "discount", "extendedprice", "tax", "quantity",
                                                    "returnflag", "linestatus"]])
    buf = aggs_buffer()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):   # two launches, no zeroing in between: the sums double
        q.launch_uncompressed(placement, c, len(cols["shipdate"]), 729999, buf.data_ptr(), stream)
    q.sync_check(stream)
    assert np.array_equal(read(buf), 2 * O.q1_uncompressed(cols)[0])


def test_device_filter_precompute(cuda):
    cols = gen_np.generate(33, 0, 100_003)
    comp = gen_np.compress(cols)
    s = dev(comp["shipdate"])
    out = torch.zeros((100_003 + 31) // 32, dtype=torch.int32, device="cuda")
    for cut in [727000, 729999, 731000]:
        q.precompute_filter(s.data_ptr(), 100_003, cut, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), gen_np.filter_bitmap(comp["shipdate"], cut))


def test_out_of_domain_rows_are_reported(cuda):
    """A discount above 100 (the compressed kernels' domain) is flagged, not silently summed."""
    cols = gen_np.generate(34, 0, 10_000)
    comp = gen_np.compress(cols)
    comp["discount"][5000] = 150
    c, keep = device_compressed(comp)
    buf = aggs_buffer()
    stream = torch.cuda.current_stream().cuda_stream
    q.launch_compressed("in_registers_per_thread", c, 10_000, 729999, False, buf.data_ptr(), stream)
    with pytest.raises(q.Q1Error) as e:
        q.sync_check(stream)
    assert e.value.status == 6
    # the status word is cleared after being reported
    q.sync_check(stream)


def test_unaligned_columns_are_rejected(cuda):
    cols = gen_np.generate(35, 0, 1000)
    comp = gen_np.compress(cols)
    c, keep = device_compressed(comp)
    c.quantity = keep["quantity"].data_ptr() + 1
    with pytest.raises(q.Q1Error) as e:
        q.launch_compressed("in_registers_per_thread", c, 999, 729999, False, aggs_buffer().data_ptr(), 0)
    assert e.value.status == 1


def test_device_generator_matches_host(cuda):
    n = 1_000_037
    words16, words32 = (n + 15) // 16, (n + 31) // 32
    out = {"shipdate": torch.zeros(n, dtype=torch.int16, device="cuda"),
           "discount": torch.zeros(n, dtype=torch.uint8, device="cuda"),
           "extendedprice": torch.zeros(n, dtype=torch.int32, device="cuda"),
           "tax": torch.zeros(n, dtype=torch.uint8, device="cuda"),
           "quantity": torch.zeros(n, dtype=torch.uint8, device="cuda"),
           "flags": torch.zeros(words16, dtype=torch.int32, device="cuda"),
           "returnflag": torch.zeros(words16, dtype=torch.int32, device="cuda"),
           "linestatus": torch.zeros(words32, dtype=torch.int32, device="cuda")}
    ref_pair = gen_np.compress(gen_np.generate(9, 64, n), "pair")
    ref_sep = gen_np.compress(gen_np.generate(9, 64, n), "sep")
    import ctypes
    for packing in [0, 1]:
        o = _lib.CompressedHostOut(*[out[k].data_ptr() for k in ["shipdate", "discount", "extendedprice", "tax",
                                                                 "quantity", "flags", "returnflag", "linestatus"]])
        _lib.check(q.lib().q1_generate_compressed_device(9, 64, n, packing, ctypes.byref(o), None))
        torch.cuda.synchronize()
        ref = ref_pair if packing == 0 else ref_sep
        for k in ["shipdate", "discount", "extendedprice", "tax", "quantity"]:
            assert np.array_equal(out[k].cpu().numpy().view(ref[k].dtype), ref[k]), k
        if packing == 0:
            assert list(ref["pair_group"]) == [0, 2, 3, 4]
            assert np.array_equal(out["flags"].cpu().numpy().view(np.uint32), ref["flags"])
        else:
            assert np.array_equal(out["returnflag"].cpu().numpy().view(np.uint32), ref["returnflag"])
            assert np.array_equal(out["linestatus"].cpu().numpy().view(np.uint32), ref["linestatus"])
