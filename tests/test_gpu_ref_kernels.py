"""The reference's own compressed GPU kernels (src/kernels/*, built unmodified for sm_100a into
oracle/_ref/libq1refgpu.so) are the same-box GPU comparator; this pins that they compute what
this library computes on the same separate-flags table: per group the count, whole-unit
quantity, price, discount, disc_price and charge (the reference's uint64 sums, which hold
exactly at this size)."""
import ctypes
import os

import numpy as np
import pytest
import torch

import gen_np
import tpchq01_gpu_b200 as q
from tpchq01_gpu_b200 import _lib

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ROWS = 1_000_003
SEED = 321


def ref_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libq1refgpu.so")
    if not os.path.exists(path):
        pytest.skip("reference GPU kernels not built (oracle/_ref/libq1refgpu.so)")
    R = ctypes.CDLL(path)
    R.refgpu_launch_compressed.restype = ctypes.c_int
    R.refgpu_launch_compressed.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 9 + [
        ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    return R


@pytest.fixture(scope="module")
def table(cuda):
    comp = gen_np.compress(gen_np.generate(SEED, 0, ROWS), packing="separate")
    dev = {k: torch.from_numpy(np.ascontiguousarray(comp[k]).view(np.uint8).copy()).cuda()
           for k in ["shipdate", "discount", "extendedprice", "tax", "quantity", "returnflag", "linestatus"]}
    filt = torch.from_numpy(gen_np.filter_bitmap(comp["shipdate"], 729999).view(np.uint8).copy()).cuda()
    return comp, dev, filt


def ours(dev, filt, pushdown, cutoff=729999):
    c = _lib.CompressedColumns()
    for k in ["shipdate", "discount", "extendedprice", "tax", "quantity", "returnflag", "linestatus"]:
        setattr(c, k, dev[k].data_ptr())
    c.filter = filt.data_ptr()
    c.flag_packing = 1
    out = torch.zeros(72, dtype=torch.int64, device="cuda")
    q.launch_compressed("in_registers_per_thread", c, ROWS, cutoff, pushdown, out.data_ptr(),
                        torch.cuda.current_stream().cuda_stream)
    q.sync_check(torch.cuda.current_stream().cuda_stream)
    return q.decode_aggregates(out.cpu().numpy().view(np.uint64))


@pytest.mark.parametrize("placement", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("pushdown", [0, 1])
def test_reference_gpu_kernels_match(table, placement, pushdown):
    R = ref_lib()
    comp, dev, filt = table
    sums = torch.zeros(32, dtype=torch.int64, device="cuda")
    counts = torch.zeros(8, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = R.refgpu_launch_compressed(placement, pushdown, sums.data_ptr(), counts.data_ptr(),
                                    (filt if pushdown else dev["shipdate"]).data_ptr(), dev["discount"].data_ptr(),
                                    dev["extendedprice"].data_ptr(), dev["tax"].data_ptr(), dev["quantity"].data_ptr(),
                                    dev["returnflag"].data_ptr(), dev["linestatus"].data_ptr(), ROWS, 256, 16, stream)
    assert rc == 0
    torch.cuda.synchronize()
    s = sums.cpu().numpy().view(np.uint64)
    n = counts.cpu().numpy().view(np.uint32)
    want = ours(dev, filt, pushdown)
    for g in range(6):
        # reference order: quantity (units), base_price, discounted_price, charge, discount
        got = [int(n[g]), int(s[g]) * 100, int(s[6 + g]), int(s[24 + g]), int(s[12 + g]), int(s[18 + g])]
        assert got == [int(v) for v in want[g]], f"group {g}"
