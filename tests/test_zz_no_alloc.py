"""q1_launch_compressed_noalloc: the scan launch for callers that may not allocate device memory.

Its scratch (a status word and one partial-sum record per CTA) is a static device array inside
libq1.so instead of memory obtained with cudaMalloc. Two calls in a row, on tables of different
sizes, must give exactly what q1_launch_compressed gives (integer aggregates: tolerance 0); the
second, smaller call also shows that the records left behind by the first are not summed again.
This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

import gen_np
import tpchq01_gpu_b200 as q
from tpchq01_gpu_b200 import _lib

pytestmark = pytest.mark.gpu


def to_device(comp):
    keep = {k: torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).copy()).cuda()
            for k, v in comp.items() if isinstance(v, np.ndarray) and k != "pair_group"}
    c = _lib.CompressedColumns()
    for k in ["shipdate", "discount", "extendedprice", "tax", "quantity", "flags", "returnflag", "linestatus"]:
        if k in keep:
            setattr(c, k, keep[k].data_ptr())
    c.flag_packing = 0 if "flags" in comp else 1
    if "flags" in comp:
        c.num_pair_codes = comp["num_pair_codes"]
        for i in range(4):
            c.pair_group[i] = int(comp["pair_group"][i])
    return c, keep


def run(entry, c, rows, cutoff, stream):
    out = torch.zeros(36 * 2, dtype=torch.int64, device="cuda")
    cfg = _lib.LaunchConfig(0, 0, 0)
    _lib.check(entry(1, ctypes.byref(c), rows, cutoff, 0, ctypes.byref(cfg), ctypes.c_void_p(out.data_ptr()),
                     ctypes.c_void_p(stream)))
    _lib.check(q.lib().q1_sync_check(ctypes.c_void_p(stream)))
    torch.cuda.synchronize()
    return q.decode_aggregates(out.cpu().numpy().view(np.uint64))


@pytest.mark.parametrize("packing", ["pair", "sep"])
def test_noalloc_matches_allocating_entry_point_twice(packing):
    assert torch.cuda.is_available()
    L = q.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for seed, rows, cutoff in [(900, 1_200_001, 729999), (901, 100_003, 729906)]:
        comp = gen_np.compress(gen_np.generate(seed, 0, rows), packing)
        c, keep = to_device(comp)
        want = run(L.q1_launch_compressed, c, rows, cutoff, stream)
        got = run(L.q1_launch_compressed_noalloc, c, rows, cutoff, stream)
        assert np.array_equal(got, want)
        assert int(want[:, 0].sum()) > 0
