"""q1_launch_compressed_noalloc: the scan launch for callers that may not allocate device memory.

Its scratch (a status word and one partial-sum record per CTA) is a static device array inside
libq1.so instead of memory obtained with cudaMalloc. Two calls in a row, on tables of different
sizes, must give exactly what q1_launch_compressed gives (integer aggregates: tolerance 0); the
second, smaller call also shows that the records left behind by the first are not summed again.
Every placement, both flag packings and filter pushdown are covered, and one-CTA launches long
enough to be split into several chunks (which reuse the records chunk after chunk).
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

PLACEMENTS = ["in_registers", "in_registers_per_thread", "local_mem", "shared_mem_per_thread", "global"]


def to_device(comp):
    keep = {k: torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).copy()).cuda()
            for k, v in comp.items() if isinstance(v, np.ndarray) and k != "pair_group"}
    c = _lib.CompressedColumns()
    for k in ["shipdate", "discount", "extendedprice", "tax", "quantity", "flags", "returnflag", "linestatus",
              "filter"]:
        if k in keep:
            setattr(c, k, keep[k].data_ptr())
    c.flag_packing = 0 if "flags" in comp else 1
    if "flags" in comp:
        c.num_pair_codes = comp["num_pair_codes"]
        for i in range(4):
            c.pair_group[i] = int(comp["pair_group"][i])
    return c, keep


def run(entry, placement, c, rows, cutoff, use_filter, stream, blocks=0):
    out = torch.zeros(36 * 2, dtype=torch.int64, device="cuda")
    cfg = _lib.LaunchConfig(0, 0, blocks)
    _lib.check(entry(q.placement_id(placement), ctypes.byref(c), rows, cutoff, int(use_filter), ctypes.byref(cfg),
                     ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream)))
    _lib.check(q.lib().q1_sync_check(ctypes.c_void_p(stream)))
    torch.cuda.synchronize()
    return q.decode_aggregates(out.cpu().numpy().view(np.uint64))


def table(seed, rows, packing, cutoff, use_filter):
    comp = gen_np.compress(gen_np.generate(seed, 0, rows), packing)
    if use_filter:
        comp["filter"] = gen_np.filter_bitmap(comp["shipdate"], cutoff)
    return to_device(comp)


@pytest.mark.parametrize("use_filter", [False, True])
@pytest.mark.parametrize("packing", ["pair", "sep"])
@pytest.mark.parametrize("placement", PLACEMENTS)
def test_noalloc_matches_allocating_entry_point_twice(placement, packing, use_filter):
    assert torch.cuda.is_available()
    L = q.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for seed, rows, cutoff in [(900, 1_200_001, 729999), (901, 100_003, 729906)]:
        c, keep = table(seed, rows, packing, cutoff, use_filter)
        want = run(L.q1_launch_compressed, placement, c, rows, cutoff, use_filter, stream)
        got = run(L.q1_launch_compressed_noalloc, placement, c, rows, cutoff, use_filter, stream)
        assert np.array_equal(got, want)
        assert int(want[:, 0].sum()) > 0


@pytest.mark.parametrize("placement,rows", [("in_registers", 4_500_001), ("in_registers_per_thread", 12_600_007)])
def test_noalloc_one_cta_several_chunks(placement, rows):
    """One CTA: the host splits the rows into launches of whole tiles and at most 2^15 rows per
    accumulating lane (pair layout, 12 consumer warps, 4608-row tiles: 3,142,656 rows for
    in_registers' 96 lanes, 12,579,840 for in_registers_per_thread's 384), and every launch reuses
    the same record, then two such calls in a row."""
    L = q.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for seed, n in [(902, rows), (903, rows // 3)]:
        c, keep = table(seed, n, "pair", 729999, False)
        want = run(L.q1_launch_compressed, placement, c, n, 729999, False, stream, blocks=1)
        got = run(L.q1_launch_compressed_noalloc, placement, c, n, 729999, False, stream, blocks=1)
        assert np.array_equal(got, want)
