"""Batched aggregation (q1_batch_*): many instances in one persistent kernel over a device tile
queue, replayed as a CUDA graph, placements chosen by the autotuner. Every instance's result
must equal the oracle and the plain per-instance launch (q1_launch_groupkey) bit for bit."""
import ctypes
import os

import numpy as np
import pytest
import torch

import gen_np
import tpchq01_gpu_b200 as q
from oracle import py_oracle as O
from tpchq01_gpu_b200 import _lib

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 100, 2047, 2048, 2049, 4096 + 3, 10_000, 65_537, 300_011, 1_000_003]
GROUPS = [1, 4, 8, 64, 1024, 3000]


def make_instances(seed=77, n=30):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        rows = SIZES[i % len(SIZES)]
        g = GROUPS[(i * 7) % len(GROUPS)]
        cutoff = int(rng.integers(729906, 730090)) if i % 5 else [727000, 740000, 728826, 729999, 729906][(i // 5) % 5]
        cols = gen_np.generate(seed * 1000 + i, 0, rows)
        comp = gen_np.compress(cols)
        if i % 7 == 3 and rows:
            # rows at the edges of the compressed domain: the shared tables' exact slow path
            r2 = np.random.default_rng(i)
            idx = r2.choice(rows, max(1, rows // 20), replace=False)
            comp["discount"][idx] = r2.integers(0, 101, len(idx))
            comp["tax"][idx] = r2.integers(0, 256, len(idx))
            comp["extendedprice"][idx] = r2.integers(0, 2**32, len(idx), dtype=np.uint64).astype(np.uint32)
            comp["quantity"][idx] = r2.integers(0, 256, len(idx))
        keys = gen_np.group_keys_uniform(seed * 1000 + i, 0, rows, g)
        out.append((comp, keys, g, cutoff))
    return out


def to_device(instances):
    keep, descs, outs = [], [], []
    for comp, keys, g, cutoff in instances:
        rows = len(keys)
        d = {k: torch.from_numpy(np.ascontiguousarray(comp[k]).view(np.uint8).copy()).cuda()
             for k in ["shipdate", "discount", "extendedprice", "tax", "quantity"]}
        d["keys"] = torch.from_numpy(np.ascontiguousarray(keys).view(np.uint8).copy()).cuda()
        out = torch.zeros(g * 12 + 2, dtype=torch.int64, device="cuda")
        bi = _lib.BatchInstance()
        for k in ["shipdate", "discount", "extendedprice", "tax", "quantity"]:
            setattr(bi.cols, k, d[k].data_ptr())
        bi.keys = d["keys"].data_ptr()
        bi.rows = rows
        bi.cutoff_day = cutoff
        bi.num_groups = g
        bi.aggregates = out.data_ptr()
        keep.append(d)
        descs.append(bi)
        outs.append(out)
    arr = (_lib.BatchInstance * len(descs))(*descs)
    return arr, outs, keep


def oracle_tables(instances):
    res = []
    for comp, keys, g, cutoff in instances:
        buf, flag = O.q1_groupkey(comp, keys, g, cutoff)
        assert flag == 0
        res.append(buf)
    return res


def read(out, g):
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint64)[: g * 12]


def run_batch(arr, n, opts, stream, runs=2):
    b = ctypes.c_void_p()
    _lib.check(q.lib().q1_batch_create(arr, n, ctypes.byref(opts), ctypes.c_void_p(stream), ctypes.byref(b)))
    try:
        for _ in range(runs):
            _lib.check(q.lib().q1_batch_run(b, ctypes.c_void_p(stream)))
        _lib.check(q.lib().q1_sync_check(ctypes.c_void_p(stream)))
        desc = _lib.BatchDesc()
        _lib.check(q.lib().q1_batch_describe(b, ctypes.byref(desc)))
        modes = []
        for i in range(n):
            m = ctypes.c_int32(-1)
            _lib.check(q.lib().q1_batch_instance_mode(b, i, ctypes.byref(m)))
            modes.append(m.value)
        return desc, modes
    finally:
        q.lib().q1_batch_destroy(b)


@pytest.fixture(scope="module")
def data(cuda):
    inst = make_instances()
    return inst, oracle_tables(inst)


@pytest.mark.parametrize("use_graph", [1, 0])
@pytest.mark.parametrize("chunk", [0, 1, 7])
def test_batch_equals_oracle(data, use_graph, chunk):
    inst, want = data
    arr, outs, keep = to_device(inst)
    opts = _lib.BatchOpts(use_graph, 0, chunk, 0, None)
    stream = torch.cuda.current_stream().cuda_stream
    desc, modes = run_batch(arr, len(inst), opts, stream)   # two runs: outputs are overwritten, not doubled
    assert desc.instances == len(inst) and desc.uses_graph == use_graph
    for i, (comp, keys, g, cutoff) in enumerate(inst):
        assert np.array_equal(read(outs[i], g), want[i]), f"instance {i} (rows={len(keys)}, groups={g})"


def test_batch_accumulate_mode(data):
    inst, want = data
    arr, outs, keep = to_device(inst)
    opts = _lib.BatchOpts(1, 1, 0, 0, None)
    stream = torch.cuda.current_stream().cuda_stream
    run_batch(arr, len(inst), opts, stream, runs=2)
    for i, (comp, keys, g, cutoff) in enumerate(inst):
        got = q.decode_aggregates(read(outs[i], g), g)
        assert np.array_equal(got, 2 * q.decode_aggregates(want[i], g))


def test_autotuner_modes_cache_and_parity(data, tmp_path):
    inst, want = data
    arr, outs, keep = to_device(inst)
    cache = str(tmp_path / "tune.txt")
    stream = torch.cuda.current_stream().cuda_stream
    desc, modes = run_batch(arr, len(inst), _lib.BatchOpts(1, 0, 0, 2, cache.encode()), stream)
    assert os.path.exists(cache) and desc.tuned_classes > 0
    text = open(cache).read()
    assert "mode " in text and "chunk " in text
    for i, (comp, keys, g, cutoff) in enumerate(inst):
        assert modes[i] in (0, 1, 2)
        if g > 4:
            assert modes[i] != 0
        assert np.array_equal(read(outs[i], g), want[i])
    # second batch reuses the cache: no class is measured again
    arr2, outs2, keep2 = to_device(inst)
    desc2, modes2 = run_batch(arr2, len(inst), _lib.BatchOpts(1, 0, 0, 1, cache.encode()), stream)
    assert desc2.tuned_classes == 0 and modes2 == modes
    for i, (comp, keys, g, cutoff) in enumerate(inst):
        assert np.array_equal(read(outs2[i], g), want[i])


def test_batch_equals_plain_launches(data):
    """One launch per instance (q1_launch_groupkey) gives the same tables as the batch."""
    inst, want = data
    arr, outs, keep = to_device(inst)
    stream = torch.cuda.current_stream().cuda_stream
    for i, (comp, keys, g, cutoff) in enumerate(inst):
        rows = len(keys)
        out = torch.zeros(g * 12 + 2, dtype=torch.int64, device="cuda")
        scratch = torch.zeros(int(q.lib().q1_groupkey_scratch_bytes(g)) // 8 + 2, dtype=torch.int64, device="cuda")
        placement = 1 if g <= 8 else 3
        _lib.check(q.lib().q1_launch_groupkey(placement, ctypes.byref(arr[i].cols), ctypes.c_void_p(arr[i].keys), g,
                                              rows, cutoff, None, ctypes.c_void_p(scratch.data_ptr()),
                                              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream)))
        _lib.check(q.lib().q1_sync_check(ctypes.c_void_p(stream)))
        assert np.array_equal(read(out, g), want[i])
