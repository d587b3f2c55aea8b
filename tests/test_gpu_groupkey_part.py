"""The high-cardinality paths of the group-key shared placement against the oracle. Above 256
groups the library chooses on the device, from a sample of the rows, among: one pass with a
shared slot per key < 4096 (3-stage ring above 2048 groups; larger keys into global
accumulators), every passing row straight into global accumulators (few passing rows over spread
keys), and, above 4096 groups, a two-pass radix partition (rows partitioned by key into 8-byte
records, then one shared-memory slot table per 4096-key partition). Q1_GROUPKEY_PATH forces each
path so that all are checked: group counts on both sides of the
partition width, uniform and Zipf keys, cutoffs from nothing to everything passing, ragged and
tiny row counts, few-CTA launches (partition changes and table flushes inside a CTA) and a
launch that crosses the 2^27-row segment boundary (against the global placement and the row
count). Tolerance 0."""
import ctypes

import numpy as np
import pytest
import torch

import gen_np
import tpchq01_gpu_b200 as q
from tpchq01_gpu_b200 import _lib
from test_gpu_groupkey import check, device_cols, keys_for, run_gpu, widen, zipf_cdf

pytestmark = pytest.mark.gpu

ROWS = 400_037
SEED = 555


PATHS = ["partitioned", "single", "global", "auto"]


@pytest.fixture(scope="module")
def table(cuda):
    comp = gen_np.compress(gen_np.generate(SEED, 0, ROWS))
    c, keep = device_cols(comp)
    return comp, c, keep


@pytest.fixture(params=PATHS)
def path(request, monkeypatch):
    if request.param == "auto":
        monkeypatch.delenv("Q1_GROUPKEY_PATH", raising=False)
    else:
        monkeypatch.setenv("Q1_GROUPKEY_PATH", request.param)
    return request.param


@pytest.mark.parametrize("num_groups", [257, 1024, 1025, 2049, 3000, 4096])
@pytest.mark.parametrize("dist", ["uniform", "zipf"])
@pytest.mark.parametrize("path", ["single", "global", "auto"], indirect=True)
def test_wide_tables_match_oracle(table, path, num_groups, dist):
    """257..4096 groups: the path is chosen on the device; the single pass keeps (group, discount)
    cells up to 1024 groups and one slot per group above."""
    comp, c, _ = table
    keys, _ = keys_for(num_groups, dist)
    for cutoff in [727000, 727600, 729999, 730089]:
        check(comp, keys, num_groups, cutoff, run_gpu(c, keys, num_groups, "shared_mem_per_thread", cutoff))


@pytest.mark.parametrize("num_groups", [4097, 8191, 12288, 65536])
@pytest.mark.parametrize("dist", ["uniform", "zipf"])
def test_two_paths_match_oracle(table, path, num_groups, dist):
    comp, c, _ = table
    keys, _ = keys_for(num_groups, dist)
    for cutoff in [727000, 727600, 729999, 730089]:
        check(comp, keys, num_groups, cutoff, run_gpu(c, keys, num_groups, "shared_mem_per_thread", cutoff))


@pytest.mark.parametrize("rows", [1, 31, 2047, 2048, 2049, 4097, 65_537])
def test_small_and_ragged(table, path, rows):
    comp, _, _ = table
    part = {k: (v[:rows].copy() if isinstance(v, np.ndarray) and len(v) == ROWS else v) for k, v in comp.items()}
    c, keep = device_cols(part)
    keys = gen_np.group_keys_uniform(SEED + rows, 0, rows, 65536)
    check(part, keys, 65536, 730089, run_gpu(c, keys, 65536, "shared_mem_per_thread", 730089))


@pytest.mark.parametrize("blocks", [1, 3])
@pytest.mark.parametrize("dist", ["uniform", "zipf"])
def test_few_ctas(table, path, blocks, dist):
    """Few CTAs: each walks many partitions in pass 2 (a table flush at every change) and stages
    every partition's records in pass 1."""
    comp, c, _ = table
    keys, _ = keys_for(65536, dist)
    check(comp, keys, 65536, 729999, run_gpu(c, keys, 65536, "shared_mem_per_thread", 729999, blocks=blocks))


def test_domain_edges(table, path):
    """Rows outside the slot tables' fast domain reduce straight into the accumulators."""
    comp, _, _ = table
    wide = widen(comp, 4242, frac=0.05)
    c, keep = device_cols(wide)
    for dist in ["uniform", "zipf"]:
        keys, _ = keys_for(40000, dist)
        for cutoff in [729999, 730089]:
            check(wide, keys, 40000, cutoff, run_gpu(c, keys, 40000, "shared_mem_per_thread", cutoff))


def test_key_out_of_range_is_reported(table, path):
    comp, c, _ = table
    keys, _ = keys_for(5000, "uniform")
    keys = keys.copy()
    keys[12345] = 5000
    with pytest.raises(q.Q1Error) as e:
        run_gpu(c, keys, 5000, "shared_mem_per_thread", 730089)
    assert e.value.status == 6


@pytest.mark.parametrize("path", ["partitioned", "auto"], indirect=True)
def test_crosses_segment_boundary(cuda, path):
    """2^27 + 4099 rows: two segments of the partitioned path. Same table as the global placement,
    and the counts add up to the rows that pass."""
    rows = (1 << 27) + 4099
    L = q.lib()
    stream = torch.cuda.current_stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    cols = {k: torch.empty(rows * w + 64, dtype=torch.uint8, device="cuda")
            for k, w in [("shipdate", 2), ("discount", 1), ("extendedprice", 4), ("tax", 1), ("quantity", 1)]}
    flags = torch.empty(4 * ((rows + 15) // 16) + 64, dtype=torch.uint8, device="cuda")
    out = _lib.CompressedHostOut()
    for k, t in cols.items():
        setattr(out, k, t.data_ptr())
    out.flags = flags.data_ptr()
    _lib.check(L.q1_generate_compressed_device(SEED + 9, 0, rows, 0, ctypes.byref(out), sh))
    c = _lib.CompressedColumns()
    for k, t in cols.items():
        setattr(c, k, t.data_ptr())
    G = 65536
    cdf = torch.from_numpy(zipf_cdf(G).view(np.int32).copy()).cuda()
    keys = torch.empty(rows + 16, dtype=torch.int32, device="cuda")
    scratch = torch.empty(int(L.q1_groupkey_scratch_bytes(G)) // 8 + 2, dtype=torch.int64, device="cuda")
    cutoff = 729999
    ship = cols["shipdate"][: 2 * rows].view(torch.int16).to(torch.int32)
    passing = int((ship <= cutoff - 727563).sum())
    del ship
    for cdf_arg in [None, cdf]:
        _lib.check(L.q1_generate_group_keys_device(SEED + 9, 0, rows, G,
                                                   None if cdf_arg is None else ctypes.c_void_p(cdf_arg.data_ptr()),
                                                   ctypes.c_void_p(keys.data_ptr()), sh))
        res = []
        for placement in ["shared_mem_per_thread", "global"]:
            o = torch.zeros(G * 12, dtype=torch.int64, device="cuda")
            _lib.check(L.q1_launch_groupkey(q.placement_id(placement), ctypes.byref(c), ctypes.c_void_p(keys.data_ptr()),
                                            G, rows, cutoff, None, ctypes.c_void_p(scratch.data_ptr()),
                                            ctypes.c_void_p(o.data_ptr()), sh))
            _lib.check(L.q1_sync_check(sh))
            res.append(o.cpu().numpy().view(np.uint64).reshape(G, 6, 2))
        assert np.array_equal(res[0], res[1])
        assert int(res[0][:, 0, 0].sum()) == passing and not res[0][:, 0, 1].any()
