"""Group-key aggregation (uint32 key, up to 65,536 groups) against the oracle: every placement,
group counts 4 / 64 / 1024 / 65536, uniform and Zipf(1.1) keys, cutoffs from ~1% to 100% passing.
Integer results, tolerance 0."""
import ctypes

import numpy as np
import pytest
import torch

import gen_np
import tpchq01_gpu_b200 as q
from oracle import py_oracle as O
from tpchq01_gpu_b200 import _lib

pytestmark = pytest.mark.gpu

ROWS = 400_037
SEED = 555


def zipf_cdf(g, s=1.1):
    cdf = np.zeros(g, dtype=np.uint32)
    _lib.check(q.lib().q1_zipf_cdf(g, s, cdf.ctypes.data_as(ctypes.c_void_p)))
    return cdf


@pytest.fixture(scope="module")
def table(cuda):
    cols = gen_np.generate(SEED, 0, ROWS)
    comp = gen_np.compress(cols)
    dev = {k: torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).copy()).cuda()
           for k, v in comp.items() if isinstance(v, np.ndarray) and k != "pair_group"}
    c = _lib.CompressedColumns()
    for k in ["shipdate", "discount", "extendedprice", "tax", "quantity"]:
        setattr(c, k, dev[k].data_ptr())
    return comp, c, dev


def keys_for(num_groups, dist):
    if dist == "uniform":
        return gen_np.group_keys_uniform(SEED, 0, ROWS, num_groups), None
    cdf = zipf_cdf(num_groups)
    return gen_np.group_keys_cdf(SEED, 0, ROWS, cdf), cdf


def widen(comp, seed, frac=0.05):
    """Copy of compressed columns with a fraction of rows moved to the edges of the compressed
    domain (discount 11..100, tax 9..255, price >= 2^24, quantity 51..255): the shared tables'
    slow path."""
    out = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in comp.items()}
    n = len(out["shipdate"])
    rng = np.random.default_rng(seed)
    idx = rng.choice(n, max(1, int(frac * n)), replace=False)
    out["discount"][idx] = rng.integers(0, 101, len(idx))
    out["tax"][idx] = rng.integers(0, 256, len(idx))
    out["extendedprice"][idx] = rng.integers(0, 2**32, len(idx), dtype=np.uint64).astype(np.uint32)
    out["quantity"][idx] = rng.integers(0, 256, len(idx))
    return out


def device_cols(comp):
    dev = {k: torch.from_numpy(np.ascontiguousarray(comp[k]).view(np.uint8).copy()).cuda()
           for k in ["shipdate", "discount", "extendedprice", "tax", "quantity"]}
    c = _lib.CompressedColumns()
    for k, t in dev.items():
        setattr(c, k, t.data_ptr())
    return c, dev


def run_gpu(c, keys, num_groups, placement, cutoff, blocks=0):
    rows = len(keys)
    dkeys = torch.from_numpy(keys.view(np.int32).copy()).cuda()
    scratch = torch.zeros(int(q.lib().q1_groupkey_scratch_bytes(num_groups)) // 8 + 2, dtype=torch.int64, device="cuda")
    out = torch.zeros(num_groups * 12, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    cfg = _lib.LaunchConfig(0, 0, blocks)
    _lib.check(q.lib().q1_launch_groupkey(q.placement_id(placement), ctypes.byref(c), ctypes.c_void_p(dkeys.data_ptr()),
                                          num_groups, rows, cutoff, ctypes.byref(cfg),
                                          ctypes.c_void_p(scratch.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                          ctypes.c_void_p(stream)))
    _lib.check(q.lib().q1_sync_check(ctypes.c_void_p(stream)))
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint64)


def check(comp, keys, num_groups, cutoff, got):
    want, flag = O.q1_groupkey(comp, keys, num_groups, cutoff)
    assert flag == 0
    assert np.array_equal(got, want), "group-key aggregates differ from the oracle"


# cutoffs: 1995-01-01-ish (~43%), 1998-09-02 (~98%), everything, ~1%
CUTOFFS = [727600, 728660, 729999, 730089]


@pytest.mark.parametrize("num_groups", [4, 64, 65, 1024, 65536])
@pytest.mark.parametrize("dist", ["uniform", "zipf"])
@pytest.mark.parametrize("placement", ["shared_mem_per_thread", "global"])
def test_groupkey_placements(table, num_groups, dist, placement):
    comp, c, _ = table
    keys, _ = keys_for(num_groups, dist)
    for cutoff in [729999, 727600]:
        check(comp, keys, num_groups, cutoff, run_gpu(c, keys, num_groups, placement, cutoff))


@pytest.mark.parametrize("num_groups", [1, 3, 4, 5, 8])
@pytest.mark.parametrize("cutoff", CUTOFFS)
def test_groupkey_registers(table, num_groups, cutoff):
    comp, c, _ = table
    keys, _ = keys_for(num_groups, "uniform")
    check(comp, keys, num_groups, cutoff, run_gpu(c, keys, num_groups, "in_registers_per_thread", cutoff))


@pytest.mark.parametrize("num_groups,placement", [
    (4, "in_registers_per_thread"), (7, "in_registers_per_thread"), (6, "shared_mem_per_thread"),
    (256, "shared_mem_per_thread"), (257, "shared_mem_per_thread"), (769, "shared_mem_per_thread"),
    (1024, "shared_mem_per_thread"), (1025, "shared_mem_per_thread"), (3000, "shared_mem_per_thread"),
    (64, "global")])
def test_domain_edges_take_exact_paths(table, num_groups, placement):
    """Rows with discount > 10, tax > 8, price >= 2^24 or quantity > 50 leave the shared tables'
    fast domain; the result must stay exact."""
    comp, _, _ = table
    wide = widen(comp, 7 + num_groups)
    c, keep = device_cols(wide)
    for dist in ["uniform", "zipf"]:
        keys, _ = keys_for(num_groups, dist)
        for cutoff in [729999, 730089]:
            check(wide, keys, num_groups, cutoff, run_gpu(c, keys, num_groups, placement, cutoff))


@pytest.mark.parametrize("rows,blocks", [(r, 1) for r in [1, 2047, 2048, 2049, 4097, 98_303, 98_304, 98_305,
                                                           101_377, 104_449]] +
                         [(r, 4) for r in [393_215, 393_216, 393_217]] + [(1_000_003, 0)])
@pytest.mark.parametrize("num_groups", [4, 8])
def test_registers_ragged_tiles(cuda, rows, blocks, num_groups):
    """Row counts around the register planes' tiles: four groups' planes take 12 consumer warps
    over 3072-row tiles on a table of at least 32 tiles per CTA (98,304 rows for one CTA, 393,216
    for four), 8 warps over 2048-row tiles below that; eight groups' planes always the latter."""
    part = gen_np.compress(gen_np.generate(SEED + 6, 0, rows))
    c, keep = device_cols(part)
    keys = gen_np.group_keys_uniform(SEED + 5, 0, rows, num_groups)
    check(part, keys, num_groups, 729999,
          run_gpu(c, keys, num_groups, "in_registers_per_thread", 729999, blocks=blocks))


@pytest.fixture(scope="module")
def long_table(cuda):
    rows = 13_000_011
    comp = widen(gen_np.compress(gen_np.generate(SEED + 1, 0, rows)), 99, frac=0.001)
    c, keep = device_cols(comp)
    return comp, c, keep, rows


@pytest.mark.parametrize("num_groups,placement", [
    (4, "in_registers_per_thread"), (8, "in_registers_per_thread"), (64, "shared_mem_per_thread"),
    (200, "shared_mem_per_thread"), (1024, "shared_mem_per_thread"), (5000, "shared_mem_per_thread")])
def test_one_cta_flushes_mid_launch(long_table, num_groups, placement):
    """One CTA over 13M rows: the per-thread planes (every 4032 tiles of 3072 or 2048 rows) and the
    shared tables (every 2^23 rows) are flushed inside the launch."""
    comp, c, _, rows = long_table
    keys = gen_np.group_keys_uniform(SEED + 2, 0, rows, num_groups)
    check(comp, keys, num_groups, 729999, run_gpu(c, keys, num_groups, placement, 729999, blocks=1))


@pytest.mark.parametrize("num_groups", [64, 1024])
def test_one_cta_zipf_keys_wrap_cells_often(long_table, num_groups):
    """One CTA over 13M rows of Zipf keys: the most frequent key's cells collect a fifth of the rows,
    so their 32-bit price and tax-price words wrap thousands of times between flushes; the wraps are
    counted in the group's shared words (1024 groups) or the cell's carry word (64 groups)."""
    comp, c, _, rows = long_table
    keys = gen_np.group_keys_cdf(SEED + 3, 0, rows, zipf_cdf(num_groups))
    check(comp, keys, num_groups, 740000, run_gpu(c, keys, num_groups, "shared_mem_per_thread", 740000, blocks=1))


def test_registers_refuse_many_groups(table):
    comp, c, _ = table
    keys, _ = keys_for(64, "uniform")
    with pytest.raises(q.Q1Error) as e:
        run_gpu(c, keys, 64, "in_registers_per_thread", 729999)
    assert e.value.status == 5


def test_key_out_of_range_is_reported(table):
    comp, c, _ = table
    keys, _ = keys_for(64, "uniform")
    keys = keys.copy()
    keys[100] = 64
    with pytest.raises(q.Q1Error) as e:
        run_gpu(c, keys, 64, "global", 730089)
    assert e.value.status == 6


@pytest.mark.parametrize("num_groups,dist", [(1024, "uniform"), (65536, "zipf")])
def test_device_key_generator(cuda, num_groups, dist):
    keys, cdf = keys_for(num_groups, dist)
    out = torch.zeros(ROWS, dtype=torch.int32, device="cuda")
    dcdf = None if cdf is None else torch.from_numpy(cdf.view(np.int32).copy()).cuda()
    _lib.check(q.lib().q1_generate_group_keys_device(SEED, 0, ROWS, num_groups,
                                                     None if dcdf is None else ctypes.c_void_p(dcdf.data_ptr()),
                                                     ctypes.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), keys)


def test_zipf_cdf_matches_restatement():
    cdf = zipf_cdf(65536)
    ref = gen_np.zipf_cdf(65536)
    assert cdf[-1] == 0xFFFFFFFF and np.all(np.diff(cdf.astype(np.int64)) >= 0)
    assert np.max(np.abs(cdf.astype(np.int64) - ref.astype(np.int64))) <= 1
