"""GPU parity: every layout x placement x pushdown x residency x coprocessing combination of
q1_run, and the kernel-level launch ABI, against the oracle on the same seeded inputs.
Integer results must be bit-exact (tolerance 0)."""
import numpy as np
import pytest

import gen_np
import tpchq01_gpu_b200 as q
from oracle import py_oracle as O

pytestmark = pytest.mark.gpu

PLACEMENTS = ["in_registers", "in_registers_per_thread", "local_mem", "shared_mem_per_thread", "global"]
ROWS = 300_001          # several tiles plus a ragged tail
SEED = 4242


def oracle(cols, cutoff=729999):
    t, flag = O.q1_uncompressed(cols, cutoff)
    assert flag == 0
    return t


@pytest.fixture(scope="module")
def cols():
    return gen_np.generate(SEED, 0, ROWS)


@pytest.fixture(scope="module")
def contexts(cuda, cols):
    ctxs = {}
    for name, layout, packing in [("unc", "uncompressed", "pair"), ("pair", "compressed", "pair"),
                                  ("sep", "compressed", "separate")]:
        c = q.Q1Context(cpu_threads=3)
        c.load_columns(cols, layout, packing, "hbm")
        ctxs[name] = c
    yield ctxs
    for c in ctxs.values():
        c.close()


@pytest.mark.parametrize("placement", PLACEMENTS)
@pytest.mark.parametrize("kind", ["unc", "pair", "sep"])
def test_hbm_every_placement(contexts, cols, kind, placement):
    res = contexts[kind].run(hash_table_placement=placement, apply_compression=kind != "unc",
                             num_query_execution_runs=2)
    assert np.array_equal(res.table(), oracle(cols))


@pytest.mark.parametrize("placement", PLACEMENTS)
@pytest.mark.parametrize("kind", ["pair", "sep"])
def test_hbm_filter_pushdown(contexts, cols, kind, placement):
    res = contexts[kind].run(hash_table_placement=placement, apply_compression=True, use_filter_pushdown=True,
                             num_query_execution_runs=1)
    assert np.array_equal(res.table(), oracle(cols))


@pytest.mark.parametrize("cutoff", [727000, 727564, 728826, 729906, 730089, 740000])
@pytest.mark.parametrize("kind", ["unc", "pair"])
def test_cutoffs(contexts, cols, kind, cutoff):
    res = contexts[kind].run(apply_compression=kind != "unc", cutoff_day=cutoff, num_query_execution_runs=1)
    assert np.array_equal(res.table(), oracle(cols, cutoff))


@pytest.mark.parametrize("fraction", [0.0, 0.1, 0.5, 1.0])
@pytest.mark.parametrize("kind", ["unc", "pair", "sep"])
def test_hbm_coprocessing_merges_exactly(contexts, cols, kind, fraction):
    res = contexts[kind].run(apply_compression=kind != "unc", use_coprocessing=True,
                             cpu_processing_fraction=fraction, num_query_execution_runs=1)
    assert np.array_equal(res.table(), oracle(cols))
    assert res.rows_gpu + res.rows_cpu == ROWS
    if 0 < fraction < 1:
        assert res.rows_cpu > 0 and res.rows_gpu > 0


@pytest.mark.parametrize("layout,packing", [("compressed", "pair"), ("compressed", "separate"),
                                            ("uncompressed", "pair")])
@pytest.mark.parametrize("mode", [dict(), dict(use_coprocessing=True, cpu_processing_fraction=0.25),
                                  dict(num_gpu_streams=1), dict(num_gpu_streams=3)])
def test_pinned_host_streaming(cuda, cols, layout, packing, mode):
    with q.Q1Context(cpu_threads=2) as c:
        c.load_columns(cols, layout, packing, "pinned")
        res = c.run(apply_compression=layout == "compressed", num_tuples_per_kernel_launch=1 << 15,
                    num_query_execution_runs=2, **mode)
        assert np.array_equal(res.table(), oracle(cols))


@pytest.mark.parametrize("packing", ["pair", "separate"])
@pytest.mark.parametrize("coproc", [False, True])
def test_pinned_filter_pushdown_with_cpu_producers(cuda, cols, packing, coproc):
    """src/main.cu:541 + :575-580: CPU workers build the bitmap chunk by chunk and queue it."""
    with q.Q1Context(cpu_threads=3) as c:
        c.load_columns(cols, "compressed", packing, "pinned")
        res = c.run(apply_compression=True, use_filter_pushdown=True, use_coprocessing=coproc,
                    cpu_processing_fraction=0.3, num_tuples_per_kernel_launch=1 << 14, num_gpu_streams=4,
                    num_query_execution_runs=2)
        assert np.array_equal(res.table(), oracle(cols))


@pytest.mark.parametrize("rows", [0, 1, 31, 32, 33, 127, 128, 4095, 4096, 4097, 4607, 4608, 4609, 8197, 9217,
                                  1_000_003])
@pytest.mark.parametrize("kind", [("compressed", "pair", "in_registers_per_thread"),
                                  ("compressed", "pair", "shared_mem_per_thread"),
                                  ("uncompressed", "pair", "in_registers"),
                                  ("compressed", "separate", "global")])
def test_ragged_and_tiny_tables(cuda, rows, kind):
    layout, packing, placement = kind
    cols = gen_np.generate(77 + rows, 0, rows)
    with q.Q1Context() as c:
        c.load_columns(cols, layout, packing, "hbm")
        res = c.run(hash_table_placement=placement, apply_compression=layout == "compressed",
                    num_query_execution_runs=1)
        assert np.array_equal(res.table(), oracle(cols))


def test_averages_and_result_fields(contexts, cols):
    res = contexts["pair"].run(apply_compression=True, num_query_execution_runs=1)
    t = oracle(cols)
    for g, r in enumerate(res.groups):
        cnt = int(t[g, 0])
        assert r["count"] == cnt
        if cnt:
            assert r["avg_qty_e4"] == int(t[g, 1]) * 100 // cnt
            assert r["avg_price_e4"] == int(t[g, 2]) * 100 // cnt
            assert r["avg_disc_e4"] == int(t[g, 3]) * 100 // cnt
    assert res.ms_last_run > 0 and res.ms_gpu_last_run > 0
    wall, gpu = contexts["pair"].run_times()
    assert len(wall) == 1 and len(gpu) == 1


def test_runs_are_deterministic(contexts):
    a = contexts["sep"].run(apply_compression=True, num_query_execution_runs=3).table()
    b = contexts["sep"].run(apply_compression=True, hash_table_placement="global", num_query_execution_runs=3).table()
    assert np.array_equal(a, b)


def test_layout_mismatch_is_rejected(contexts):
    with pytest.raises(q.Q1Error):
        contexts["unc"].run(apply_compression=True)
    with pytest.raises(q.Q1Error):
        contexts["pair"].run(apply_compression=False)
