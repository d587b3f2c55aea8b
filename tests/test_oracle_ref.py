"""The oracle against the reference's own CPU kernels run live (oracle/_ref/libq1ref.so) on
fresh seeded inputs: KernelHyPer<true>, KernelX100 single-threaded and on a thread pool."""
import numpy as np
import pytest

import gen_np
from oracle import py_oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("seed,rows,cutoff", [(101, 200_000, 729999), (102, 77_777, 729906),
                                              (103, 50_000, 730089), (104, 65_536, 728500)])
def test_restatement_equals_reference_kernels(seed, rows, cutoff):
    cols = gen_np.generate(seed, 0, rows)
    mine, f1 = O.q1_uncompressed(cols, cutoff)
    t = O.RefTable(cols, cutoff)
    hyper, f2 = t.hyper()
    x100, rc = t.x100()
    par, rc2 = t.x100_parallel(3, morsel=4096)
    t.close()
    assert f1 == 0 and f2 == 0 and rc == 0 and rc2 == 0
    assert np.array_equal(mine, hyper)
    assert np.array_equal(mine, x100)
    assert np.array_equal(mine, par)


def test_x100_partial_ranges_add_up():
    cols = gen_np.generate(105, 0, 30_000)
    t = O.RefTable(cols)
    a, _ = t.x100(0, 10_000)
    b, _ = t.x100(10_000, 20_000)
    whole, _ = t.x100()
    t.close()
    assert np.array_equal(a + b, whole)


@pytest.mark.parametrize("seed,rows,cutoff", [(106, 120_000, 729999), (107, 33_333, 729906), (108, 50_000, 727600)])
def test_hyper_compact_equals_restatement(seed, rows, cutoff):
    """The reference's KernelHyPerCompact (compact int8/int16/int32 columns) gives the same tables,
    with the ship-date shift its int16 cutoff needs under the GPU build."""
    cols = gen_np.generate(seed, 0, rows)
    mine, _ = O.q1_uncompressed(cols, cutoff)
    t = O.RefTable(cols, cutoff - O.HYPER_COMPACT_SHIFT)
    compact, flag = t.hyper_compact()
    t.close()
    assert flag == 0
    assert np.array_equal(mine, compact)


@pytest.mark.parametrize("seed,first,rows", [(201, 0, 100_001), (202, 12_345_678, 7)])
def test_bridge_generator_equals_pushed_columns(seed, first, rows):
    """q1ref_table_generate (the oracle's own generator, pushed by the bridge) builds the same
    lineitem as pushing the numpy restatement's columns."""
    a = O.RefTable.generated(seed, first, rows)
    b = O.RefTable(gen_np.generate(seed, first, rows))
    ha, fa = a.hyper()
    hb, fb = b.hyper()
    a.close()
    b.close()
    assert fa == 0 and fb == 0
    assert np.array_equal(ha, hb)


@pytest.mark.parametrize("rows,chunk,threads,cutoff", [(1_000_001, 250_000, 3, 729999),
                                                       (777_777, 1 << 20, 2, 729906),
                                                       (300_000, 100_000, 4, 728000)])
def test_chunked_x100_equals_whole_table(rows, chunk, threads, cutoff):
    """KernelX100 over chunks of compact copies (a ragged last chunk included) gives the table of
    one lineitem holding every row, run after run."""
    seed, first = 301, 5
    whole = O.RefTable(gen_np.generate(seed, first, rows), cutoff)
    want, rc = whole.x100_parallel(2, morsel=8192)
    whole.close()
    assert rc == 0
    assert np.array_equal(want, O.q1_uncompressed(gen_np.generate(seed, first, rows), cutoff)[0])
    ch = O.RefChunks(seed, first, rows, chunk_rows=chunk, cutoff_day=cutoff, threads=threads)
    try:
        assert ch.chunks() == (rows + chunk - 1) // chunk and ch.threads() == threads
        for _ in range(2):
            got, rc = ch.run(morsel=4096)
            assert rc == 0
            assert np.array_equal(got, want)
    finally:
        ch.close()
