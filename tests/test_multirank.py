"""N>1 path on CPU: two gloo ranks each aggregate their row-range shard of the generator (the
oracle stands in for the GPU scan here) and exchange partials through the product's
gather/merge; the merged table must equal the oracle over the whole row range, and every rank
must see the same result."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import gen_np
from oracle import py_oracle as O

ROWS_PER_RANK = 50_017
SEED = 99
CUTOFF = 729999


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    from tpchq01_gpu_b200 import shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        first, rows = shard.shard_rows(ROWS_PER_RANK, rank)
        cols = gen_np.generate(SEED, first, rows)
        table, flag = O.q1_uncompressed(cols, CUTOFF)
        assert flag == 0
        words = torch.from_numpy(shard.encode_aggregates(table).view(np.int64).copy())
        parts = shard.gather_partials(words, dist)
        merged = shard.merge_partials(parts)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array(merged.tolist(), dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_exchange_equals_whole_table(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    whole = gen_np.generate(SEED, 0, world * ROWS_PER_RANK)
    want, flag = O.q1_uncompressed(whole, CUTOFF)
    assert flag == 0
    got = [np.load(tmp_path / f"rank{r}.npy", allow_pickle=True) for r in range(world)]
    for g in got:
        assert g.tolist() == want.tolist()


def test_encode_merge_roundtrip_negative_and_wide():
    from tpchq01_gpu_b200 import shard
    a = [[(1 << 100) + 5, -3, 0, 7, -(1 << 90), 1] for _ in range(6)]
    b = [[(1 << 100), 3, 1, -7, (1 << 90), (1 << 127) - 2] for _ in range(6)]
    m = shard.merge_partials([shard.encode_aggregates(a), shard.encode_aggregates(b)])
    for g in range(6):
        assert list(m[g]) == [x + y for x, y in zip(a[g], b[g])]
