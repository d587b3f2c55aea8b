"""Row-range sharding across ranks (one process per GPU) and the exact merge of their partials.

Rows are independent and every aggregate is a sum, so the table shards by row range with no
exchange on the data path; the only collective is one all-gather of each rank's per-group
int128 partials (groups x 6 x (lo, hi) uint64 words), summed exactly as Python integers. The
reference runs on one GPU and merges its CPU share the same way (src/main.cu:720-736).
"""
import numpy as np

from .api import decode_aggregates


def shard_rows(rows_per_rank, rank):
    """(first_row, rows) of `rank`'s shard of the generator's row space (weak scaling)."""
    return rank * rows_per_rank, rows_per_rank


def encode_aggregates(table):
    """[groups][6] Python ints -> uint64 words [groups*6*2] (two's-complement int128, lo then hi)."""
    groups = len(table)
    out = np.zeros(groups * 12, dtype=np.uint64)
    for g in range(groups):
        for a in range(6):
            v = int(table[g][a]) & ((1 << 128) - 1)
            out[12 * g + 2 * a] = v & 0xFFFFFFFFFFFFFFFF
            out[12 * g + 2 * a + 1] = v >> 64
    return out


def merge_partials(parts, groups=6):
    """Exact sum of the ranks' int128 tables -> [groups][6] ints. Each part is groups*6*2 words
    (lo, hi): a uint64 numpy array or an int64 torch tensor (copied to the host here)."""
    total = np.zeros((groups, 6), dtype=object)
    total[:, :] = 0
    for p in parts:
        if hasattr(p, "cpu"):
            p = p.cpu().numpy()
        total = total + decode_aggregates(np.asarray(p).view(np.uint64), groups)
    return total


def gather_partials(words, dist):
    """All-gathers this rank's int128 table (an int64 torch tensor of groups*12 words, on the
    device for NCCL) into one tensor per rank, rank order, without a host synchronisation. Every
    rank calls it once per step."""
    import torch
    parts = [torch.zeros_like(words) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, words)
    return parts
