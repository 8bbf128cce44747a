"""Row sharding across ranks (one process per GPU).

The scan shards by rows with no exchange on the data path: rank r owns rows
[begin_r, end_r) of every column (boundaries on multiples of 32 rows, so a
bitmap word never straddles two ranks), answers every query on them, and
its bitmap words are words [begin_r/32, ...) of the global bitmap.  Counts
combine with one sum all-reduce of Q uint64; a caller that wants a whole
bitmap on one rank gathers the rank slices (concatenation, no merging).
The reference has no multi-GPU path (every entry point pins device 0,
cuda_and.cu:265).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np


def shard_bounds(nrows: int, world: int, rank: int, align: int = 32) -> Tuple[int, int]:
    """[begin, end) rows of `rank`: contiguous, in `align`-row units, sizes
    differing by at most one unit, the last rank taking the tail."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    units = (nrows + align - 1) // align
    base, extra = divmod(units, world)
    u0 = rank * base + min(rank, extra)
    u1 = u0 + base + (1 if rank < extra else 0)
    return min(nrows, u0 * align), min(nrows, u1 * align)


def shard_columns(cols: Sequence[np.ndarray], world: int, rank: int) -> List[np.ndarray]:
    n = len(cols[0])
    b, e = shard_bounds(n, world, rank)
    return [c[b:e] for c in cols]


def word_offset(nrows: int, world: int, rank: int) -> int:
    return shard_bounds(nrows, world, rank)[0] // 32


def all_reduce_counts(counts, group=None):
    """Sum per-query counts over ranks (torch.distributed, any backend);
    returns the global counts as a numpy uint64 array."""
    import torch
    import torch.distributed as dist
    t = torch.as_tensor(np.asarray(counts, dtype=np.int64))
    if t.device.type == "cpu" and dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy().astype(np.uint64)


def gather_bitmap(local_words: np.ndarray, nrows: int, dst: int = 0, group=None):
    """Concatenate the ranks' bitmap slices on rank `dst` (None elsewhere)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    sizes = [(shard_bounds(nrows, world, r)[1] - shard_bounds(nrows, world, r)[0] + 31) // 32 for r in range(world)]
    mx = max(sizes)
    buf = np.zeros(mx, dtype=np.uint32)
    buf[:len(local_words)] = local_words
    t = torch.from_numpy(buf.view(np.int32))
    parts = [torch.empty_like(t) for _ in range(world)] if rank == dst else None
    dist.gather(t, parts, dst=dst, group=group)
    if rank != dst:
        return None
    return np.concatenate([p.numpy().view(np.uint32)[:sizes[r]] for r, p in enumerate(parts)])
