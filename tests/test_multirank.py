"""The N>1 path on CPU: two gloo ranks shard the rows, answer the same
queries on their slices (the oracle stands in for each rank's GPU), combine
counts with one all-reduce and gather the bitmap slices; the result must
equal the single-rank answer bit for bit.  Also checks the shard bounds."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from rtscan_b200 import datagen as D
from rtscan_b200 import shard as S


def test_shard_bounds_cover_rows_in_word_units():
    for n in (1, 31, 32, 33, 1000, 100_000_007, 1 << 28):
        for world in (1, 2, 3, 8):
            prev = 0
            for r in range(world):
                b, e = S.shard_bounds(n, world, r)
                assert b == prev and b <= e <= n
                assert b % 32 == 0 or b == e == n  # empty trailing shards sit at n
                prev = e
            assert prev == n


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, n, q):
    import torch.distributed as dist

    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cols = [D.uniform(n, 1), D.uniform(n, 2, 256), D.zipf(n, 3, 1.3)]
        local = S.shard_columns(cols, world, rank)
        queries = D.batch_queries(cols, 6, seed=5)
        counts, bitmaps = [], []
        for terms in queries:
            bm, c = O.range_scan([local[c] for c, _, _ in terms], [t[1] for t in terms], [t[2] for t in terms])
            counts.append(c)
            bitmaps.append(bm)
        total = S.all_reduce_counts(counts)
        full = [S.gather_bitmap(bm, n) for bm in bitmaps]
        if rank == 0:
            for i, terms in enumerate(queries):
                ref, rc = O.range_scan([cols[c] for c, _, _ in terms], [t[1] for t in terms], [t[2] for t in terms])
                assert int(total[i]) == rc
                assert np.array_equal(full[i], ref)
            q.put("ok")
    except Exception as e:  # report to the parent instead of hanging it
        q.put(repr(e))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [100_003, 65_536])
def test_two_rank_shard_allreduce_gather(n):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) == "ok"
