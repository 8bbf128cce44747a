"""bench.py's multi-GPU launcher on the CPU: `--gpus N` starts N ranks under
torch.distributed.run (or checks the world it runs in), every rank answers
rank 0's queries, and the counts summed over the ranks' row shards equal
the single-rank count."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

import bench
from rtscan_b200 import datagen as D
from rtscan_b200 import shard as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(args, env=None):
    e = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        e.pop(k, None)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                          timeout=300, env=e)


def test_gpus_n_starts_n_ranks():
    r = run_bench(["--gpus", "2", "--dry-run"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert sorted(d["rank"] for d in lines) == [0, 1]
    assert all(d["world"] == 2 and d["gpus"] == 2 for d in lines)


def test_world_size_must_match_gpus():
    r = run_bench(["--gpus", "1", "--dry-run"], env={"WORLD_SIZE": "2", "RANK": "0", "LOCAL_RANK": "0"})
    assert r.returncode != 0 and "WORLD_SIZE=2" in r.stderr
    r = run_bench(["--gpus", "1", "--dry-run"])
    assert r.returncode == 0 and json.loads(r.stdout.strip())["world"] == 1


def test_launch_command_is_one_node_torchrun():
    cmd = bench.launch_command(4, ["--steps", "2"])
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "--nnodes=1" in cmd
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-3:] == [os.path.join(ROOT, "bench.py"), "--steps", "2"]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, n, q):
    import torch.distributed as dist

    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cols = [D.uniform(n, 1), D.zipf(n, 2, 1.3)]
        local = S.shard_columns(cols, world, rank)
        # each rank draws queries from its own rows; the bench keeps rank 0's
        mine = D.batch_queries(local, 5, seed=100 + rank)
        queries = bench.agree_queries(mine, world)
        counts = [O.range_scan([local[c] for c, _, _ in t], [x[1] for x in t], [x[2] for x in t])[1]
                  for t in queries]
        total = S.all_reduce_counts(counts)
        box = [queries]
        dist.broadcast_object_list(box, src=1)  # rank 1's view of the agreed queries
        if rank == 0:
            assert queries == mine and box[0] == queries
            for i, t in enumerate(queries):
                want = O.range_scan([cols[c] for c, _, _ in t], [x[1] for x in t], [x[2] for x in t])[1]
                assert int(total[i]) == want
            q.put("ok")
    except Exception as e:  # report to the parent instead of hanging it
        q.put(repr(e))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [100_003])
def test_ranks_answer_rank0_queries_and_counts_sum(n):
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
