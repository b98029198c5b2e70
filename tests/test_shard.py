"""Ligand sharding for N > 1 GPUs, checked with world_size-2 gloo ranks on CPU:
the ranks' shares are disjoint, cover every ligand, are balanced by cost, and
the bench's timing reduction (max over ranks) sees the slowest rank."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from unidock_tools.shard import shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, costs, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    mine = shard(len(costs), rank, world, costs)
    parts = [None] * world
    dist.all_gather_object(parts, mine)
    t = torch.tensor([0.5 + rank])            # per-rank elapsed time
    dist.all_reduce(t, op=dist.ReduceOp.MAX)  # as bench.py times a step
    if rank == 0:
        q.put((parts, float(t.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_shards_cover_all_ligands_once_and_balance():
    costs = [float((7 * i) % 23 + 1) for i in range(103)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    parts, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b = set(parts[0]), set(parts[1])
    assert not (a & b) and (a | b) == set(range(len(costs)))
    la, lb = sum(costs[i] for i in a), sum(costs[i] for i in b)
    assert max(la, lb) / min(la, lb) < 1.05
    assert tmax == 1.5


def test_round_robin_and_argument_checks():
    assert shard(7, 1, 3) == [1, 4]
    assert shard(0, 0, 1) == []
    with pytest.raises(ValueError):
        shard(4, 2, 2)
    with pytest.raises(ValueError):
        shard(3, 0, 2, cost=[1.0])


def test_bench_launches_one_rank_per_gpu():
    """`bench.py --gpus 2` run directly starts two ranks itself (under
    torch.distributed.run) and reports n_gpus 2; the dry run does no GPU work:
    each rank shards the first step's ligands and meets the other at the
    timing barrier and max-reduction over gloo."""
    import json
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--gpus", "2", "--dry-run", "--batch", "64"],
                       capture_output=True, text=True, timeout=600, cwd=str(root))
    assert r.returncode == 0, r.stderr[-2000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
    res = json.loads(line)
    assert res["n_gpus"] == 2
    assert res["ligands_per_step"] == 128 and res["ligands_sharded"] == 128
    assert res["max_rank_ligands"] == 64


def test_bench_refuses_rank_count_mismatch():
    """A rank whose WORLD_SIZE differs from --gpus stops before any timing."""
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--gpus", "2", "--dry-run"], capture_output=True,
                       text=True, timeout=300, env=env, cwd=str(root))
    assert r.returncode != 0
    assert "one rank per GPU" in (r.stdout + r.stderr)
