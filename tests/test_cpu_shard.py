"""Sharding of batched sets over ranks (host logic, CPU): two gloo ranks each take their
shard of the 256-set batch workload; together the shards cover every set exactly once and
the largest modelled load is within the greedy bound of the average."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bbfmm_b200 import batch_depth, set_cost, shard_sets
    rng = np.random.default_rng(5)
    Ns = [int(round(np.exp(rng.uniform(np.log(4096), np.log(262144))))) for _ in range(256)]
    ns = [int(rng.choice([4, 8])) for _ in range(256)]
    costs = [set_cost(N, n, batch_depth(N)) for N, n in zip(Ns, ns)]
    mine = shard_sets(costs, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, (mine, sum(costs[i] for i in mine)))
    if rank == 0:
        q.put((got, sum(costs), max(costs)))
    dist.destroy_process_group()


def test_two_ranks_cover_every_set_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got, total, biggest = q.get(timeout=120)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    sets = sorted(i for shard, _ in got for i in shard)
    assert sets == list(range(256))
    loads = [l for _, l in got]
    assert max(loads) <= total / 2 + biggest  # greedy list-scheduling bound


def test_shard_sets_single_rank_and_empty():
    from bbfmm_b200 import shard_sets
    assert shard_sets([3.0, 1.0, 2.0], 1) == [[0, 1, 2]]
    assert shard_sets([], 3) == [[], [], []]
    assert shard_sets([5.0, 4.0, 3.0, 3.0], 2) == [[0, 3], [1, 2]]
