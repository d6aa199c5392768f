"""World-size-2 gloo run of the sharded path on CPU: the shards cover every root
once and the summed per-rank counts equal the single-process count."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime

    import torch.distributed as dist

    import oracle
    import vsgm_b200 as vs
    from vsgm_b200.shard import allreduce_counts, roots_of_rank

    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}",
                            timeout=datetime.timedelta(seconds=60))
    g = vs.gen_rmat(8, 8, seed=7)
    plans = [vs.plan_clique(3), vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(2)]
    roots = roots_of_rank(g.V, rank, world)
    mine = [oracle.count(p, g, roots, threads=1) for p in plans]
    total = allreduce_counts(mine)
    out[rank] = (roots.tolist(), total)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_and_count_sum():
    import oracle
    import vsgm_b200 as vs

    world, port = 2, _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    g = vs.gen_rmat(8, 8, seed=7)
    plans = [vs.plan_clique(3), vs.plan_clique(4), vs.plan_pattern(1), vs.plan_pattern(2)]
    want = [oracle.count(p, g) for p in plans]
    r0, t0 = out[0]
    r1, t1 = out[1]
    assert sorted(r0 + r1) == list(range(g.V)) and not set(r0) & set(r1)
    assert t0 == t1 == want
