"""The replica plumbing of bench.py (cpu-vh_b200/replicas.py) as two gloo
ranks on CPU: disjoint and complete event shards, max/sum over ranks, and a
throughput taken over the slowest rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n_events, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import replicas
    R = replicas.Replicas(backend="gloo", timeout_s=60)
    mine = list(R.shard(n_events))
    R.barrier()
    # a fake timed region: rank r "takes" 1 + r seconds for its events
    t_max = R.max(1.0 + rank)
    units = R.sum(len(mine))
    q.put((rank, mine, t_max, units))
    R.close()


@pytest.mark.parametrize("n_events", [256, 7, 1])
def test_two_gloo_ranks(n_events):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n_events, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    shards = [r[1] for r in res]
    assert sorted(sum(shards, [])) == list(range(n_events))          # complete
    assert not set(shards[0]) & set(shards[1])                        # disjoint
    assert abs(len(shards[0]) - len(shards[1])) <= 1
    for _, _, t_max, units in res:
        assert t_max == 2.0 and units == n_events
