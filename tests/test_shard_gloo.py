"""Multi-rank placement of the batched form, run as two gloo ranks on CPU.

Every rank computes the longest-first assignment independently; the test
gathers the shares and checks that all ranks agree, that each index is built
by exactly one rank, that the loads are balanced within one item's cost, and
that the reporting collective sums the ranks' counts.
"""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, costs, q):
    import torch.distributed as dist

    from rinnd_b200 import shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard.my_share(costs, rank, world)
        shares = [None] * world
        dist.all_gather_object(shares, (rank, mine))
        items, points = shard.gather_counts(len(mine), int(sum(costs[i] for i in mine)))
        q.put((rank, shares, items, points))
    finally:
        dist.destroy_process_group()


def test_longest_first_is_a_partition():
    from rinnd_b200 import shard

    rng = np.random.default_rng(0)
    costs = [shard.build_cost(int(n), int(d), 15) for n, d in zip(rng.integers(2000, 200000, 97),
                                                                  rng.choice([32, 64, 128, 256], 97))]
    for world in (1, 2, 3, 8):
        parts = shard.assign_longest_first(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs) + 1e-6
    with pytest.raises(ValueError):
        shard.assign_longest_first(costs, 0)


def test_two_gloo_ranks_agree_on_the_shares():
    import torch.multiprocessing as mp

    costs = [float(c) for c in np.random.default_rng(1).integers(1, 1000, 41)]
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get() for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shares = {r: dict(s) for r, s, _, _ in results}
    assert shares[0] == shares[1]  # both ranks saw the same assignment
    got = sorted(shares[0][0] + shares[0][1])
    assert got == list(range(len(costs)))
    for _, _, items, points in results:
        assert items == len(costs)
        assert points == int(sum(int(c) for c in costs))
