"""Multi-GPU replicas, host side, on CPU: two gloo ranks partition a request stream into
disjoint, complete, cost-balanced shares and reduce timing scalars (max over ranks, sum of
solves) as bench.py does under torchrun."""

import os
import socket

import numpy as np

from materialite_b200.replicas import partition, request_cost


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank)})
    from materialite_b200 import replicas
    from materialite_b200.serving import request_stream
    w, r, local = replicas.init(backend="gloo", timeout_s=60)
    assert (w, r) == (world, rank)
    reqs = request_stream(16, 10.0, seed=1000)
    mine = replicas.partition(reqs, w, r)
    replicas.barrier(w)
    t_max = replicas.max_over_ranks(1.0 + rank, w, local)
    total = replicas.sum_over_ranks(len(mine), w, local)
    np.save(os.path.join(out_dir, f"rank{rank}.npy"),
            np.array([t_max, total] + [q.tag for q in mine], dtype=np.float64))
    replicas.destroy(w)


def test_two_gloo_ranks_partition_and_reduce(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    res = [np.load(tmp_path / f"rank{k}.npy") for k in range(world)]
    for r in res:
        assert r[0] == 2.0            # max over ranks of (1 + rank)
        assert r[1] == 16.0           # every request solved once in total
    tags = [set(r[2:].astype(int).tolist()) for r in res]
    assert tags[0].isdisjoint(tags[1]) and tags[0] | tags[1] == set(range(16))


def test_partition_balances_cost():
    from materialite_b200.serving import request_stream
    reqs = request_stream(64, 10.0, seed=1000)
    shares = [partition(reqs, 4, k) for k in range(4)]
    assert sorted(r.tag for s in shares for r in s) == list(range(64))
    costs = [sum(request_cost(r) for r in s) for s in shares]
    biggest = max(request_cost(r) for r in reqs)
    # LPT: no share exceeds the mean by more than one request
    assert max(costs) - np.mean(costs) <= biggest
