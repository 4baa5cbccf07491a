"""The multi-GPU host logic on CPU: world_size-2 gloo process groups (no GPU)."""
import os
import socket

import torch.multiprocessing as mp

from qcb import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist = replicas.init("gloo", timeout_s=60)
    try:
        r, w, _ = replicas.env_rank()
        slow = replicas.max_over_ranks(10.0 * (rank + 1), dist)
        total = replicas.sum_over_ranks(rank + 1, dist)
        costs = [4096, 20736, 65536, 160000, 331776, 4096, 65536, 20736]
        mine = replicas.shard(costs, w)[r]
        dist.barrier()
        q.put((rank, slow, total, mine, replicas.replica_seed(7, r)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [20.0, 20.0]            # max over ranks
    assert [o[2] for o in out] == [3.0, 3.0]              # sum over ranks
    parts = [o[3] for o in out]
    assert sorted(parts[0] + parts[1]) == list(range(8))  # every lattice on exactly one rank
    assert out[0][4] != out[1][4]                         # independent replica seeds


def test_shard_balances_cost():
    costs = [100, 1, 1, 1, 50, 50]
    parts = replicas.shard(costs, 2)
    loads = [sum(costs[i] for i in p) for p in parts]
    assert sorted(loads) == [101, 102]
    assert replicas.shard([5.0], 3) == [[0], [], []]


def test_single_process_is_a_no_op(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.init("gloo") is None
    assert replicas.max_over_ranks(3.5) == 3.5


def test_slab_split_and_flow_buffers():
    from qcb import slabs

    assert slabs._split((4, 4, 4, 16), 4) == [(0, 4), (4, 4), (8, 4), (12, 4)]
    for bad in ((4, 4, 4, 12), 5), ((4, 4, 4, 12), 4):  # 12 / 5 not whole; 12 / 4 = 3 is odd
        try:
            slabs._split(*bad)
            raise AssertionError("accepted a bad split")
        except ValueError:
            pass
    # stage 1 and 3 write the work buffer on even steps, stage 2 the links; odd steps swap
    assert [slabs.flow_dst(s, 0) for s in (1, 2, 3)] == [slabs.WORK, slabs.LINKS, slabs.WORK]
    assert [slabs.flow_dst(s, 1) for s in (1, 2, 3)] == [slabs.LINKS, slabs.WORK, slabs.LINKS]
