"""Host-side multi-GPU logic on CPU: gloo, world size 2 (no GPU involved)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from strut_b200 import distributed as D


def test_partition_is_balanced_and_complete():
    w = [97680, 11100, 44400, 60000, 23000, 5000, 81000, 33000, 12000]
    bins = D.partition_by_weight(w, 3)
    assert sorted(i for b in bins for i in b) == list(range(len(w)))
    loads = [sum(w[i] for i in b) for b in bins]
    assert max(loads) - min(loads) <= max(w)
    assert D.partition_by_weight(w, 3) == bins  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = [float(10 + 3 * i) for i in range(16)]
        share = D.rank_share(w, world, rank)
        t = D.max_over_ranks(1.5 + rank)
        stats = D.gather_stats({"rank": rank, "n": len(share), "share": share})
        q.put((rank, share, t, stats))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    shares = [r[1] for r in res]
    assert sorted(shares[0] + shares[1]) == list(range(16))
    assert not set(shares[0]) & set(shares[1])
    assert all(r[2] == 2.5 for r in res)  # max over ranks
    assert [s["rank"] for s in res[0][3]] == [0, 1]
