"""The multi-GPU path (independent replicas, one process per GPU) on CPU
with the gloo backend and world size 2: rendezvous, distinct replica seeds,
the max-over-ranks of the timed region and a clean shutdown."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from bd_box_b200 import ranks
    dist, r, w, local = ranks.init("gloo", timeout_s=60)
    assert (r, w, local) == (rank, world, rank)
    ranks.barrier(dist)
    t = ranks.max_over_ranks(dist, 10.0 + 5.0 * rank)
    seed = ranks.replica_seed(2, r)
    out.put((r, t, seed))
    ranks.finish(dist)


def test_two_ranks_gloo():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [t for _, t, _ in res] == [15.0, 15.0]          # the slowest rank's time
    assert len({s for _, _, s in res}) == 2                # replicas draw distinct noise


def test_single_process_needs_no_group():
    from bd_box_b200 import ranks
    for k in ("RANK", "WORLD_SIZE"):
        os.environ.pop(k, None)
    dist, r, w, _ = ranks.init("gloo")
    assert dist is None and (r, w) == (0, 1)
    assert ranks.max_over_ranks(dist, 3.5) == 3.5
    ranks.finish(dist)
