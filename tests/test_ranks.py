"""The multi-GPU path (independent replicas, one process per GPU) on CPU
with the gloo backend and world size 2: rendezvous, distinct replica seeds,
the max-over-ranks of the timed region, the replica sharder
(bdb_shard_replicas, host-only) and a clean shutdown."""
import os
import socket

import numpy as np
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
    # every rank shards the same replica list by itself: the answers agree
    from bd_box_b200 import decks, engine
    mine = [int(k) for k in np.flatnonzero(engine.shard_replicas(decks.replica_sizes(), w) == r)]
    gathered = [None] * w
    dist.all_gather_object(gathered, mine)
    assert sorted(sum(gathered, [])) == list(range(len(decks.replica_sizes())))
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


def _cost(n):
    return n.astype(np.int64) ** 2 + n


@pytest.mark.parametrize("nshards", [1, 2, 3, 4, 8])
def test_shard_replicas_balances(nshards):
    from bd_box_b200 import decks, engine
    sizes = decks.replica_sizes()
    sh = engine.shard_replicas(sizes, nshards)
    assert sh.shape == sizes.shape and sh.min() >= 0 and sh.max() < nshards
    load = np.bincount(sh, weights=_cost(sizes), minlength=nshards)
    c = _cost(sizes)
    # longest-processing-time greedy: within 4/3 of the optimum, which is
    # at least the mean load and at least the largest replica
    assert load.max() <= 4 / 3 * max(c.sum() / nshards, c.max()) + 1e-9
    assert np.array_equal(sh, engine.shard_replicas(sizes, nshards))


def test_shard_replicas_small_cases():
    from bd_box_b200 import engine
    # decreasing cost to the least-loaded shard, ties to the lower index
    assert engine.shard_replicas([10, 10, 10, 10], 2).tolist() == [0, 1, 0, 1]
    assert engine.shard_replicas([100, 3, 3, 3], 2).tolist() == [0, 1, 1, 1]
    # more shards than replicas: the extra shards stay empty
    assert engine.shard_replicas([5, 7], 4).tolist() == [1, 0]
    assert engine.shard_replicas([], 3).size == 0
    for bad in (([5, 1], 2), ([5, 6], 0)):
        with pytest.raises(engine.BDBError):
            engine.shard_replicas(*bad)


def test_bench_gpus_flag_launches_that_many_ranks():
    """`bench.py --gpus 2` started without torchrun starts two ranks itself
    (torch.distributed.run on this node) and reports n_gpus 2 with the
    slowest rank's time; the stub step keeps the GPU out of it."""
    import json
    import subprocess
    import sys
    pytest.importorskip("torch")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--stub", "--steps", "5",
                        "--warmup", "3"], capture_output=True, text=True, timeout=240, env=env, cwd=root)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    out = json.loads(lines[0])
    assert out["n_gpus"] == 2 and out["steps"] == 5
    # rank 1 sleeps 20 ms per step: the job's time is its time
    assert out["ms_per_step"] >= 19.0
