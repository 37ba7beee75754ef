"""Batches shard by instance across ranks with no collective in the step loop.

The instances of a batch are independent cloths, so ranks split them:
scenes.shard_instances packs instances onto ranks by estimated cost, every
rank builds the block-diagonal scene of its shard (each instance at its
offset in the whole batch) and steps it alone; only the final per-rank
records are gathered on the host.  Checked with two gloo ranks on the CPU
(the FP64 oracle steps the shards): every instance is stepped exactly once,
the loads are balanced, and each instance's positions equal those of the
single-process batch."""
import os
import socket
import time

import numpy as np
import torch.multiprocessing as mp

from climatenet_b200 import abi, scenes

N_INSTANCES = 5
STEPS = 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _split(q, scene, ids):
    return {k: q[m["vertex_offset"]:m["vertex_offset"] + m["n_vertices"]].copy()
            for k, m in zip(ids, scene.meshes)}


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from oracle.oracle import Oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    insts = scenes.batch_instances(N_INSTANCES, seed=4)
    shard = scenes.shard_instances(insts, world)[rank]
    s, _, pk = scenes.batch_scene(n_instances=N_INSTANCES, seed=4, subset=shard)
    o = Oracle(s, abi.params(**pk))
    t0 = time.time()
    o.step(STEPS)                      # no collective while stepping
    ms = 1e3 * (time.time() - t0)
    qs, _ = o.state()
    records = [None] * world
    dist.all_gather_object(records, {"rank": rank, "instances": shard, "ms": ms})
    q.put((rank, _split(qs, s, shard), records))
    dist.destroy_process_group()


def test_partition_is_a_balanced_cover():
    insts = scenes.batch_instances(64, seed=4)
    for world in (1, 2, 4, 8):
        shards = scenes.shard_instances(insts, world)
        assert sorted(k for sh in shards for k in sh) == list(range(64))
        loads = [sum(scenes.instance_cost(insts[k]) for k in sh) for sh in shards]
        biggest = max(scenes.instance_cost(i) for i in insts)
        assert max(loads) - min(loads) <= biggest      # greedy LPT bound
        assert shards == scenes.shard_instances(insts, world)   # deterministic


def test_two_ranks_step_their_shards_like_the_whole_batch():
    from oracle.oracle import Oracle
    s, insts, pk = scenes.batch_scene(n_instances=N_INSTANCES, seed=4)
    o = Oracle(s, abi.params(**pk))
    o.step(STEPS)
    qa, _ = o.state()
    whole = _split(qa, s, range(N_INSTANCES))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seen = []
    for rank, parts, records in out:
        assert [r["rank"] for r in records] == [0, 1]
        assert sorted(k for r in records for k in r["instances"]) == list(range(N_INSTANCES))
        for k, qk in parts.items():
            seen.append(k)
            ref = whole[k]
            assert np.abs(qk - ref).max() <= 1e-9 * max(1.0, np.abs(ref).max()), (rank, k)
    assert sorted(seen) == list(range(N_INSTANCES))
