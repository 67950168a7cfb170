"""Multi-rank paths on CPU (gloo, world size 2): sharding one job over ranks
and summing the tallies reproduces the single-device run exactly; replica
timing/count reductions behave as bench.py uses them."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from mcpet import inputs, parallel


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, workdir, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "mcgpu-pet_b200"), root, os.path.join(root, "tests")]
    from oracle import pyoracle
    import scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = scenes.sample_scene(workdir, seed=4321)
        osc = pyoracle.OracleScene(sc)
        voxels = parallel.shard_voxels(osc.act, rank, world).astype(np.int32)
        out = osc.run(n_threads=2, voxel_list=voxels)
        t = {k: torch.from_numpy(out[k].astype(np.int64)) for k in ("trues", "scatter", "image_trues",
                                                                     "image_scatter", "spectrum")}
        t["histories"] = torch.tensor([out["total_histories"]], dtype=torch.int64)
        parallel.allreduce_tallies(t)
        # replica-style reductions used by bench.py: max of times, sum of counts
        tm = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        if rank == 0:
            q.put({k: v.numpy() for k, v in t.items()} | {"tmax": float(tm.item()), "n_mine": len(voxels)})
        sc.close()
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_shards_sum_to_single_run(workdir):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, workdir, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    import scenes
    from oracle import pyoracle
    sc = scenes.sample_scene(workdir, seed=4321)
    full = pyoracle.OracleScene(sc).run(n_threads=2)
    for k in ("trues", "scatter", "image_trues", "image_scatter", "spectrum"):
        np.testing.assert_array_equal(res[k], full[k].astype(np.int64), err_msg=k)
    assert int(res["histories"][0]) == full["total_histories"]
    assert res["tmax"] == float(world)
    sc.close()


def test_shard_partition_is_complete_and_balanced():
    rng = np.random.default_rng(0)
    act = rng.gamma(0.5, 100.0, 10000).astype(np.float32)
    act[rng.random(10000) < 0.3] = 0.0
    for world in (1, 2, 3, 8):
        parts = [parallel.shard_voxels(act, r, world) for r in range(world)]
        allv = np.sort(np.concatenate(parts))
        np.testing.assert_array_equal(allv, np.nonzero(act > 1e-7)[0])
        loads = np.array([act[p].sum() for p in parts])
        assert loads.max() / loads.mean() < 1.05
        total = sum(parallel.shard_activity(act, r, world) for r in range(world))
        np.testing.assert_array_equal(total, np.where(act > 1e-7, act, 0))
    with pytest.raises(ValueError):
        parallel.shard_voxels(act, 2, 2)


def _replica_main(rank, world, port, workdir, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "mcgpu-pet_b200"), root, os.path.join(root, "tests")]
    from oracle import pyoracle
    import scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # every rank the whole job with its own seed (the benchmark's replicas)
        sc = scenes.sample_scene(workdir, seed=5000 + rank)
        out = pyoracle.OracleScene(sc).run(n_threads=2)
        t = {k: torch.from_numpy(out[k].astype(np.int64)) for k in ("trues", "scatter", "spectrum")}
        t["histories"] = torch.tensor([out["total_histories"]], dtype=torch.int64)
        parallel.allreduce_tallies(t)
        if rank == 0:
            q.put({k: v.numpy() for k, v in t.items()})
        sc.close()
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_replicas_reduce_to_the_sum_of_independent_runs(workdir):
    """Replicas (one seed per rank) summed by allreduce_tallies: the tallies of
    one acquisition world times as long, i.e. the sum of the single runs."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_replica_main, args=(r, world, port, workdir, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    import scenes
    from oracle import pyoracle
    want = {k: 0 for k in ("trues", "scatter", "spectrum", "histories")}
    for r in range(world):
        sc = scenes.sample_scene(workdir, seed=5000 + r)
        o = pyoracle.OracleScene(sc).run(n_threads=2)
        for k in ("trues", "scatter", "spectrum"):
            want[k] = want[k] + o[k].astype(np.int64)
        want["histories"] += o["total_histories"]
        sc.close()
    for k in ("trues", "scatter", "spectrum"):
        np.testing.assert_array_equal(res[k], want[k], err_msg=k)
    assert int(res["histories"][0]) == want["histories"]
