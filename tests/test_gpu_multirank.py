"""Shards of one job on the GPU, two ranks (gloo), summed by
mcpet.parallel.allreduce_tallies: the library's own transport in each rank.

Each rank runs the head phantom with only its shard's emitting voxels
(mcpet.parallel.shard_activity) on the same GPU -- the ranks' kernels are
independent and never wait on one another -- and the integer tallies are
summed over the ranks.  With the reference lane layout every voxel keeps its
RANECU streams, so the sum equals one run of the whole job bit for bit.  The
ranks are spawned processes; the all-reduce runs over gloo on host tensors
(NCCL needs one GPU per rank).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
KEYS = ("trues", "scatter", "image_trues", "image_scatter", "spectrum")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _phantom():
    from mcpet import inputs
    return inputs.head_phantom(shape=(24, 48, 48), voxel_cm=0.5, seed=3, total_bq=4e5)


def _rank_main(rank, world, port, workdir, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "mcgpu-pet_b200"), root, os.path.join(root, "tests")]
    import mcpet
    from mcpet import inputs, parallel
    import scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mat, rho, act, vs, used = _phantom()
        sc = scenes.scene_from_arrays(workdir, mat, rho, parallel.shard_activity(act, rank, world), vs,
                                      tissues=used, seed=2468, **inputs.scanner_batch())
        r = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE))
        t = {k: torch.from_numpy(getattr(r, k).astype(np.int64)) for k in KEYS}
        t["histories"] = torch.tensor([r.total_histories], dtype=torch.int64)
        parallel.allreduce_tallies(t)
        if rank == 0:
            q.put({k: v.numpy() for k, v in t.items()} | {"mine": int(r.coincidences)})
        sc.close()
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_gpu_shards_sum_to_single_run(workdir):
    import mcpet
    from mcpet import inputs
    import scenes
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, workdir, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=600)
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    mat, rho, act, vs, used = _phantom()
    sc = scenes.scene_from_arrays(workdir, mat, rho, act, vs, tissues=used, seed=2468, **inputs.scanner_batch())
    full = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE))
    sc.close()
    assert 0 < res["mine"] < full.coincidences
    for k in KEYS:
        np.testing.assert_array_equal(res[k], getattr(full, k).astype(np.int64), err_msg=k)
    assert int(res["histories"][0]) == full.total_histories
