"""Multi-device use of the transport path (one process per GPU).

The path has no exchange step: lanes (voxel emission processes) are
independent.  Two ways to use N devices:

* replicas -- every rank runs the whole job with its own seed; the results are
  independent samples (the benchmark's weak-scaling mode);
* shards   -- the emitting voxels of ONE job are dealt to the ranks
  (``shard_activity``).  With the reference lane layout every voxel keeps its
  RANECU streams (stream id = voxel * threads_per_block + thread), so the sum
  over ranks of the integer tallies equals the single-device run exactly;
  ``allreduce_tallies`` adds them up (one int32/int64 sum-reduction per
  buffer, NCCL between GPUs or gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def shard_voxels(activity: np.ndarray, rank: int, world: int) -> np.ndarray:
    """Indices of the emitting voxels (activity > 1e-7 Bq, the reference's
    threshold) owned by ``rank``.  Voxels are sorted by decreasing activity
    and dealt in a serpentine order (0..w-1, w-1..0, ...), which balances the
    expected decays per rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    a = np.asarray(activity, dtype=np.float32).ravel()
    idx = np.nonzero(a > np.float32(1.0e-7))[0]
    order = idx[np.argsort(-a[idx], kind="stable")]
    pos = np.arange(len(order)) % (2 * world)
    owner = np.where(pos < world, pos, 2 * world - 1 - pos)
    return np.sort(order[owner == rank]).astype(np.int64)


def shard_activity(activity: np.ndarray, rank: int, world: int) -> np.ndarray:
    """Activity map of this rank's shard (zero outside it), same shape."""
    a = np.asarray(activity, dtype=np.float32)
    out = np.zeros(a.size, np.float32)
    mine = shard_voxels(a, rank, world)
    out[mine] = a.ravel()[mine]
    return out.reshape(a.shape)


def allreduce_tallies(tallies: dict, group=None) -> None:
    """Sum the integer tallies of all ranks in place (torch.distributed)."""
    import torch.distributed as dist
    for key in sorted(tallies):
        t = tallies[key]
        if t is None:
            continue
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
