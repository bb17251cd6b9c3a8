"""Multi-GPU splits of the hot path (one process per GPU, torch.distributed).

* Independent slices (the fan batches): each rank takes its own slices; no
  collective on the data path (bench.py's weak-scaling mode).
* One large volume (the cylindrical cone-beam pair): the views are split
  into contiguous shards.  The forward projection of a shard needs nothing
  from the other ranks; the backprojection of a shard is a partial volume,
  and the volume is their sum -- one all-reduce (NCCL over NVLink on GPUs)
  per backprojection, of nx*ny*nz floats.  ``ViewShardedPair`` implements that
  split over any local projector pair, so the partition and the summation
  are tested on CPU ranks (gloo) with the oracle as the local pair.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple

import numpy as np
import torch
import torch.distributed as dist


def view_shards(nview: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous [begin, end) view ranges, one per rank, sizes differing by at most one."""
    base, extra = divmod(nview, world)
    out, b = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((b, b + n))
        b += n
    return out


class ViewShardedPair:
    """A projector pair over the views [begin, end) of this rank.

    project(vol) -> this rank's projections [B, nu, n_local, nv];
    backproject(prj_local) -> the full backprojection (partial volumes summed
    over the ranks with one all-reduce); gather(prj_local) -> all projections.
    ``make_local(angles_local)`` returns (fp, bp) callables for the rank's
    views: a CylPlan's project / backproject on a GPU, or any other pair."""

    def __init__(self, angles, make_local: Callable, group=None):
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        ang = np.asarray(angles, np.float32)
        self.shards = view_shards(ang.size, self.world)
        b, e = self.shards[self.rank]
        self.begin, self.end = b, e
        self.fp, self.bp = make_local(np.ascontiguousarray(ang[b:e]))

    def project(self, vol: torch.Tensor) -> torch.Tensor:
        return self.fp(vol)

    def backproject(self, prj_local: torch.Tensor) -> torch.Tensor:
        part = self.bp(prj_local)
        if self.world > 1:
            dist.all_reduce(part, op=dist.ReduceOp.SUM, group=self.group)
        return part

    def gather(self, prj_local: torch.Tensor) -> torch.Tensor:
        """All ranks' projections along the view axis (dim 2)."""
        if self.world == 1:
            return prj_local
        sizes = [e - b for b, e in self.shards]
        width = max(sizes)
        pad = torch.zeros(prj_local.shape[:2] + (width,) + prj_local.shape[3:], dtype=prj_local.dtype,
                          device=prj_local.device)
        pad[:, :, :prj_local.shape[2]] = prj_local
        bufs = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(bufs, pad, group=self.group)
        return torch.cat([t[:, :, :n] for t, n in zip(bufs, sizes)], dim=2)


def cyl_sharded_pair(geom, angles, device=None, group=None) -> ViewShardedPair:
    """ViewShardedPair over the sm_100a cylindrical cone-beam kernels."""
    from .torch_ops import CylPlan

    def make(ang_local):
        plan = CylPlan(geom, ang_local, device=device)
        return plan.project, plan.backproject

    return ViewShardedPair(angles, make, group)
