"""Shot-parallel gradients over ranks (one process per GPU).

Shots are independent, so each rank evaluates the misfit gradient of its own
shots with the whole model resident on its GPU, and one all-reduce sums the
3*nxyz gradient and the FP64 misfit (NCCL over NVLink on GPUs, gloo on CPU).
The split follows the reference's GPU groups: contiguous shot ranges, the
first `len(shots) % world` ranks taking one extra shot
(lib/vti-fwi-3d/gpu/objFuncGradient3d_f.cu:321-340).
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def shard(shots: Sequence[int], rank: int, world: int) -> list[int]:
    """Contiguous share of `shots` for `rank` of `world`."""
    n = len(shots)
    base, extra = divmod(n, world)
    if rank < extra:
        b = rank * (base + 1)
        e = b + base + 1
    else:
        b = extra * (base + 1) + (rank - extra) * base
        e = b + base
    return list(shots[b:e])


def gradient(local: Callable[[list[int]], tuple], shots: Sequence[int], group=None):
    """Sum over ranks of local(my_shots) = (gradient tensor, misfit).

    `local` returns a torch tensor (on the rank's device, or CPU under gloo)
    holding the local gradient and the local FP64 misfit; ranks without shots
    contribute zeros. Every rank returns the global (gradient, misfit).
    """
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return local(list(shots))
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    mine = shard(shots, rank, world)
    g, mis = local(mine)
    dist.all_reduce(g, group=group)
    m = torch.tensor([mis], dtype=torch.float64, device=g.device)
    dist.all_reduce(m, group=group)
    return g, float(m.item())


def plan_local(plan, souloc, dobs, dobs_mem, out):
    """local() for a vtib200.Plan3d: gradient of the given shots into the
    device tensor `out` (1 + 3*nxyz floats, entry 0 = misfit/2)."""
    from . import MEM_DEVICE

    def local(shots):
        if not shots:
            out.zero_()
            return out, 0.0
        _, mis = plan.gradient(souloc, np.asarray(shots, dtype=np.int32), dobs, dobs_mem,
                               out.data_ptr(), MEM_DEVICE)
        out[0] = 0.0  # the float misfit slot is rebuilt from the FP64 sum
        return out, mis

    return local
