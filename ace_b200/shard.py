"""Splitting a batch of structures over ranks (one process per GPU).

Structures are independent, so inference needs no exchange: each rank
evaluates its own structures.  Training has one exchange per step, the
reference's MPI_Reduce + MPI_Bcast of the gradient (nnptefr.cpp:992,1074):
every rank returns the loss and gradient averaged over its own B_r
structures, and the batch average over B = sum_r B_r is
sum_r (B_r / B) (loss_r, grad_r), one all-reduce of a few thousand doubles.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np


def split_by_atoms(atom_off: np.ndarray, world: int) -> List[Tuple[int, int]]:
    """Contiguous structure ranges [s0, s1) per rank with about equal atom
    counts (every rank gets at least one structure when there are enough)."""
    atom_off = np.asarray(atom_off, dtype=np.int64)
    S = len(atom_off) - 1
    if world < 1:
        raise ValueError("world size must be positive")
    total = int(atom_off[-1])
    enough = S >= world
    bounds = [0]
    for r in range(1, world):
        s = int(np.searchsorted(atom_off, total * r / world, side="left"))
        lo = bounds[-1] + (1 if enough else 0)          # this rank keeps >= 1 structure
        hi = S - (world - r) if enough else S           # each later rank keeps >= 1
        bounds.append(min(max(s, lo), hi))
    bounds.append(S)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def local_batch(batch, rank: int, world: int):
    """This rank's sub-batch of a synth.Batch (same CSR layout)."""
    s0, s1 = split_by_atoms(batch.atom_off, world)[rank]
    return batch.subset(range(s0, s1)), (s0, s1)


def combine_loss_grad(loss: float, grad: np.ndarray, n_local: int, group=None):
    """Batch-average loss and gradient over all ranks from each rank's
    local average over n_local structures (torch.distributed all-reduce on
    `group`; any backend)."""
    import torch
    import torch.distributed as dist
    buf = torch.zeros(len(grad) + 2, dtype=torch.float64)
    buf[0] = float(loss) * n_local
    buf[1] = float(n_local)
    buf[2:] = torch.from_numpy(np.asarray(grad, dtype=np.float64) * n_local)
    if dist.is_available() and dist.is_initialized():
        dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else None
        if dev is not None:
            buf = buf.to(dev)
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
        buf = buf.cpu()
    B = float(buf[1])
    return float(buf[0]) / B, (buf[2:] / B).numpy()
