"""One solve split over several GPUs by k-grid rows.

k-points are independent for the whole pulse, so a solve splits into row slabs with no exchange
while it runs; each rank propagates its slab (SWESim_set_k_rows) and the partial currents, already
normalised by the full grid, are summed once at the end (nt x 3 complex values).  With
torch.distributed this is one all_reduce over NCCL (GPUs) or gloo (CPU).
"""
from __future__ import annotations

import numpy as np


def row_slab(rank: int, world: int, n_rows: int) -> tuple[int, int]:
    """Rows [r0, r1) of `rank`: contiguous, sizes differing by at most one, in rank order."""
    if not (0 <= rank < world) or n_rows < world:
        raise ValueError(f"cannot split {n_rows} rows over {world} ranks")
    base, extra = divmod(n_rows, world)
    r0 = rank * base + min(rank, extra)
    return r0, r0 + base + (1 if rank < extra else 0)


def reduce_current(J_partial: np.ndarray, group=None, device=None) -> np.ndarray:
    """Sum the [3, nt] complex partial currents of all ranks (every rank gets the total)."""
    import torch
    import torch.distributed as dist

    t = torch.from_numpy(np.ascontiguousarray(J_partial).view(np.float64).copy())
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy().view(np.complex128).reshape(J_partial.shape)


def run_slab(param: dict, rank: int, world: int, device: int | None = None):
    """Propagate this rank's slab on its GPU; returns (t, partial J[3, nt])."""
    from pySWE import pyswe

    r0, r1 = row_slab(rank, world, int(param["nr1"]))
    swe = pyswe.SWE(pyswe.Settings(dict(param)), device=device, k_rows=(r0, r1))
    swe.run_simulation()
    t, jx, jy, jz = swe.get_current()
    swe.delete()
    return np.real(t), np.stack([jx, jy, jz])
