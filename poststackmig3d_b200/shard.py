"""One migration sharded over the GPUs of a node: one process per GPU (torch.distributed),
each migrating a slab of consecutive output inlines with the input inlines its buffers read
(psm_split_slabs / psm_slab_geometry).  Output-inline slabs of the forward operator are
independent, so there is no collective on the data path; the image rows are gathered on
rank 0 at the end.  The reference has no counterpart (one process, OpenMP over output inlines,
src/main.cpp:291-361).

The split balances work: the weight of an output inline is its term count when known
(Migrator.count_terms_rows), else 1.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np

from .migration import Geometry, Migrator, Slab, slab_geometry, split_slabs


def shard_slab(g: Geometry, rank: int, world: int, weight=None) -> Slab:
    """The slab (o0, o1, i0, i1) of `rank` among `world` ranks."""
    return split_slabs(g, world, weight)[rank]


def _gpu_migrate(lg: Geometry, traces: np.ndarray, vrms: np.ndarray,
                 device: int) -> np.ndarray:
    with Migrator(device) as m:
        m.set_geometry(lg)
        m.set_traces(traces)
        m.set_vrms(vrms)
        return m.forward()


def migrate_shard(g: Geometry, traces: np.ndarray, vrms: np.ndarray, rank: int, world: int,
                  device: int = 0, weight=None,
                  migrate: Optional[Callable] = None):
    """Migrate this rank's slab: returns (slab, rows [o1 - o0][n_ox][n_t]).  traces and vrms
    are the whole cube's [n_il][n_xl][n_t] (only inlines [i0, i1) are read).  `migrate`
    (local geometry, traces, vrms, device) -> rows replaces the GPU operator (tests)."""
    slab = shard_slab(g, rank, world, weight)
    o0, o1, i0, i1 = slab
    if o1 <= o0:
        return slab, np.zeros((0, g.n_ox, g.n_t), dtype=np.float32)
    lg = slab_geometry(g, slab)
    rows = (migrate or _gpu_migrate)(lg, np.ascontiguousarray(traces[i0:i1]),
                                     np.ascontiguousarray(vrms[i0:i1]), device)
    return slab, np.asarray(rows, dtype=np.float32)


def gather_rows(g: Geometry, slab: Slab, rows: np.ndarray, rank: int, world: int,
                weight=None, device=None) -> Optional[np.ndarray]:
    """Collect every rank's rows into the whole image on rank 0 (None on other ranks).
    Point-to-point sends of each slab's rows: CPU tensors with gloo, device tensors with
    NCCL (`device` set)."""
    import torch
    import torch.distributed as dist

    def as_tensor(a):
        t = torch.from_numpy(np.ascontiguousarray(a))
        return t.to(device) if device is not None else t

    if world == 1:
        return rows
    slabs = split_slabs(g, world, weight)
    if rank != 0:
        if slab[1] > slab[0]:
            dist.send(as_tensor(rows), dst=0)
        return None
    image = np.zeros((g.n_oi, g.n_ox, g.n_t), dtype=np.float32)
    image[slab[0]:slab[1]] = rows
    for r in range(1, world):
        o0, o1 = slabs[r][0], slabs[r][1]
        if o1 <= o0:
            continue
        buf = as_tensor(np.empty((o1 - o0, g.n_ox, g.n_t), dtype=np.float32))
        dist.recv(buf, src=r)
        image[o0:o1] = buf.cpu().numpy()
    return image


def migrate_sharded(g: Geometry, traces: np.ndarray, vrms: np.ndarray, rank: int,
                    world: int, device: int = 0, weight=None,
                    migrate: Optional[Callable] = None, nccl: bool = False):
    """The whole image on rank 0 (None elsewhere), each rank migrating its slab."""
    slab, rows = migrate_shard(g, traces, vrms, rank, world, device, weight, migrate)
    return gather_rows(g, slab, rows, rank, world, weight,
                       device=f"cuda:{device}" if nccl else None)
