"""One migration sharded over the GPUs of a node: one process per GPU (torch.distributed),
each migrating a slab of consecutive output inlines with the input inlines its buffers read
(psm_split_slabs / psm_slab_geometry).  Output-inline slabs of the forward operator are
independent, so there is no collective on the data path; the image rows are gathered on
rank 0 at the end.  The reference has no counterpart (one process, OpenMP over output inlines,
src/main.cpp:291-361).

Least-squares migration sharded the same way (lsm_sharded): image vectors are split in the
output-inline slabs, data vectors are held on each rank's halo of input inlines.  The adjoint
(spray) of a slab reaches its whole halo, and neighbouring halos overlap, so its contributions
are summed over the ranks that share an inline (halo_sum, point-to-point), and the CG inner
products are summed over ranks (each data inline counted once, by its owner).
lsm_sharded_resident runs the same iteration with every vector in device memory (torch
tensors, the library's device-pointer operators, halos swapped over NCCL).

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


# ----------------------------------------------------------------------------- sharded LSM


def owned_ranges(slabs):
    """Input inlines [a, b) each rank owns for the data-space inner products: consecutive
    ranges that partition the cube's inlines, each inside its rank's halo [i0, i1) (halos of
    neighbouring slabs overlap or touch, since every output inline reads its own centre)."""
    out, e = [], 0
    for o0, o1, i0, i1 in slabs:
        if o1 <= o0:
            out.append((e, e))
            continue
        if i0 > e:
            raise ValueError(f"halo [{i0}, {i1}) leaves inlines [{e}, {i0}) to no rank")
        out.append((e, max(e, i1)))
        e = max(e, i1)
    return out


class _Comm:
    """Exchanges of numpy arrays between ranks: CPU tensors (gloo) or device tensors (NCCL,
    `device` set)."""

    def __init__(self, rank: int, world: int, device=None):
        self.rank, self.world, self.device = rank, world, device

    def _t(self, a):
        import torch
        t = torch.from_numpy(np.ascontiguousarray(a))
        return t.to(self.device) if self.device is not None else t

    def allsum(self, x: float) -> float:
        """Sum of one float64 per rank, added in rank order (the same bits on every rank)."""
        if self.world == 1:
            return float(x)
        import torch
        import torch.distributed as dist
        mine = self._t(np.array([x], dtype=np.float64))
        parts = [torch.empty_like(mine) for _ in range(self.world)]
        dist.all_gather(parts, mine)
        total = 0.0
        for t in parts:
            total += float(t.cpu().numpy()[0])
        return total

    def halo_sum(self, part: np.ndarray, halo) -> np.ndarray:
        """This rank's halo of the sum over ranks of their halo arrays: every pair of ranks
        whose halos overlap swaps the overlap; the terms are added in rank order, so every
        rank holding an inline gets the same bits."""
        if self.world == 1:
            return part
        import torch
        import torch.distributed as dist
        i0, i1 = halo[self.rank]
        works, recv = [], {}
        for s in range(self.world):
            if s == self.rank:
                continue
            a0, a1 = max(i0, halo[s][0]), min(i1, halo[s][1])
            if a1 <= a0:
                continue
            send = self._t(part[a0 - i0:a1 - i0])
            buf = torch.empty_like(send)
            works.append(dist.isend(send, dst=s))
            works.append(dist.irecv(buf, src=s))
            recv[s] = (a0, a1, buf)
        for w in works:
            w.wait()
        total = np.zeros_like(part)
        for s in range(self.world):
            if s == self.rank:
                total += part
            elif s in recv:
                a0, a1, buf = recv[s]
                total[a0 - i0:a1 - i0] += buf.cpu().numpy()
        return total


class _SlabOps:
    """Forward (migration) and adjoint (spray) of one slab on a GPU, host arrays in and out."""

    def __init__(self, lg: Geometry, vrms: np.ndarray, device: int):
        self.m = Migrator(device)
        self.m.set_geometry(lg)
        self.m.set_vrms(vrms)

    def forward(self, d: np.ndarray) -> np.ndarray:
        self.m.set_traces(d)
        return self.m.forward()

    def adjoint(self, rows: np.ndarray) -> np.ndarray:
        return self.m.adjoint(rows)

    def close(self):
        self.m.close()


def lsm_sharded(g: Geometry, data: np.ndarray, vrms: np.ndarray, rank: int, world: int,
                iters: int, device: int = 0, weight=None, make_ops: Optional[Callable] = None,
                nccl: bool = False):
    """CGLS on min ||M^T m - data||^2 (M the migration, M^T the spray), as Migrator.lsm_cg, with
    the image split in output-inline slabs over `world` ranks.  Returns (slab, this rank's image
    rows [o1 - o0][n_ox][n_t], data-residual norms [iters + 1]); gather_rows collects the
    image.  data and vrms are the whole cube's [n_il][n_xl][n_t] (only this rank's halo is
    read).  `make_ops` (local geometry, halo Vrms, device) -> object with forward(halo data)
    -> rows and adjoint(rows) -> halo data replaces the GPU operators (tests).

    Per iteration: one adjoint and one forward per rank on its slab, one halo exchange (the
    adjoint's contributions to inlines that neighbouring halos share) and three scalar sums.
    Every rank takes the same collective steps, empty slabs included."""
    slabs = split_slabs(g, world, weight)
    owned = owned_ranges(slabs)
    halo = [(s[2], s[3]) if s[1] > s[0] else (a, a) for s, (a, _) in zip(slabs, owned)]
    o0, o1 = slabs[rank][0], slabs[rank][1]
    i0, i1 = halo[rank]
    a0, a1 = owned[rank]
    comm = _Comm(rank, world, f"cuda:{device}" if nccl else None)
    shape_d = (i1 - i0, g.n_xl, g.n_t)
    shape_m = (max(o1 - o0, 0), g.n_ox, g.n_t)
    ops = None
    if o1 > o0:
        lg = slab_geometry(g, slabs[rank])
        ops = (make_ops or _SlabOps)(lg, np.ascontiguousarray(vrms[i0:i1], dtype=np.float32),
                                     device)

    def fwd(d):
        return np.asarray(ops.forward(d), dtype=np.float32) if ops else np.zeros(shape_m,
                                                                                  np.float32)

    def adj(rows):
        part = (np.asarray(ops.adjoint(rows), dtype=np.float32) if ops
                else np.zeros(shape_d, np.float32))
        return comm.halo_sum(part, halo)

    def ddot(x, y):  # data space: owned inlines only
        lo, hi = a0 - i0, a1 - i0
        return comm.allsum(float(np.dot(x[lo:hi].ravel().astype(np.float64),
                                        y[lo:hi].ravel().astype(np.float64))))

    def mdot(x, y):
        return comm.allsum(float(np.dot(x.ravel().astype(np.float64),
                                        y.ravel().astype(np.float64))))

    try:
        r = np.ascontiguousarray(data[i0:i1], dtype=np.float32).copy()  # d - M^T 0
        m = np.zeros(shape_m, dtype=np.float32)
        hist = [ddot(r, r)]
        s = fwd(r)
        p = s.copy()
        gamma = mdot(s, s)
        for _ in range(iters):
            q = adj(p)                                     # q = M^T p
            delta = ddot(q, q)
            alpha = np.float32(gamma / delta if delta > 0.0 else 0.0)
            m += alpha * p
            r -= alpha * q
            hist.append(ddot(r, r))
            s = fwd(r)                                     # s = M r
            gamma_new = mdot(s, s)
            beta = np.float32(gamma_new / gamma if gamma > 0.0 else 0.0)
            gamma = gamma_new
            p = s + beta * p
    finally:
        if ops is not None and hasattr(ops, "close"):
            ops.close()
    return slabs[rank], m, np.sqrt(np.maximum(np.array(hist), 0.0))


# ------------------------------------------------------------ sharded LSM, vectors on the device


class _TorchComm:
    """Exchanges of torch tensors between ranks: device tensors over NCCL, CPU tensors over
    gloo.  Sums are formed in rank order, so every rank gets the same bits."""

    def __init__(self, rank: int, world: int):
        self.rank, self.world = rank, world

    def allsum(self, x):
        """Sum over ranks of a 0-d float64 tensor (stays on its device)."""
        if self.world == 1:
            return x
        import torch
        import torch.distributed as dist
        mine = x.reshape(1)
        parts = [torch.empty_like(mine) for _ in range(self.world)]
        dist.all_gather(parts, mine)
        total = parts[0]
        for t in parts[1:]:
            total = total + t
        return total.reshape(())

    def halo_sum(self, part, halo):
        """As _Comm.halo_sum, on tensors: each pair of ranks whose halos overlap swaps the
        overlap point to point (device memory over NCCL: only the halo crosses NVLink)."""
        if self.world == 1:
            return part
        import torch
        import torch.distributed as dist
        i0, i1 = halo[self.rank]
        works, recv = [], {}
        for s in range(self.world):
            if s == self.rank:
                continue
            a0, a1 = max(i0, halo[s][0]), min(i1, halo[s][1])
            if a1 <= a0:
                continue
            send = part[a0 - i0:a1 - i0].contiguous()
            buf = torch.empty_like(send)
            works.append(dist.isend(send, dst=s))
            works.append(dist.irecv(buf, src=s))
            recv[s] = (a0, a1, buf)
        for w in works:
            w.wait()
        total = torch.zeros_like(part)
        for s in range(self.world):
            if s == self.rank:
                total += part
            elif s in recv:
                a0, a1, buf = recv[s]
                total[a0 - i0:a1 - i0] += buf
        return total


class _DeviceSlabOps:
    """Forward and adjoint of one slab on device tensors (psm_forward_device /
    psm_adjoint_device), enqueued on the library context's stream, which the solver's torch
    work also runs on."""

    def __init__(self, lg: Geometry, vrms: np.ndarray, device: int):
        import torch
        self.m = Migrator(device)
        self.m.set_geometry(lg)
        self.m.set_vrms(vrms)
        self.dev = torch.device(f"cuda:{device}")
        self.stream = torch.cuda.ExternalStream(self.m.stream_handle(), device=self.dev)
        self.shape_m = (lg.n_oi, lg.n_ox, lg.n_t)
        self.shape_d = (lg.n_il, lg.n_xl, lg.n_t)

    def forward(self, d):
        import torch
        d = d.contiguous()
        out = torch.empty(self.shape_m, dtype=torch.float32, device=self.dev)
        self.m.forward_device(d.data_ptr(), out.data_ptr())
        return out

    def adjoint(self, rows):
        import torch
        rows = rows.contiguous()
        out = torch.empty(self.shape_d, dtype=torch.float32, device=self.dev)
        self.m.adjoint_device(rows.data_ptr(), out.data_ptr())
        return out

    def close(self):
        self.m.synchronize()  # raises on a device error of the last operators
        self.m.close()


def lsm_sharded_resident(g: Geometry, data: np.ndarray, vrms: np.ndarray, rank: int, world: int,
                         iters: int, device: Optional[int] = 0, weight=None,
                         make_ops: Optional[Callable] = None):
    """lsm_sharded with every vector in device memory: the data residual r and q on this
    rank's halo of input inlines, the image m, s and p on its slab, all torch tensors on
    cuda:`device`, and the CG scalars (inner products, alpha, beta) as device scalars, so no
    iteration waits for the host.  Per iteration each rank runs one adjoint and one forward on
    its slab (psm_adjoint_device / psm_forward_device on the library's stream, which the torch
    work shares), swaps the overlap of neighbouring halos point to point and sums three
    scalars over the ranks; with the nccl backend only those halos and scalars leave the GPU.

    device None runs on CPU tensors (gloo), with `make_ops` (local geometry, halo Vrms, None)
    -> an object whose forward(halo data) -> rows and adjoint(rows) -> halo data take and return
    numpy arrays (tests; the oracle stands in for the GPU operators).  Returns (slab, this
    rank's image rows as a tensor on the solver's device, data-residual norms [iters + 1])."""
    import contextlib
    import torch
    slabs = split_slabs(g, world, weight)
    owned = owned_ranges(slabs)
    halo = [(s[2], s[3]) if s[1] > s[0] else (a, a) for s, (a, _) in zip(slabs, owned)]
    o0, o1 = slabs[rank][0], slabs[rank][1]
    i0, i1 = halo[rank]
    a0, a1 = owned[rank]
    comm = _TorchComm(rank, world)
    dev = torch.device("cpu") if device is None else torch.device(f"cuda:{device}")
    shape_d = (i1 - i0, g.n_xl, g.n_t)
    shape_m = (max(o1 - o0, 0), g.n_ox, g.n_t)
    ops = None
    if o1 > o0:
        lg = slab_geometry(g, slabs[rank])
        ops = (make_ops or _DeviceSlabOps)(
            lg, np.ascontiguousarray(vrms[i0:i1], dtype=np.float32), device)

    def fwd(d):
        if ops is None:
            return torch.zeros(shape_m, dtype=torch.float32, device=dev)
        if device is None:
            return torch.from_numpy(np.asarray(ops.forward(d.numpy()), dtype=np.float32))
        return ops.forward(d)

    def adj(rows):
        if ops is None:
            part = torch.zeros(shape_d, dtype=torch.float32, device=dev)
        elif device is None:
            part = torch.from_numpy(np.asarray(ops.adjoint(rows.numpy()), dtype=np.float32))
        else:
            part = ops.adjoint(rows)
        return comm.halo_sum(part, halo)

    def ddot(x, y):  # data space: owned inlines only
        lo, hi = a0 - i0, a1 - i0
        return comm.allsum(torch.dot(x[lo:hi].reshape(-1).double(),
                                     y[lo:hi].reshape(-1).double()))

    def mdot(x, y):
        return comm.allsum(torch.dot(x.reshape(-1).double(), y.reshape(-1).double()))

    def ratio(a, b):  # a / b, 0 where b is not positive (device scalars)
        return torch.where(b > 0, a / torch.where(b > 0, b, torch.ones_like(b)),
                           torch.zeros_like(a))

    stream = getattr(ops, "stream", None) if device is not None else None
    ctx = torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()
    try:
        with ctx:
            r = torch.from_numpy(np.ascontiguousarray(data[i0:i1], dtype=np.float32)).to(dev)
            m = torch.zeros(shape_m, dtype=torch.float32, device=dev)
            hist = [ddot(r, r)]
            s = fwd(r)
            p = s.clone()
            gamma = mdot(s, s)
            for _ in range(iters):
                q = adj(p)                                   # q = M^T p
                delta = ddot(q, q)
                alpha = ratio(gamma, delta).float()
                m += alpha * p
                r -= alpha * q
                hist.append(ddot(r, r))
                s = fwd(r)                                   # s = M r
                gamma_new = mdot(s, s)
                beta = ratio(gamma_new, gamma).float()
                gamma = gamma_new
                p = s + beta * p
            res = torch.stack(hist).cpu().numpy()
    finally:
        if ops is not None and hasattr(ops, "close"):
            ops.close()
    return slabs[rank], m, np.sqrt(np.maximum(res, 0.0))
