"""Least-squares migration sharded over ranks (poststackmig3d_b200.shard.lsm_sharded) on CPU:
gloo ranks each hold a slab of image rows and the halo of data inlines it reads; the spray's
contributions to shared inlines are summed between neighbours and the CG inner products over
ranks.  The oracle's forward and adjoint stand in for the GPU operators, so the sharded run
must follow the single-rank run of the same algorithm to summation-order rounding.  The
device-resident form (lsm_sharded_resident: torch tensors, CG scalars kept as tensors) runs
here on CPU tensors and must follow it too."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ITERS = 4


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from poststackmig3d_b200 import synth as S
    from helpers import geometry_for
    W = S.random_workload(82, 16, 6, 90, vel_kind="lateral", pad_il=2, pad_xl=1, d_il=80.0)
    rng = np.random.default_rng(3)
    data = (W.data + 0.05 * rng.standard_normal(W.data.shape)).astype(np.float32)
    return W, geometry_for(W), data


class OracleOps:
    """The oracle's migration and spray of one slab (test stand-in for the GPU operators)."""

    def __init__(self, lg, vrms, device):
        self.lg, self.vrms = lg, vrms

    def forward(self, d):
        import oracle as O
        lg = self.lg
        return O.migrate_volume(d, self.vrms, lg.out_center, lg.n_ox, lg.pad_il, lg.pad_xl,
                                lg.m_il, np.float32(lg.dt_seconds), lg.t0(),
                                np.float32(lg.tan2), lg.d_il, lg.d_xl, lg.amp)[0]

    def adjoint(self, rows):
        import oracle as O
        lg = self.lg
        return O.adjoint_volume(rows.astype(np.float64), self.vrms, lg.n_il, lg.n_xl,
                                lg.out_center, lg.pad_il, lg.pad_xl, lg.m_il,
                                np.float32(lg.dt_seconds), lg.t0(), np.float32(lg.tan2),
                                lg.d_il, lg.d_xl, lg.amp).astype(np.float32)


def _worker(rank, world, port, out_path, weight, resident):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime
    import torch.distributed as dist
    from poststackmig3d_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        W, g, data = _case()
        if resident:
            slab, rows, hist = shard.lsm_sharded_resident(g, data, W.vrms_cube(), rank, world,
                                                          ITERS, device=None, weight=weight,
                                                          make_ops=OracleOps)
            rows = rows.numpy()
        else:
            slab, rows, hist = shard.lsm_sharded(g, data, W.vrms_cube(), rank, world, ITERS,
                                                 weight=weight, make_ops=OracleOps)
        img = shard.gather_rows(g, slab, rows, rank, world, weight)
        np.save(out_path + f".hist{rank}.npy", hist)
        if rank == 0:
            np.save(out_path, img)
    finally:
        dist.destroy_process_group()


def _run(tmp_path, world, weight, resident=False):
    out = str(tmp_path / "img.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out, weight, resident))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert not p.is_alive() and p.exitcode == 0
    return out


def _single():
    from poststackmig3d_b200 import shard
    W, g, data = _case()
    slab, rows, hist = shard.lsm_sharded(g, data, W.vrms_cube(), 0, 1, ITERS,
                                         make_ops=OracleOps)
    assert slab[:2] == (0, g.n_oi)
    return rows, hist


def test_owned_ranges_partition_the_inlines():
    from poststackmig3d_b200 import shard
    slabs = [(0, 3, 0, 7), (3, 3, 0, 0), (3, 8, 1, 12), (8, 12, 5, 12)]
    assert shard.owned_ranges(slabs) == [(0, 7), (7, 7), (7, 12), (12, 12)]
    with pytest.raises(ValueError):
        shard.owned_ranges([(0, 2, 0, 4), (2, 4, 6, 9)])


def test_resident_single_rank_follows_host_arrays():
    from poststackmig3d_b200 import shard
    W, g, data = _case()
    rows1, hist1 = _single()
    slab, rows, hist = shard.lsm_sharded_resident(g, data, W.vrms_cube(), 0, 1, ITERS,
                                                  device=None, make_ops=OracleOps)
    assert slab[:2] == (0, g.n_oi)
    assert np.abs(rows.numpy() - rows1).max() <= 1e-5 * np.abs(rows1).max()
    np.testing.assert_allclose(hist, hist1, rtol=1e-6)


@pytest.mark.parametrize("resident", [False, True])
@pytest.mark.parametrize("world,skew", [(2, False), (3, True)])
def test_sharded_lsm_follows_single_rank(tmp_path, world, skew, resident):
    W, g, _ = _case()
    # a skewed work split gives uneven slabs and halos that overlap across two neighbours
    weight = np.linspace(1.0, 6.0, g.n_oi) if skew else None
    out = _run(tmp_path, world, weight, resident)
    rows1, hist1 = _single()
    img = np.load(out)
    assert img.shape == rows1.shape
    scale = np.abs(rows1).max()
    assert np.abs(img - rows1).max() <= 1e-4 * scale
    for r in range(world):  # every rank saw the same residual history
        h = np.load(out + f".hist{r}.npy")
        np.testing.assert_allclose(h, hist1, rtol=1e-5)
    assert hist1[-1] < hist1[0]
