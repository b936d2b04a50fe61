"""The GPU side of sharded least-squares migration (poststackmig3d_b200.shard.lsm_sharded).
The CPU tests run the exchange with the oracle's operators; here each slab's GPU operators
(migration and spray of psm_slab_geometry's local problem, on the rank's halo) must match the
oracle's, and one rank on the GPU must follow Migrator.lsm_cg, the same algorithm on the
resident cube, with host arrays (lsm_sharded) and with every vector in device memory
(lsm_sharded_resident, through psm_forward_device / psm_adjoint_device)."""
import numpy as np
import pytest

import oracle as O
from poststackmig3d_b200 import Migrator, shard
from poststackmig3d_b200 import synth as S
from poststackmig3d_b200.migration import slab_geometry, split_slabs

from helpers import MAX_REL_TOL, REL_RMS_TOL, geometry_for, rel_err

pytestmark = pytest.mark.gpu


def _case():
    W = S.random_workload(83, 14, 9, 150, vel_kind="lateral", pad_il=2, pad_xl=1, d_il=60.0)
    return W, geometry_for(W)


def test_slab_operators_match_oracle():
    W, g = _case()
    rng = np.random.default_rng(4)
    vr = W.vrms_cube()
    for slab in split_slabs(g, 2, np.linspace(1.0, 3.0, g.n_oi)):
        o0, o1, i0, i1 = slab
        assert o1 > o0 and i1 > i0
        lg = slab_geometry(g, slab)
        d = rng.standard_normal((i1 - i0, g.n_xl, g.n_t)).astype(np.float32)
        rows = rng.standard_normal((o1 - o0, g.n_ox, g.n_t)).astype(np.float32)
        ops = shard._SlabOps(lg, np.ascontiguousarray(vr[i0:i1]), 0)
        try:
            fwd, adj = ops.forward(d), ops.adjoint(rows)
        finally:
            ops.close()
        t0 = lg.t0()
        ref_f = O.migrate_volume(d, vr[i0:i1], lg.out_center, lg.n_ox, lg.pad_il, lg.pad_xl,
                                 lg.m_il, np.float32(lg.dt_seconds), t0, np.float32(lg.tan2),
                                 lg.d_il, lg.d_xl, lg.amp, want64=True)[1]
        ref_a = O.adjoint_volume(rows.astype(np.float64), vr[i0:i1], lg.n_il, lg.n_xl,
                                 lg.out_center, lg.pad_il, lg.pad_xl, lg.m_il,
                                 np.float32(lg.dt_seconds), t0, np.float32(lg.tan2), lg.d_il,
                                 lg.d_xl, lg.amp, flags=O.CONTRACT)
        # the slab's image rows are the whole migration's rows [o0, o1)
        rms, mx = rel_err(fwd, ref_f)
        assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (slab, rms, mx)
        rms, mx = rel_err(adj, ref_a)
        assert rms <= 1e-4 and mx <= 1e-4, (slab, rms, mx)


def test_single_rank_follows_lsm_cg():
    W, g = _case()
    rng = np.random.default_rng(5)
    data = (W.data + 0.05 * rng.standard_normal(W.data.shape)).astype(np.float32)
    _, rows, hist = shard.lsm_sharded(g, data, W.vrms_cube(), 0, 1, 5)
    with Migrator(0) as m:
        m.set_geometry(g)
        m.set_vrms(W.vrms_cube())
        img, hist_ref = m.lsm_cg(data, 5)
    np.testing.assert_allclose(hist, hist_ref, rtol=1e-4)
    assert np.abs(rows - img).max() <= 1e-3 * np.abs(img).max()
    assert hist[-1] < hist[0]


def test_device_operators_equal_host_operators():
    """psm_forward_device / psm_adjoint_device on torch tensors give the host-array operators'
    bits (the same kernels on the same inputs)."""
    import torch
    W, g = _case()
    rng = np.random.default_rng(6)
    d = rng.standard_normal((g.n_il, g.n_xl, g.n_t)).astype(np.float32)
    rows = rng.standard_normal((g.n_oi, g.n_ox, g.n_t)).astype(np.float32)
    with Migrator(0) as m:
        m.set_geometry(g)
        m.set_vrms(W.vrms_cube())
        m.set_traces(d)
        fwd_host = m.forward()
        adj_host = m.adjoint(rows)
        stream = torch.cuda.ExternalStream(m.stream_handle())
        with torch.cuda.stream(stream):
            d_t = torch.from_numpy(d).cuda()
            rows_t = torch.from_numpy(rows).cuda()
            img_t = torch.empty(rows.shape, dtype=torch.float32, device="cuda")
            dat_t = torch.empty(d.shape, dtype=torch.float32, device="cuda")
            m.forward_device(d_t.data_ptr(), img_t.data_ptr())
            m.adjoint_device(rows_t.data_ptr(), dat_t.data_ptr())
        m.synchronize()
        assert np.array_equal(img_t.cpu().numpy(), fwd_host)
        # the spray's atomics add in a run-dependent order: equal to FP32 summation noise
        assert np.abs(dat_t.cpu().numpy() - adj_host).max() <= 1e-5 * np.abs(adj_host).max()


def test_resident_single_rank_follows_lsm_cg():
    """The device-resident sharded solver on one GPU (vectors as device tensors, CG scalars on
    the device) follows Migrator.lsm_cg."""
    W, g = _case()
    rng = np.random.default_rng(5)
    data = (W.data + 0.05 * rng.standard_normal(W.data.shape)).astype(np.float32)
    _, rows, hist = shard.lsm_sharded_resident(g, data, W.vrms_cube(), 0, 1, 5, device=0)
    assert rows.is_cuda
    rows = rows.cpu().numpy()
    with Migrator(0) as m:
        m.set_geometry(g)
        m.set_vrms(W.vrms_cube())
        img, hist_ref = m.lsm_cg(data, 5)
    np.testing.assert_allclose(hist, hist_ref, rtol=1e-4)
    assert np.abs(rows - img).max() <= 1e-3 * np.abs(img).max()
    assert hist[-1] < hist[0]
