"""Slabs of output inlines (psm_plan_slabs / psm_split_slabs / psm_slab_geometry): the
planner runs on the host without a GPU, and a slab migrated on its own must give exactly the
rows of the whole image.  The oracle stands in for the operator here (CPU); the GPU path of
the same geometry is tested in test_slabs_gpu.py."""
import numpy as np
import pytest

import oracle as O
from poststackmig3d_b200 import synth as S
from poststackmig3d_b200.migration import plan_slabs, slab_bytes, slab_geometry, split_slabs

from helpers import geometry_for, oracle_forward

CASES = [  # short inline halos (m_il 3 and 2), so that slabs are much smaller than the cube
    dict(seed=61, n_il=20, n_xl=6, n_t=90, vel_kind="linear", pad_il=3, pad_xl=1, d_il=100.0),
    dict(seed=62, n_il=15, n_xl=5, n_t=70, vel_kind="lateral", angle=20.0, d_il=60.0),
]


def _workload(case):
    c = dict(case)
    return S.random_workload(c.pop("seed"), c.pop("n_il"), c.pop("n_xl"), c.pop("n_t"), **c)


def _reads(g, o):
    c = int(g.out_center[o])
    return max(0, c - g.m_il - g.pad_il), min(g.n_il, c + g.m_il + 1 + g.pad_il)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"seed{c['seed']}")
def test_plan_slabs_covers_rows_within_budget(case):
    g = geometry_for(_workload(case))
    one = max(slab_bytes(g, _reads(g, o)[1] - _reads(g, o)[0], 1) for o in range(g.n_oi))
    for budget in (0, one, int(one * 1.7), 10 * one):
        slabs = plan_slabs(g, budget)
        assert slabs[0][0] == 0 and slabs[-1][1] == g.n_oi
        for a, b in zip(slabs, slabs[1:]):
            assert a[1] == b[0]
        for o0, o1, i0, i1 in slabs:
            lo = min(_reads(g, o)[0] for o in range(o0, o1))
            hi = max(_reads(g, o)[1] for o in range(o0, o1))
            assert (i0, i1) == (lo, hi)
            if budget:
                assert slab_bytes(g, i1 - i0, o1 - o0) <= budget
        if budget == 0:
            assert len(slabs) == 1
        if budget == one:
            assert len(slabs) > 1
    with pytest.raises(Exception):
        plan_slabs(g, one - 1)


def test_split_slabs_balances_work():
    g = geometry_for(_workload(CASES[0]))
    w = np.linspace(1.0, 3.0, g.n_oi)
    for n in (1, 2, 3, 5):
        parts = split_slabs(g, n, w)
        assert parts[0][0] == 0 and parts[-1][1] == g.n_oi
        work = [w[a:b].sum() for a, b, _, _ in parts]
        assert max(work) - min(work) <= w.max() + 1e-9, (n, work)
    parts = split_slabs(g, g.n_oi + 3)  # more parts than rows: some are empty
    assert sum(b - a for a, b, _, _ in parts) == g.n_oi


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"seed{c['seed']}")
def test_slab_migrated_alone_equals_rows_of_whole_image(case):
    W = _workload(case)
    g = geometry_for(W)
    whole, _, _ = oracle_forward(W, g)
    vr = W.vrms_cube()
    one = max(slab_bytes(g, _reads(g, o)[1] - _reads(g, o)[0], 1) for o in range(g.n_oi))
    slabs = plan_slabs(g, int(one * 1.1))
    assert len(slabs) >= 2
    for s in slabs:
        o0, o1, i0, i1 = s
        lg = slab_geometry(g, s)
        assert lg.n_il == i1 - i0 and lg.n_oi == o1 - o0
        part = O.migrate_volume(W.data[i0:i1], vr[i0:i1], lg.out_center, lg.n_ox, lg.pad_il,
                                lg.pad_xl, lg.m_il, np.float32(lg.dt_seconds), lg.t0(),
                                np.float32(lg.tan2), lg.d_il, lg.d_xl, lg.amp)[0]
        assert np.array_equal(part, whole[o0:o1]), s
