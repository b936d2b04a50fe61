"""Batched migration: velocity-scan panels over one cube and uneven sub-volumes in one
persistent launch (replayed as a CUDA graph) against the same problems run one at a time.

Each output sample is summed by one CTA over the same trace sequence whether its tile runs in
the grid kernel or in the persistent kernel, so the images must be bit-identical; the
single-problem path itself is held to the oracle by test_forward_gpu.py (and one panel is
checked against the oracle here)."""
import dataclasses

import numpy as np
import pytest

import oracle as O
from poststackmig3d_b200 import Batch, Migrator, Problem
from poststackmig3d_b200 import synth as S

from helpers import MAX_REL_TOL, REL_RMS_TOL, geometry_for, oracle_forward, rel_err

pytestmark = pytest.mark.gpu

PANEL_V = [1800.0, 2300.0, 3100.0]


def _problems(precision="f32"):
    """Three constant-velocity panels over one cube, a sub-volume with a Vrms cube and
    padding, and one with a single Vrms(t) trace."""
    base = S.random_workload(31, 12, 11, 230, vel_kind="const", angle=40.0, pad_xl=2)
    cube = np.ascontiguousarray(base.data)
    out = []
    for v in PANEL_V:
        W = dataclasses.replace(base, velocity=v)
        g = dataclasses.replace(geometry_for(W), precision=precision)
        out.append((W, g, Problem(g, cube, velocity=v)))
    W = S.random_workload(32, 9, 14, 300, vel_kind="lateral", pad_il=2, pad_xl=1)
    g = dataclasses.replace(geometry_for(W), precision=precision)
    out.append((W, g, Problem(g, W.data, W.vrms_cube())))
    W = S.random_workload(33, 16, 7, 130, vel_kind="linear", angle=55.0)
    g = dataclasses.replace(geometry_for(W), precision=precision)
    out.append((W, g, Problem(g, W.data, W.vrms_cube()[0, 0].copy())))
    return out


def _single(W, g, variant=0):
    with Migrator(0) as m:
        m.set_geometry(g)
        m.set_traces(W.data)
        m.set_vrms(W.vrms_cube())
        if variant:
            m.set_variant(variant)
        img = m.forward()
        n = m.count_terms()
    return img, n


@pytest.mark.parametrize("variant", [0, 5, 1, 11, 13])
@pytest.mark.parametrize("mode,order", [(Batch.PERSISTENT, Batch.DEPTH_FIRST),
                                        (Batch.PERSISTENT, Batch.PROBLEM_ORDER),
                                        (Batch.PER_PROBLEM, Batch.DEPTH_FIRST),
                                        (Batch.ONE_GRID, Batch.DEPTH_FIRST),
                                        (Batch.ONE_GRID, Batch.PROBLEM_ORDER)])
def test_batch_matches_single_problem_runs(mode, order, variant):
    probs = _problems()
    singles = [_single(W, g, variant) for W, g, _ in probs]
    with Migrator(0) as m, Batch(m, [p for _, _, p in probs]) as b:
        b.set_mode(mode)
        b.set_order(order)
        if variant:
            b.set_variant(variant)
        for rep in range(2):  # capture, then replay of the graph
            b.run()
            for i, (img1, _) in enumerate(singles):
                assert np.array_equal(b.image(i), img1), (rep, i)
        assert b.count_terms() == sum(n for _, n in singles)


def test_batch_panel_against_oracle():
    probs = _problems()
    with Migrator(0) as m, Batch(m, [p for _, _, p in probs]) as b:
        b.run()
        for i in (0, 3):
            W, g, _ = probs[i]
            ref, _, _ = oracle_forward(W, g)
            rms, mx = rel_err(b.image(i), ref)
            assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (i, rms, mx)


def test_batch_bf16_and_reload():
    probs = _problems("bf16")
    singles = [_single(W, g, 4)[0] for W, g, _ in probs]
    with Migrator(0) as m, Batch(m, [p for _, _, p in probs]) as b:
        best, order, mode, ms = b.autotune()
        assert best in (4, 5, 9, 11, 12) and order in (0, 1) and mode in (0, 1, 2)
        assert {v for v, _ in ms} == {4, 5, 9, 11, 12}
        assert {s for _, s in ms} == {0, 1, 2, 3, 4}
        b.set_variant(4)
        b.set_mode(Batch.PERSISTENT)
        b.set_order(Batch.PROBLEM_ORDER)
        b.run()
        first = [b.image(i) for i in range(len(probs))]
        for i, img1 in enumerate(singles):
            assert np.array_equal(first[i], img1), i
        b.reload()
        b.run()
        for i in range(len(probs)):
            assert np.array_equal(b.image(i), first[i]), i


def test_batch_rejects_mixed_modes():
    probs = _problems()
    W, g, _ = probs[3]
    mixed = [probs[0][2], Problem(dataclasses.replace(g, amp=not g.amp), W.data,
                                  W.vrms_cube())]
    with Migrator(0) as m:
        with pytest.raises(Exception):
            Batch(m, mixed)
