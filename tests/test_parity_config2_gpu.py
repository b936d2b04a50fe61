"""Parity of the production workloads against the reference's own kernel and the FP64 oracle.

The config-2 recipe (Vrms 1500 -> 3500 m/s with a 5% lateral bump, 60 diffractors + 5 dipping
planes, 30 Hz Ricker, 5% noise, 45 deg, amp on) on 201x201 traces x 1001 samples, migrated
whole on the GPU; two central output inlines are compared with
  * the reference's kirchhoffKernel3DWithPadding compiled from its sources (oracle/_ref, the
    OpenMP build, src/migration_kernel.cpp:17-383) on the buffers its driver prepares
    (src/main.cpp:291-361): FP32 parity bar, 1e-4 relative RMS and 1e-4 of the peak;
  * the FP64 oracle of the same operator: no further from it than 3x the reference's own
    FP32 arithmetic.
16-bit storage is held to the same FP32 bars against the FP64 oracle fed the dequantised
samples, and its quantisation error against the FP64 image of the original samples to the
storage's unit roundoff (2^-8 for BF16, 2^-11 for FP16; BF16 measured 1.4e-3 relative RMS
on this crop).  Velocity-scan panels of the batched form (config 4's cube, one persistent
launch) are checked the same way against the reference at their constant velocity."""
import dataclasses
import os

import numpy as np
import pytest

import oracle as O
from poststackmig3d_b200 import Batch, Migrator, Problem, plan_geometry
from poststackmig3d_b200 import synth as S

from helpers import FP32_FLOOR_FACTOR, MAX_REL_TOL, REL_RMS_TOL, geometry_for, rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")]

THREADS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def config2_201():
    W = S.workload_config2(n=201)
    return W, geometry_for(W)


def _oracle_rows(W, g, rows, data=None):
    sub = np.ascontiguousarray(g.out_center[rows])
    r32, r64, _ = O.migrate_volume(W.data if data is None else data, W.vrms_cube(), sub,
                                   g.n_ox, g.pad_il, g.pad_xl, g.m_il,
                                   np.float32(g.dt_seconds), g.t0(), np.float32(g.tan2),
                                   g.d_il, g.d_xl, g.amp, O.CONTRACT | O.F64, THREADS, True)
    return r64


def _reference_rows(W, g, rows, velocity=None):
    vr = W.vrms_cube() if velocity is None else np.full(W.data.shape, np.float32(velocity),
                                                        dtype=np.float32)
    out, _ = O.reference_rows(W.data, vr, g.out_center, rows, g.n_ox, g.pad_il, g.pad_xl,
                              g.m_il, g.dt_seconds, g.t0(), g.tan2, g.d_il, g.d_xl, g.amp)
    return out


def test_config2_crop_fp32_against_reference_and_fp64(config2_201):
    W, g = config2_201
    rows = [100, 101]
    with Migrator(0) as m:
        m.set_geometry(g)
        m.set_traces(W.data)
        m.set_vrms(W.vrms_cube())
        img = m.forward()
    ref = _reference_rows(W, g, rows)
    r64 = _oracle_rows(W, g, rows)
    rms, mx = rel_err(img[rows], ref)
    assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (rms, mx)
    e_gpu = rel_err(img[rows], r64)[0]
    e_ref = rel_err(ref, r64)[0]
    assert e_gpu <= FP32_FLOOR_FACTOR * e_ref + 1e-7, (e_gpu, e_ref)


@pytest.mark.parametrize("precision", ["bf16", "f16"])
def test_config2_crop_16bit_storage_against_fp64(config2_201, precision):
    W, g0 = config2_201
    g = dataclasses.replace(g0, precision=precision)
    rows = [100, 101]
    with Migrator(0) as m:
        m.set_geometry(g)
        m.set_traces(W.data)
        m.set_vrms(W.vrms_cube())
        img = m.forward()
    deq = O.dequantized(W.data, precision)
    r64q = _oracle_rows(W, g0, rows, deq)  # the same operator on the samples held
    rms, mx = rel_err(img[rows], r64q)
    assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (rms, mx)
    r64 = _oracle_rows(W, g0, rows)  # the original fp32 samples: quantisation error
    unit_roundoff = {"bf16": 2.0 ** -8, "f16": 2.0 ** -11}[precision]
    assert rel_err(img[rows], r64)[0] <= unit_roundoff


def test_velocity_panels_of_one_persistent_launch_against_reference():
    panels, _ = S.workload_config4(n_panels=32, n_sub=0)
    chosen = [panels[0], panels[31]]  # 1800 and 3350 m/s
    cube = np.ascontiguousarray(chosen[0].data)
    probs = []
    for W in chosen:
        g = plan_geometry(*cube.shape, W.dt, W.d_il, W.d_xl, W.angle, W.velocity, 0, 0,
                          W.amp)
        probs.append(Problem(g, cube, velocity=W.velocity))
    rows = [100]
    with Migrator(0) as m:
        with Batch(m, probs) as b:
            b.set_mode(Batch.PERSISTENT)
            b.run()
            imgs = [b.image(i) for i in range(len(probs))]
    for W, p, img in zip(chosen, probs, imgs):
        ref = _reference_rows(W, p.geom, rows, velocity=W.velocity)
        rms, mx = rel_err(img[rows], ref)
        assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (W.velocity, rms, mx)
