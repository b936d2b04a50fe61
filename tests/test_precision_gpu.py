"""16-bit trace storage (bf16 / fp16 with a per-trace fp32 scale) and compensated summation.

Every image is measured against the FP64 oracle of the same operator: for 16-bit storage the
oracle is fed the dequantised samples (the values the storage represents), so the distance is
the kernel's fp32 arithmetic alone; the distance to the FP64 image of the original fp32 samples
(quantisation included) is bounded by the storage's unit roundoff."""
import dataclasses

import numpy as np
import pytest

import oracle as O
from poststackmig3d_b200 import Migrator
from poststackmig3d_b200 import synth as S

from helpers import (MAX_REL_TOL, REL_RMS_TOL, dequantized, fp32_floor_ok, geometry_for,
                     oracle_forward, rel_err)

pytestmark = pytest.mark.gpu

# Arithmetic bar of 16-bit storage, against the oracle fed the dequantised samples: the FP32
# parity bar against its FP32 restatement, and at most 3x that restatement's own distance to
# the FP64 oracle (fp32_floor_ok).
# quantisation bar against the FP64 image of the fp32 samples: unit roundoff of the storage
QUANT_RMS_TOL = {"bf16": 2.0 ** -8, "f16": 2.0 ** -11}

CASES = [
    dict(seed=21, n_il=14, n_xl=12, n_t=300, vel_kind="lateral", pad_il=2, pad_xl=3),
    dict(seed=22, n_il=9, n_xl=15, n_t=200, vel_kind="linear", amp=False, angle=50.0),
    dict(seed=23, n_il=6, n_xl=5, n_t=70, vel_kind="const", pad_xl=1),
]


def _workload(case):
    c = dict(case)
    return S.random_workload(c.pop("seed"), c.pop("n_il"), c.pop("n_xl"), c.pop("n_t"), **c)


def _forward(W, g):
    with Migrator(0) as m:
        m.set_geometry(g)
        m.set_traces(W.data)
        m.set_vrms(W.vrms_cube())
        return m.forward()


@pytest.mark.parametrize("precision", ["bf16", "f16"])
@pytest.mark.parametrize("compensated", [False, True])
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"seed{c['seed']}")
def test_16bit_storage_against_fp64_oracle(case, precision, compensated):
    W = _workload(case)
    g = dataclasses.replace(geometry_for(W), precision=precision, compensated=compensated)
    img = _forward(W, g)
    Wq = dataclasses.replace(W, data=dequantized(W.data, precision))
    ref32q, _, _ = oracle_forward(Wq, g)
    _, ref64q, _ = oracle_forward(Wq, g, O.CONTRACT | O.F64, want64=True)
    rms, mx = rel_err(img, ref32q)
    assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (rms, mx)
    ok, errs = fp32_floor_ok(img, ref32q, ref64q)
    assert ok, errs
    _, ref64, _ = oracle_forward(W, g, O.CONTRACT | O.F64, want64=True)
    rms_q, _ = rel_err(img, ref64)
    assert rms_q <= QUANT_RMS_TOL[precision], rms_q


def test_16bit_storage_is_deterministic_and_scale_invariant():
    """Scaling a trace by a power of two scales its stored values exactly, so the image is
    the same up to that factor; two uploads give the same bits."""
    W = _workload(CASES[0])
    g = dataclasses.replace(geometry_for(W), precision="bf16")
    a = _forward(W, g)
    assert np.array_equal(a, _forward(W, g))
    W4 = dataclasses.replace(W, data=(W.data * np.float32(4.0)).astype(np.float32))
    b = _forward(W4, g)
    assert np.array_equal(b, a * np.float32(4.0))


def test_compensated_summation_removes_accumulation_error():
    """Constant traces (0.1 in fp32) with the amplitude weight off: every term is exactly
    0.1f whatever its sample position, so the distance to the FP64 oracle is the fp32
    accumulation error alone.  Over a long aperture (60 degrees, 600 samples) the compensated
    sum must remove most of it."""
    W = S.random_workload(24, 40, 40, 600, vel_kind="linear", angle=60.0, dt=0.002, amp=False)
    W = dataclasses.replace(W, data=np.full_like(W.data, np.float32(0.1)))
    g = geometry_for(W)
    plain = _forward(W, g)
    comp = _forward(W, dataclasses.replace(g, compensated=True))
    _, ref64, _ = oracle_forward(W, g, O.CONTRACT | O.F64, want64=True)
    e_plain = rel_err(plain, ref64)[0]
    e_comp = rel_err(comp, ref64)[0]
    assert e_comp <= 0.1 * e_plain and e_comp <= 1e-6, (e_comp, e_plain)


def test_compensated_summation_on_random_traces():
    """Random traces with the amplitude weight: the fp32 error is dominated by the rounding
    of each term's sample position t / dt, which no summation order changes; the
    compensated image keeps the FP32 parity bars and is no further from FP64 than the
    plain sum."""
    W = S.random_workload(25, 30, 30, 500, vel_kind="lateral", angle=60.0, dt=0.002)
    g = geometry_for(W)
    plain = _forward(W, g)
    comp = _forward(W, dataclasses.replace(g, compensated=True))
    ref32, ref64, _ = oracle_forward(W, g, O.CONTRACT | O.F64, want64=True)
    ref32, _, _ = oracle_forward(W, g)
    rms, mx = rel_err(comp, ref32)
    assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (rms, mx)
    e_plain = rel_err(plain, ref64)[0]
    e_comp = rel_err(comp, ref64)[0]
    assert e_comp <= 1.05 * e_plain, (e_comp, e_plain)


def test_precision_argument_checked():
    W = _workload(CASES[2])
    g = geometry_for(W)
    gc = g.to_c()
    gc.precision = 7
    from poststackmig3d_b200 import _lib
    with Migrator(0) as m:
        rc = _lib.cuda().psm_set_geometry(m._ctx, gc, None)
        assert rc == -1
