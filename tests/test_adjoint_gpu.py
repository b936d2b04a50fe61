"""Adjoint (demigration / spray) operator and least-squares migration on the GPU.

M: data -> image is the forward migration; M^T: image -> data its transpose (psm_adjoint).
The pair must pass the dot-product test <M d, m> = <d, M^T m> to 1e-5 (FP64 inner products),
M^T must match the oracle's FP64 transpose, and the gradient of J(m) = ||M^T m - d||^2,
2 M (M^T m - d), must agree with finite differences of J."""
import numpy as np
import pytest

import oracle as O
from poststackmig3d_b200 import Migrator
from poststackmig3d_b200 import synth as S

from helpers import geometry_for, rel_err

pytestmark = pytest.mark.gpu

CASES = [
    dict(seed=51, n_il=10, n_xl=12, n_t=200, vel_kind="lateral", angle=45.0),
    dict(seed=52, n_il=8, n_xl=9, n_t=96, vel_kind="const", pad_il=2, pad_xl=2),
    dict(seed=53, n_il=9, n_xl=7, n_t=300, vel_kind="linear", amp=False, pad_xl=1),
]


def _setup(case):
    c = dict(case)
    W = S.random_workload(c.pop("seed"), c.pop("n_il"), c.pop("n_xl"), c.pop("n_t"), **c)
    g = geometry_for(W)
    m = Migrator(0)
    m.set_geometry(g)
    m.set_vrms(W.vrms_cube())
    return W, g, m


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"seed{c['seed']}")
def test_dot_product(case):
    W, g, mig = _setup(case)
    rng = np.random.default_rng(7)
    d = rng.standard_normal(W.data.shape).astype(np.float32)
    im = rng.standard_normal((g.n_oi, g.n_ox, g.n_t)).astype(np.float32)
    mig.set_traces(d)
    Md = mig.forward()
    MTm = mig.adjoint(im)
    mig.close()
    lhs = float(np.sum(Md.astype(np.float64) * im.astype(np.float64)))
    rhs = float(np.sum(d.astype(np.float64) * MTm.astype(np.float64)))
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), abs(rhs)), (lhs, rhs)


ACCUMS = ["fixed", "f32"]


@pytest.mark.parametrize("accum", ACCUMS)
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"seed{c['seed']}")
def test_adjoint_matches_oracle(case, accum, monkeypatch):
    """Both accumulations of the spray (PSM_ADJ_ACCUM, read when the context is created):
    fp32 shared-memory atomics into an fp32 cube (the default) and 64-bit fixed-point windows
    into an FP64 data cube."""
    monkeypatch.setenv("PSM_ADJ_ACCUM", accum)
    W, g, mig = _setup(case)
    rng = np.random.default_rng(8)
    im = rng.standard_normal((g.n_oi, g.n_ox, g.n_t)).astype(np.float32)
    got = mig.adjoint(im)
    mig.close()
    ref = O.adjoint_volume(im.astype(np.float64), W.vrms_cube(), g.n_il, g.n_xl,
                           g.out_center, g.pad_il, g.pad_xl, g.m_il, np.float32(g.dt_seconds),
                           g.t0(), np.float32(g.tan2), g.d_il, g.d_xl, g.amp,
                           flags=O.CONTRACT)
    rms, mx = rel_err(got, ref)
    # FP32 atomic accumulation of many contributions per data sample, against FP64 sums: the
    # FP32 parity bar of the forward operator
    assert rms <= 1e-4 and mx <= 1e-4, (rms, mx)


@pytest.mark.parametrize("accum", ACCUMS)
def test_adjoint_coherent_image(accum, monkeypatch):
    """A constant image at a wide aperture (85 deg, no amplitude weight): the shares of a
    window sample all have one sign, and near the aperture's edge (ds/dt0 = cos 85 deg) one
    tile puts up to about 43 of its largest shares on one sample, where the fixed-point
    windows' tile scale leaves the least headroom.  The sums must match the FP64 oracle."""
    monkeypatch.setenv("PSM_ADJ_ACCUM", accum)
    W, g, mig = _setup(dict(seed=55, n_il=12, n_xl=14, n_t=260, vel_kind="const",
                            angle=85.0, amp=False))
    im = np.ones((g.n_oi, g.n_ox, g.n_t), dtype=np.float32)
    got = mig.adjoint(im)
    mig.close()
    ref = O.adjoint_volume(im.astype(np.float64), W.vrms_cube(), g.n_il, g.n_xl,
                           g.out_center, g.pad_il, g.pad_xl, g.m_il, np.float32(g.dt_seconds),
                           g.t0(), np.float32(g.tan2), g.d_il, g.d_xl, g.amp,
                           flags=O.CONTRACT)
    rms, mx = rel_err(got, ref)
    assert rms <= 1e-5 and mx <= 1e-4, (rms, mx)


def test_gradient_matches_finite_differences():
    W, g, mig = _setup(CASES[0])
    rng = np.random.default_rng(9)
    d = rng.standard_normal(W.data.shape).astype(np.float32)
    m0 = rng.standard_normal((g.n_oi, g.n_ox, g.n_t)).astype(np.float32)
    dm = rng.standard_normal((g.n_oi, g.n_ox, g.n_t)).astype(np.float32)

    def J(m):
        r = mig.adjoint(m).astype(np.float64) - d
        return float(np.sum(r * r))

    r0 = (mig.adjoint(m0).astype(np.float64) - d).astype(np.float32)
    mig.set_traces(r0)
    grad = 2.0 * mig.forward().astype(np.float64)  # 2 M (M^T m - d)
    eps = 1.0  # J is quadratic: central differences have no truncation error at any step
    fd = (J(m0 + eps * dm) - J(m0 - eps * dm)) / (2 * eps)
    an = float(np.sum(grad * dm))
    mig.close()
    assert abs(fd - an) <= 2e-4 * abs(an), (fd, an)


def test_lsm_cg_reduces_the_residual():
    """10 CG iterations of least-squares migration on data modelled from a sparse
    reflectivity plus noise: the data residual falls monotonically."""
    W, g, mig = _setup(dict(seed=54, n_il=12, n_xl=12, n_t=160, vel_kind="const"))
    rng = np.random.default_rng(10)
    mtrue = np.zeros((g.n_oi, g.n_ox, g.n_t), dtype=np.float32)
    mask = rng.random(mtrue.shape) < 0.02
    mtrue[mask] = rng.laplace(0.0, 1.0, mask.sum()).astype(np.float32)
    d = mig.adjoint(mtrue)
    d = d + (0.05 * np.abs(d).max() * rng.standard_normal(d.shape)).astype(np.float32)
    m, hist = mig.lsm_cg(d, 10)
    mig.close()
    assert m.shape == mtrue.shape and len(hist) == 11
    assert np.all(np.diff(hist) <= 1e-6 * hist[0])  # CGLS residuals do not increase
    assert hist[-1] < 0.9 * hist[0]


def _dot_test(n, n_t, seed, compensated):
    import dataclasses
    from poststackmig3d_b200 import plan_geometry
    g = plan_geometry(n, n, n_t, 0.002, 25.0, 25.0, 30.0, 2000.0, 0, 0, True)
    g = dataclasses.replace(g, compensated=compensated)
    vr = np.full((n, n, n_t), 2000.0, dtype=np.float32)
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, n, n_t)).astype(np.float32)
    im = rng.standard_normal((g.n_oi, g.n_ox, n_t)).astype(np.float32)
    with Migrator(0) as mig:
        mig.set_geometry(g)
        mig.set_vrms(vr)
        mig.set_traces(d)
        Md = mig.forward()
        MTm = mig.adjoint(im)
    lhs = float(np.sum(Md.astype(np.float64) * im.astype(np.float64)))
    rhs = float(np.sum(d.astype(np.float64) * MTm.astype(np.float64)))
    return abs(lhs - rhs) / max(abs(lhs), abs(rhs))


@pytest.mark.parametrize("seed", [1, 2])
def test_dot_product_at_size(seed):
    """The operator pair on 101x101 traces x 1001 samples (V 2000 m/s, 30 deg, amp on),
    about 1e10 terms, where FP32 sums of thousands of terms per sample show.  Both operators
    use the same fp32 travel times, fractions and weights, so they differ from exact
    transposes by their summation rounding only (about 4e-7 of a vector's norm); the
    compensated forward sums its stages with Kahan's compensation.  The two inner products
    of independent random vectors nearly cancel (|cos| ~ 1e-4), which magnifies that
    rounding in the relative error."""
    assert _dot_test(101, 1001, seed, compensated=True) <= 1e-5
