"""GPU forward operator vs the oracle (and the reference's golden outputs).

Parity bar: relative RMS <= 1e-5 and max error <= 1e-4 of the image peak against the
oracle's FP32 restatement, whose own distance to the reference build is <= 2e-7 relative
RMS (tests/test_oracle.py).  Term counts must agree with the oracle's masks."""
import numpy as np
import pytest

import oracle as O
from poststackmig3d_b200 import synth as S
from poststackmig3d_b200 import MigrationKernel, Migrator, plan_geometry

from helpers import (MAX_REL_TOL, REL_RMS_TOL, fp32_floor_ok, geometry_for, gpu_forward,
                     oracle_forward, rel_err)

pytestmark = pytest.mark.gpu


CASES = [
    dict(seed=1, n_il=9, n_xl=11, n_t=64, vel_kind="const"),
    dict(seed=2, n_il=12, n_xl=10, n_t=96, vel_kind="linear", angle=45.0),
    dict(seed=3, n_il=10, n_xl=13, n_t=300, vel_kind="lateral", pad_il=2, pad_xl=3),
    dict(seed=4, n_il=7, n_xl=7, n_t=129, vel_kind="linear", amp=False, pad_xl=2),
    dict(seed=5, n_il=16, n_xl=21, n_t=520, vel_kind="lateral", angle=60.0, dt=0.002),
    dict(seed=6, n_il=5, n_xl=1, n_t=40, vel_kind="const", pad_il=1),
    dict(seed=7, n_il=1, n_xl=17, n_t=77, vel_kind="linear", pad_xl=1),
    dict(seed=8, n_il=20, n_xl=9, n_t=33, vel_kind="lateral", angle=10.0),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"seed{c['seed']}")
def test_forward_matches_oracle(case):
    c = dict(case)
    W = S.random_workload(c.pop("seed"), c.pop("n_il"), c.pop("n_xl"), c.pop("n_t"), **c)
    img, n_gpu, g = gpu_forward(W)
    ref, _, counts = oracle_forward(W, g)
    rms, mx = rel_err(img, ref)
    assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (rms, mx)
    _, ref64, _ = oracle_forward(W, g, O.CONTRACT | O.F64, want64=True)
    ok, errs = fp32_floor_ok(img, ref, ref64)
    assert ok, errs
    # real-trace terms: the kernel's masks are the reference's FP32 arithmetic exactly
    assert n_gpu == counts[1], (n_gpu, counts)


def test_config1_full_size():
    """Config 1 (101x101x501, 30 deg, pad 30/30, V=2000) against the oracle."""
    W = S.workload_config1()
    img, n_gpu, g = gpu_forward(W)
    assert img.shape == (161, 161, 501)
    ref, _, counts = oracle_forward(W, g)
    rms, mx = rel_err(img, ref)
    assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (rms, mx)
    _, ref64, _ = oracle_forward(W, g, O.CONTRACT | O.F64, want64=True)
    ok, errs = fp32_floor_ok(img, ref, ref64)
    assert ok, errs
    assert counts[0] == 2855016288  # all accumulated terms, zero padding traces included
    assert n_gpu == counts[1] == 2672050496  # terms on real input traces
    # padded output inlines repeat the edge inlines; padded crosslines are zero
    assert np.array_equal(img[0], img[30]) and np.array_equal(img[160], img[130])
    assert not img[:, :30].any() and not img[:, 131:].any()
    # the diffractor focuses at its apex (t0 = 0.5 s at the centre trace)
    assert np.unravel_index(np.argmax(img), img.shape) == (80, 80, 250)


def test_inline_dropin_matches_oracle():
    """psm_kirchhoff_inline (the kirchhoffKernel3DWithPadding drop-in) on a reference-style
    buffer, including an off-centre current_xl_start and out-of-buffer output crosslines."""
    rng = np.random.default_rng(11)
    n_buf_il, n_buf_xl, n_t = 9, 14, 150
    buf = rng.standard_normal((n_buf_il, n_buf_xl, n_t)).astype(np.float32)
    vel = (1800 + 400 * rng.random((n_buf_xl, n_t))).astype(np.float32)
    vel[:2] = 0.0  # padded crosslines carry v = 0
    il_pos = np.arange(20, 20 + n_buf_il, dtype=np.int32)
    t0 = O.t0_times(n_t, 0.004)
    tan2 = O.tan2_theta(40.0)
    for cur_il, xs, n_out in [(4, 0, 14), (0, -3, 20), (8, 2, 12), (-1, 0, 14)]:
        out = np.full((n_out, n_t), np.nan, dtype=np.float32)
        MigrationKernel.kirchhoff_kernel_3d_with_padding(
            buf, n_buf_il, n_buf_xl, n_t, vel, out, il_pos, None, cur_il, xs, 0.004, t0, tan2,
            25.0, 20.0, True)
        ref, _, _ = O.kirchhoff_inline(buf, vel, n_out, il_pos, cur_il, xs, 0.004, t0, tan2,
                                       25.0, 20.0, True)
        rms, mx = rel_err(out, ref)
        assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (cur_il, xs, rms, mx)


PAIRED = {11, 12, 13}  # variants that add mirrored traces' samples before the weight


@pytest.mark.parametrize("seed,pad_il,angle", [(31, 0, 50.0), (32, 3, 35.0)])
def test_variants_are_bit_identical_and_autotune_picks_one(seed, pad_il, angle):
    """Packed (f32x2) and scalar arithmetic perform the same IEEE operations per term, and
    masked terms add exact zeros, so every variant gives the same image bit for bit.  The
    paired variants sum the same terms in another order: they meet the FP32 parity bars
    against the oracle instead."""
    W = S.random_workload(seed, 14, 17, 400, vel_kind="lateral", angle=angle, pad_xl=2,
                          pad_il=pad_il)
    g = geometry_for(W)
    with Migrator(0) as m:
        m.set_geometry(g)
        m.set_traces(W.data)
        m.set_vrms(W.vrms_cube())
        imgs = {}
        for v in Migrator.VARIANTS:
            m.set_variant(v)
            assert m.variant() == v
            imgs[v] = m.forward()
        best, ms = m.autotune()
        assert best in Migrator.VARIANTS and all(t > 0 for t in ms.values())
        assert m.variant() == best
        after = m.forward()
    ref = imgs[1]
    for v, img in imgs.items():
        if v not in PAIRED:
            assert np.array_equal(img, ref), v
    assert np.array_equal(after, imgs[best])
    ref32, _, _ = oracle_forward(W, g)
    _, ref64, _ = oracle_forward(W, g, O.CONTRACT | O.F64, want64=True)
    for v in PAIRED:
        rms, mx = rel_err(imgs[v], ref32)
        assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (v, rms, mx)
        ok, errs = fp32_floor_ok(imgs[v], ref32, ref64)
        assert ok, (v, errs)
        assert np.array_equal(imgs[v] == 0, ref == 0), v  # the same terms: zero where it is


def test_forward_is_linear_and_repeatable():
    W = S.random_workload(21, 10, 12, 200, vel_kind="lateral", angle=50.0)
    g = geometry_for(W)
    with Migrator(0) as m:
        m.set_geometry(g)
        m.set_vrms(W.vrms_cube())
        m.set_traces(W.data)
        a = m.forward()
        a2 = m.forward()
        m.set_traces(2.0 * W.data)
        b = m.forward()
    assert np.array_equal(a, a2)  # deterministic
    assert np.array_equal(2.0 * a, b)  # power-of-two scaling is exact through every op


def test_golden_constant_velocity_cases():
    """The reference's own outputs (tests/golden, made by running its binary) for the
    constant-velocity cases, recomputed on the GPU from the same SEG-Y input."""
    import io
    import json
    import os
    here = os.path.join(os.path.dirname(__file__), "golden")
    for name in ["diffractor_pad", "fmt3_single_xl"]:
        z = np.load(os.path.join(here, name + ".npz"))
        meta = json.loads(str(z["meta"]))
        cfg = meta["config"]
        tmp = io.BytesIO(z["input"].tobytes())
        raw = np.frombuffer(tmp.getvalue(), dtype=np.uint8)
        bh = raw[3200:3600].tobytes()
        dt_us = int.from_bytes(bh[16:18], "big")
        n_t = int.from_bytes(bh[20:22], "big")
        n_tr = (len(raw) - 3600) // (240 + 4 * n_t)
        body = raw[3600:3600 + n_tr * (240 + 4 * n_t)].reshape(n_tr, -1)
        ils = S.header_i32(body[:, :240], 188)
        xls = S.header_i32(body[:, :240], 192)
        samples = S.decode_samples(body[:, 240:].copy().view(">u4").reshape(n_tr, n_t), 5)
        il_l = np.unique(ils)
        xl_l = np.unique(xls)
        cube = np.zeros((len(il_l), len(xl_l), n_t), dtype=np.float32)
        cube[np.searchsorted(il_l, ils), np.searchsorted(xl_l, xls)] = samples
        v = float(cfg["velocity"])
        g = plan_geometry(len(il_l), len(xl_l), n_t, dt_us * 1e-6, float(cfg["inline_step"]),
                          float(cfg["crossline_step"]), float(cfg["angle_aperture"]), v,
                          int(cfg["inline_padding"]), int(cfg["crossline_padding"]),
                          bool(cfg["amp_correction"]), il_l, xl_l)
        with Migrator(0) as m:
            m.set_geometry(g)
            m.set_traces(cube)
            m.set_vrms(np.full(cube.shape, np.float32(v), dtype=np.float32))
            img = m.forward()
        _, _, oh, ow = S.read_segy_raw_bytes(z["output"].tobytes())
        ref = S.decode_samples(ow, 5).reshape(img.shape)
        rms, mx = rel_err(img, ref)
        assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (name, rms, mx)


@pytest.mark.parametrize("seed,pad_il,pad_xl,n_il,precision,compensated",
                         [(41, 3, 2, 30, "f32", False), (42, 0, 0, 7, "f32", False),
                          (43, 5, 1, 3, "f32", False), (44, 2, 1, 20, "bf16", False),
                          (45, 1, 0, 18, "f32", True)])
def test_forward_host_pipeline_equals_resident_forward(seed, pad_il, pad_xl, n_il, precision,
                                                       compensated):
    """psm_forward_host (inline blocks uploaded on a copy stream, waves of output inlines,
    rows streamed back) gives the resident forward's image bit for bit, repeated padded rows
    included, twice in a row; with 16-bit storage and with compensated summation too."""
    import dataclasses
    W = S.random_workload(seed, n_il, 11, 230, vel_kind="lateral", pad_il=pad_il,
                          pad_xl=pad_xl, d_il=60.0)
    g = dataclasses.replace(geometry_for(W), precision=precision, compensated=compensated)
    ref, _, _ = gpu_forward(W, g)
    with Migrator(0) as m:
        m.set_geometry(g)
        for _ in range(2):
            img = m.forward_host(W.data, W.vrms_cube())
            assert np.array_equal(img, ref)
        assert np.array_equal(m.forward(), ref)  # the traces and Vrms stay resident
