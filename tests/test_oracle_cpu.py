"""The oracle (CPU restatement) pinned against the reference's own outputs.

Every golden case is the reference binary run on a seeded SEG-Y (tests/golden/make_golden.py).
The oracle, fed the same cube and the Vrms the host builds from the same velocity file,
must reproduce the reference's image to FP32 summation-order noise (the reference's
-ffast-math build reorders its sums, so bit equality is not expected) with every
aperture/range mask decision identical."""
import json
import os

import numpy as np
import pytest

import oracle as O
from poststackmig3d_b200 import host as H
from poststackmig3d_b200 import plan_geometry
from poststackmig3d_b200 import synth as S

from helpers import rel_err

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["diffractor_pad", "ibm_segy_vel", "table_vel_noamp", "irregular_idw",
         "fmt3_single_xl"]


def _case(tmp_path, name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    inp = tmp_path / "in.sgy"
    inp.write_bytes(z["input"].tobytes())
    cfg = dict(meta["config"])
    if meta["velocity_file"]:
        vp = tmp_path / meta["velocity_file"]
        vp.write_bytes(z["velocity"].tobytes())
        cfg["velocity"] = str(vp)
    return z, str(inp), cfg


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_outputs(tmp_path, name):
    z, inp, cfg = _case(tmp_path, name)
    il, xl, cube, info = H.read_segy(inp)
    n_t = info["num_samples"]
    vr = H.velocity_cube(cfg["velocity"], il, xl, n_t, info["dt_seconds"])
    lines = [f"input_data={inp}", f"output_data={tmp_path / 'o.sgy'}"]
    lines += [f"{k}={str(v).lower() if isinstance(v, bool) else v}" for k, v in cfg.items()]
    (tmp_path / "c.txt").write_text("\n".join(lines) + "\n")
    plan = H.plan_config(str(tmp_path / "c.txt"))
    g = plan_geometry(len(il), len(xl), n_t, info["dt_seconds"], float(cfg["inline_step"]),
                      float(cfg["crossline_step"]), float(cfg["angle_aperture"]),
                      plan["max_v"], int(cfg["inline_padding"]),
                      int(cfg["crossline_padding"]), bool(cfg["amp_correction"]), il, xl)
    assert g.m_il == plan["m_il"] and (g.n_oi, g.n_ox) == (plan["n_oi"], plan["n_ox"])
    img, img64, _ = O.migrate_volume(cube, vr, g.out_center, g.n_ox, g.pad_il, g.pad_xl,
                                     g.m_il, np.float32(g.dt_seconds), g.t0(),
                                     np.float32(g.tan2), g.d_il, g.d_xl, g.amp)
    _, _, _, words = S.read_segy_raw_bytes(z["output"].tobytes())
    fmt = int.from_bytes(z["output"].tobytes()[3224:3226], "big")
    ref = S.decode_samples(words, fmt).reshape(img.shape)
    if fmt == 1:  # the output went through IBM encoding: compare on the same grid
        img = H.ibm_to_ieee(H.ieee_to_ibm(img)).reshape(img.shape)
    rms, mx = rel_err(img, ref)
    if name in ("table_vel_noamp", "irregular_idw"):
        # Vrms from inverse-distance blends differs from the reference's -ffast-math build
        # in the last bit or two, which can move a single term across the aperture edge
        assert rms <= 1e-5 and mx <= 1e-4, (rms, mx)
    else:
        assert rms <= 1e-6 and mx <= 1e-6, (rms, mx)
    # zero samples (masked or invalid) agree exactly: no mask decision differs
    assert np.array_equal(img == 0, ref == 0)


def test_oracle_counts_config1():
    """Config 1 term count: the reference masks applied to real traces (an independent
    replica of the masks counted 2,855,016,288 terms with the zero padding traces too)."""
    W = S.workload_config1()
    t0 = O.t0_times(501, 0.002)
    tan2 = O.tan2_theta(30.0)
    rows = O.count_rows(W.vrms_cube(), O.output_centers(101, 30), 0, 161, 161, 30, 30, 24,
                        np.float32(0.002), t0, tan2, 25.0, 25.0)
    assert int(rows.sum()) == 2672050496  # real traces (2,855,016,288 with zero padding)


def test_oracle_fp64_mode_is_close_to_fp32():
    W = S.random_workload(4, 8, 9, 120, vel_kind="lateral", pad_xl=2)
    g = plan_geometry(8, 9, 120, W.dt, W.d_il, W.d_xl, W.angle, 2500.0, 0, 2, True)
    a, _, c1 = O.migrate_volume(W.data, W.vrms_cube(), g.out_center, g.n_ox, 0, 2, g.m_il,
                                np.float32(W.dt), g.t0(), np.float32(g.tan2), g.d_il, g.d_xl)
    _, b, c2 = O.migrate_volume(W.data, W.vrms_cube(), g.out_center, g.n_ox, 0, 2, g.m_il,
                                np.float32(W.dt), g.t0(), np.float32(g.tan2), g.d_il, g.d_xl,
                                flags=O.CONTRACT | O.F64, want64=True)
    assert np.array_equal(c1, c2)
    assert rel_err(a, b)[0] < 1e-5


def test_adjoint_oracle_dot_product():
    """<L m, d> = <m, L^T d> for the oracle's FP64 operator pair."""
    W = S.random_workload(6, 7, 8, 80, vel_kind="linear")
    g = plan_geometry(7, 8, 80, W.dt, W.d_il, W.d_xl, W.angle, 2500.0, 0, 0, True)
    rng = np.random.default_rng(1)
    d = rng.standard_normal((7, 8, 80)).astype(np.float32)
    m = rng.standard_normal((g.n_oi, g.n_ox, 80))
    _, Ld, _ = O.migrate_volume(d, W.vrms_cube(), g.out_center, g.n_ox, 0, 0, g.m_il,
                                np.float32(W.dt), g.t0(), np.float32(g.tan2), g.d_il, g.d_xl,
                                flags=O.CONTRACT | O.F64, want64=True)
    Ltm = O.adjoint_volume(m, W.vrms_cube(), 7, 8, g.out_center, 0, 0, g.m_il,
                           np.float32(W.dt), g.t0(), np.float32(g.tan2), g.d_il, g.d_xl,
                           flags=O.CONTRACT | O.F64)
    lhs = float(np.sum(Ld * m))
    rhs = float(np.sum(d.astype(np.float64) * Ltm))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), 1.0)


@pytest.mark.skipif(not O.ref_available(), reason="the reference was not built (oracle/_ref)")
@pytest.mark.parametrize("pad", [0, 3])
def test_reference_rows_threaded_equal_whole_inline_calls(pad):
    """The CPU baseline's threaded form of the reference kernel (blocks of output crosslines
    on host threads, each through the reference's serial build) gives the rows of the
    whole-inline calls of the same build bit for bit."""
    W = S.random_workload(61, 14, 23, 120, vel_kind="lateral", pad_il=pad, pad_xl=pad)
    vr = W.vrms_cube()
    g = plan_geometry(14, 23, 120, W.dt, W.d_il, W.d_xl, W.angle, float(vr.max()), pad, pad,
                      True)
    rows = [0, g.n_oi // 2, g.n_oi - 1]
    args = (W.data, vr, g.out_center, rows, g.n_ox, g.pad_il, g.pad_xl, g.m_il, g.dt_seconds,
            g.t0(), g.tan2, g.d_il, g.d_xl, True)
    whole, _ = O.reference_rows(*args, kind="serial")
    threaded, secs = O.reference_rows_threaded(*args, threads=4, xl_block=5)
    assert secs >= 0.0
    assert np.array_equal(threaded, whole)
