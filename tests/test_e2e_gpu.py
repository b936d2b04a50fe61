"""The poststackmig binary (C++ host + GPU) against the reference binary's own outputs.

For every golden case the same SEG-Y input, velocity file and config go through
poststackmig3d_b200/bin/poststackmig; the output file must have the reference's text and
binary headers and trace headers byte for byte, and samples within the FP32 parity bar."""
import json
import os

import numpy as np
import pytest

from poststackmig3d_b200 import host as H
from poststackmig3d_b200 import synth as S

from helpers import MAX_REL_TOL, REL_RMS_TOL, rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["diffractor_pad", "ibm_segy_vel", "table_vel_noamp", "irregular_idw",
         "fmt3_single_xl"]


def _write_case(tmp_path, name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    inp = tmp_path / "in.sgy"
    inp.write_bytes(z["input"].tobytes())
    cfg = dict(meta["config"])
    if meta["velocity_file"]:
        vp = tmp_path / meta["velocity_file"]
        vp.write_bytes(z["velocity"].tobytes())
        cfg["velocity"] = str(vp)
    out = tmp_path / "out.sgy"
    lines = [f"input_data={inp}", f"output_data={out}"]
    lines += [f"{k}={str(v).lower() if isinstance(v, bool) else v}" for k, v in cfg.items()]
    cp = tmp_path / "config.txt"
    cp.write_text("\n".join(lines) + "\n")
    return z, cp, out


@pytest.mark.parametrize("name", CASES)
def test_binary_matches_reference_output(tmp_path, name):
    z, cp, out = _write_case(tmp_path, name)
    r = H.run_binary(str(cp), timeout=300)
    assert r.returncode == 0, r.stderr
    got = S.read_segy_raw(str(out))
    ref = S.read_segy_raw_bytes(z["output"].tobytes())
    assert got[0] == ref[0]  # text header
    assert got[1] == ref[1]  # binary header (ns and format rewritten)
    assert np.array_equal(got[2], ref[2])  # every trace header
    fmt = int.from_bytes(ref[1][24:26], "big")
    a = S.decode_samples(got[3], fmt)
    b = S.decode_samples(ref[3], fmt)
    rms, mx = rel_err(a, b)
    assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (rms, mx)
    if fmt == 1:  # IBM output: decoding the words round-trips the same values
        assert np.array_equal(H.ieee_to_ibm(a), got[3].astype(np.uint32).ravel())


def test_binary_reports_errors_like_the_reference(tmp_path):
    cp = tmp_path / "c.txt"
    cp.write_text("input_data=nope.sgy\noutput_data=o.sgy\ninline_step=1\n"
                  "crossline_step=1\nvelocity=2000\n")
    r = H.run_binary(str(cp), timeout=60)
    assert r.returncode == 1 and "Error: Cannot open SEGY file: nope.sgy" in r.stderr
    r = H.run_binary(str(tmp_path / "missing.txt"), timeout=60)
    assert r.returncode == 1 and "Error: Config file not found" in r.stderr


def test_compat_omp_pad_matches_the_reference_openmp_binary(tmp_path):
    """compat_omp_pad=true reproduces the reference's OpenMP build, trailing padded
    crosslines included (there its per-sample caches keep the last real crossline's values,
    migration_kernel.cpp:60-72); without it those crosslines are zero, as in the serial
    build.  Every other trace is the same in both builds."""
    import oracle as O
    if not os.path.exists(O.ref_binary("omp")):
        pytest.skip("the reference binary was not built")
    W = S.random_workload(61, 11, 9, 160, vel_kind="lateral", pad_il=2, pad_xl=3, angle=40.0,
                          dt=0.004)
    ref_cfg = S.write_run(str(tmp_path), W, output="ref.sgy", n_threads=4)
    rr = O.run_ref_binary(ref_cfg, "omp", timeout=600)
    assert rr.returncode == 0, rr.stderr
    ref = S.read_segy_raw(str(tmp_path / "ref.sgy"))
    n_ox = 9 + 2 * 3
    b = S.decode_samples(ref[3], 5).reshape(-1, n_ox, 160)
    assert np.abs(b[:, -3:]).max() > 0  # the quirk shows in this case
    for compat in (True, False):
        cfg = S.write_run(str(tmp_path), W, output=f"ours{int(compat)}.sgy",
                          compat_omp_pad=compat)
        r = H.run_binary(cfg, timeout=300)
        assert r.returncode == 0, r.stderr
        got = S.read_segy_raw(str(tmp_path / f"ours{int(compat)}.sgy"))
        assert got[0] == ref[0] and got[1] == ref[1] and np.array_equal(got[2], ref[2])
        a = S.decode_samples(got[3], 5).reshape(-1, n_ox, 160)
        if compat:
            rms, mx = rel_err(a, b)
            assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (rms, mx)
        else:
            assert not a[:, -3:].any()
            rms, mx = rel_err(a[:, :-3], b[:, :-3])
            assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (rms, mx)
