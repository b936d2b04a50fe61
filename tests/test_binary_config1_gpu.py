"""The poststackmig binary against the reference binary on the full config-1 run.

Config 1 (101x101 traces x 501 samples at 2 ms, 25 m bins, one point diffractor plus noise,
V = 2000 m/s, 30 deg, amp on, padding 30 each side) is written once as a SEG-Y file with a
config.txt; the same files go through poststackmig3d_b200/bin/poststackmig and through the
reference's own binary compiled from its sources (oracle/_ref/poststackmig_serial, the
serial build, whose padded crosslines are exact zeros; src/main.cpp:66-442).  The output
files must agree byte for byte in every header (text, binary, all 161x161 trace headers) and
within the FP32 parity bar in the samples."""
import os

import numpy as np
import pytest

import oracle as O
from poststackmig3d_b200 import host as H
from poststackmig3d_b200 import synth as S

from helpers import MAX_REL_TOL, REL_RMS_TOL, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(O.ref_binary("serial")),
                    reason="the reference binary was not built (make -C oracle ref REF=...)")
def test_config1_binary_against_reference_binary(tmp_path):
    W = S.workload_config1()
    ours = S.write_run(str(tmp_path), W, output="ours.sgy")
    r = H.run_binary(ours, timeout=600)
    assert r.returncode == 0, r.stderr
    ref_cfg = S.write_run(str(tmp_path), W, output="ref.sgy", n_threads=1)
    rr = O.run_ref_binary(ref_cfg, "serial", timeout=1200)
    assert rr.returncode == 0, rr.stderr
    got = S.read_segy_raw(str(tmp_path / "ours.sgy"))
    ref = S.read_segy_raw(str(tmp_path / "ref.sgy"))
    assert got[0] == ref[0]  # text header
    assert got[1] == ref[1]  # binary header (ns and format rewritten)
    assert got[2].shape == (161 * 161, 240)
    assert np.array_equal(got[2], ref[2])  # every trace header, padded traces included
    a = S.decode_samples(got[3], 5).reshape(161, 161, 501)
    b = S.decode_samples(ref[3], 5).reshape(161, 161, 501)
    rms, mx = rel_err(a, b)
    assert rms <= REL_RMS_TOL and mx <= MAX_REL_TOL, (rms, mx)
    # padded crosslines are zero in both; the migrated diffractor focuses at its apex
    assert not a[:, :30].any() and not a[:, -30:].any()
    assert np.unravel_index(np.abs(a).argmax(), a.shape) == (80, 80, 250)
