"""Host surface (libpsm_host.so) against the reference, on CPU.

Golden data: tests/golden/*.npz, produced by running the reference itself
(tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

from poststackmig3d_b200 import host as H
from poststackmig3d_b200 import synth as S
from poststackmig3d_b200._lib import PsmError

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


# --------------------------------------------------------------------------- IBM / IEEE


def test_ibm_ieee_match_reference_vectors():
    z = _golden("ibm_vectors")
    assert np.array_equal(H.ieee_to_ibm(z["floats"]), z["ibm"])
    assert np.array_equal(H.ibm_to_ieee(z["words"]).view(np.uint32),
                          z["decoded"].view(np.uint32))


def test_ibm_known_values():
    # IBM single: 0x41100000 = +1.0, 0xC1100000 = -1.0, 0x42640000 = 100.0,
    # 0x40800000 = 0.5, 0x3F100000 = 16^-2
    words = np.array([0x41100000, 0xC1100000, 0x42640000, 0x40800000, 0x3F100000, 0],
                     dtype=np.uint32)
    vals = np.array([1.0, -1.0, 100.0, 0.5, 1.0 / 256, 0.0], dtype=np.float32)
    assert np.array_equal(H.ibm_to_ieee(words), vals)
    assert np.array_equal(H.ieee_to_ibm(vals), words)
    # -0.0 encodes as 0; the decoder keeps the sign of 0x80000000
    assert H.ieee_to_ibm([-0.0])[0] == 0
    assert np.signbit(H.ibm_to_ieee([0x80000000])[0])
    # non-finite inputs terminate (the reference loops on inf)
    assert H.ieee_to_ibm([np.inf])[0] == 0x7FFFFFFF
    assert H.ieee_to_ibm([-np.inf])[0] == 0xFFFFFFFF
    assert H.ieee_to_ibm([np.nan])[0] == 0x40000000


def test_ibm_roundtrip_is_within_truncation():
    rng = np.random.default_rng(0)
    x = (rng.standard_normal(5000) * 10.0 ** rng.integers(-10, 10, 5000)).astype(np.float32)
    y = H.ibm_to_ieee(H.ieee_to_ibm(x))
    # 24-bit base-16 fraction keeps >= 21 significant bits
    assert np.all(np.abs(y - x) <= np.abs(x) * 2.0 ** -20)


# --------------------------------------------------------------------------- config


def _cfg(tmp_path, text):
    p = tmp_path / "config.txt"
    p.write_text(text)
    return str(p)


BASE = ("input_data=in.sgy\noutput_data=out.sgy\ninline_step=25\ncrossline_step=12.5\n"
        "velocity=2000\n")


def test_config_defaults(tmp_path):
    c = H.load_config(_cfg(tmp_path, BASE))
    assert c["input_data"] == "in.sgy" and c["output_data"] == "out.sgy"
    assert c["inline_step"] == 25.0 and c["crossline_step"] == 12.5
    assert c["inline_padding"] == 0 and c["crossline_padding"] == 0
    assert c["angle_aperture"] == 30.0 and c["amp_correction"] is True
    assert c["n_threads"] == 0 and c["velocity"] == "2000"
    assert c["precision"] == 0 and c["compensated"] is False and c["device"] == 0
    assert c["compat_omp_pad"] is False


def test_config_every_key_quotes_comments_duplicates(tmp_path):
    text = ("# comment\n\n   input_data = \"a b.sgy\"  \noutput_data='o.sgy'\n"
            "inline_step=10\ninline_step=20\ncrossline_step=5.5m\nvelocity = v.sgy\n"
            "inline_padding=3\ncrossline_padding=4\nangle_aperture=45.5\n"
            "amp_correction=OFF\nn_threads=8\nunknown_key=whatever\nprecision=bf16\n"
            "compensated=yes\ndevice=0\ncompat_omp_pad=on\n")
    c = H.load_config(_cfg(tmp_path, text))
    assert c["input_data"] == "a b.sgy" and c["output_data"] == "o.sgy"
    assert c["inline_step"] == 20.0          # last duplicate wins
    assert c["crossline_step"] == 5.5        # std::stod takes the leading number
    assert c["velocity"] == "v.sgy"
    assert (c["inline_padding"], c["crossline_padding"]) == (3, 4)
    assert c["angle_aperture"] == 45.5 and c["amp_correction"] is False
    assert c["n_threads"] == 8 and c["precision"] == 1 and c["compensated"] is True
    assert c["compat_omp_pad"] is True


@pytest.mark.parametrize("spelling,value", [("true", True), ("1", True), ("Yes", True),
                                            ("on", True), ("false", False), ("0", False),
                                            ("NO", False), ("off", False)])
def test_config_bool_spellings(tmp_path, spelling, value):
    c = H.load_config(_cfg(tmp_path, BASE + f"amp_correction={spelling}\n"))
    assert c["amp_correction"] is value


@pytest.mark.parametrize("extra,msg", [
    ("amp_correction=maybe\n", "Cannot parse boolean value"),
    ("inline_padding=x\n", "Cannot parse int value"),
    ("angle_aperture=abc\n", "Cannot parse double value"),
    ("angle_aperture=90\n", "angle_aperture must be in range (0, 90)"),
    ("angle_aperture=0\n", "angle_aperture must be in range (0, 90)"),
    ("inline_padding=-1\n", "inline_padding must be non-negative"),
    ("crossline_padding=-2\n", "crossline_padding must be non-negative"),
    ("n_threads=-1\n", "n_threads must be non-negative"),
    ("inline_step=0\n", "inline_step must be positive"),
    ("crossline_step=-5\n", "crossline_step must be positive"),
    ("this line has no equals\n", "Invalid format at line 6"),
    ("precision=fp8\n", "Cannot parse precision value"),
])
def test_config_errors(tmp_path, extra, msg):
    with pytest.raises(PsmError, match=msg.replace("(", r"\(").replace(")", r"\)")):
        H.load_config(_cfg(tmp_path, BASE + extra))


def test_config_missing_keys(tmp_path):
    with pytest.raises(PsmError, match="Missing required parameters: output_data, velocity"):
        H.load_config(_cfg(tmp_path, "input_data=a\ninline_step=1\ncrossline_step=1\n"))
    with pytest.raises(PsmError, match="Config file not found"):
        H.load_config(str(tmp_path / "nope.txt"))


def test_negative_constant_velocity_fails_at_the_provider(tmp_path):
    # validation lets it through (config_parser.cpp:201-211), the provider rejects it
    H.load_config(_cfg(tmp_path, BASE.replace("velocity=2000", "velocity=-5")))
    with pytest.raises(PsmError, match="Velocity must be positive"):
        H.velocity_point("-5", 1, 1, 0, 0.002, 10)


# --------------------------------------------------------------------------- SEG-Y


@pytest.mark.parametrize("name", ["diffractor_pad", "ibm_segy_vel", "table_vel_noamp",
                                  "irregular_idw", "fmt3_single_xl"])
def test_segy_read_matches_independent_reader(tmp_path, name):
    z = _golden(name)
    p = tmp_path / "in.sgy"
    p.write_bytes(z["input"].tobytes())
    il, xl, cube, info = H.read_segy(str(p))
    text, binary, hdrs, words = S.read_segy_raw(str(p))
    fmt = int.from_bytes(binary[24:26], "big")
    assert info["format"] == (fmt if fmt in (1, 5) else 5)
    ils = S.header_i32(hdrs, 188)
    xls = S.header_i32(hdrs, 192)
    keep = (ils != 0) & (xls != 0)
    assert np.array_equal(il, np.unique(ils[keep])) and np.array_equal(xl, np.unique(xls[keep]))
    samples = S.decode_samples(words, info["format"])
    ref = np.zeros_like(cube)
    for t in np.nonzero(keep)[0]:  # later duplicates win, missing traces stay zero
        ref[np.searchsorted(il, ils[t]), np.searchsorted(xl, xls[t])] = samples[t]
    assert np.array_equal(cube, ref)
    assert info["num_traces"] == len(ils) and info["n_mapped"] == int(keep.sum())


def test_segy_errors(tmp_path):
    p = tmp_path / "bad.sgy"
    p.write_bytes(b"\0" * 100)
    with pytest.raises(PsmError, match="Failed to read text header"):
        H.segy_info(str(p))
    p.write_bytes(b"\0" * 3300)
    with pytest.raises(PsmError, match="Failed to read binary header"):
        H.segy_info(str(p))
    hdr = bytearray(3600)
    p.write_bytes(bytes(hdr))
    with pytest.raises(PsmError, match="Sample interval"):
        H.segy_info(str(p))
    hdr[3216:3218] = (2000).to_bytes(2, "big")
    p.write_bytes(bytes(hdr))
    with pytest.raises(PsmError, match="Number of samples"):
        H.segy_info(str(p))
    hdr[3220:3222] = (10).to_bytes(2, "big")
    p.write_bytes(bytes(hdr) + b"\0" * 100)  # shorter than one trace
    with pytest.raises(PsmError, match="No traces found"):
        H.segy_info(str(p))
    with pytest.raises(PsmError, match="Cannot open SEGY file"):
        H.segy_info(str(tmp_path / "missing.sgy"))


def test_segy_zero_labels_skipped_and_truncated_tail_ignored(tmp_path):
    d = np.arange(3 * 2 * 8, dtype=np.float32).reshape(3, 2, 8)
    p = tmp_path / "x.sgy"
    S.write_segy(str(p), d, [0, 5, 6], [1, 2], 1000, 5)  # inline label 0 is skipped
    raw = p.read_bytes() + b"\1" * 50  # a partial trailing trace is not a trace
    p.write_bytes(raw)
    il, xl, cube, info = H.read_segy(str(p))
    assert info["num_traces"] == 6 and info["n_mapped"] == 4
    assert list(il) == [5, 6] and list(xl) == [1, 2]
    assert np.array_equal(cube, d[1:])


# --------------------------------------------------------------------------- velocity


def test_velocity_providers_match_reference(tmp_path):
    v = _golden("velocity_vectors")
    p = tmp_path / "v.sgy"
    p.write_bytes(v["segy_bytes"].tobytes())
    for k in ["exact", "exact_dt", "idw"]:
        nt, dt = v[f"segy_{k}_meta"]
        c = H.velocity_cube(str(p), v[f"segy_{k}_il"], v[f"segy_{k}_xl"], int(nt), float(dt))
        ref = v[f"segy_{k}_cube"]
        if k == "idw":
            # the reference's -ffast-math build reorders the 2x2 weighted sum
            np.testing.assert_allclose(c, ref, rtol=4e-7, atol=0)
        else:
            assert np.array_equal(c, ref), k  # copy and time-interpolation paths: exact
    t = tmp_path / "t.txt"
    t.write_text(str(v["table_text"]))
    c = H.velocity_cube(str(t), v["table_il"], v["table_xl"], 25, 0.04)
    np.testing.assert_allclose(c, v["table_cube"], rtol=4e-7, atol=0)


def test_velocity_table_errors(tmp_path):
    t = tmp_path / "t.txt"
    t.write_text("1 1 0.0 2000\n   # indented comment is not a comment\n")
    with pytest.raises(PsmError, match="Invalid format at line 2"):
        H.velocity_point(str(t), 1, 1, 0, 0.002, 10)
    t.write_text("# only comments\n\n")
    with pytest.raises(PsmError, match="No valid data found"):
        H.velocity_point(str(t), 1, 1, 0, 0.002, 10)
    with pytest.raises(PsmError, match="Cannot open velocity table file"):
        H.velocity_point(str(tmp_path / "none.txt"), 1, 1, 0, 0.002, 10)


def test_velocity_constant_and_exact_table_hit(tmp_path):
    assert H.velocity_point("2500.5", 3, 4, 7, 0.002, 10) == np.float32(2500.5)
    t = tmp_path / "t.txt"
    t.write_text("1 1 0.0 2000\n2 2 0.004 2500\n2 2 0.004 9999\n")
    assert H.velocity_point(str(t), 2, 2, 2, 0.002, 10) == 2500.0  # first exact hit


# --------------------------------------------------------------------------- plan


@pytest.mark.parametrize("name", ["diffractor_pad", "ibm_segy_vel", "table_vel_noamp",
                                  "irregular_idw", "fmt3_single_xl"])
def test_plan_matches_reference_log(tmp_path, name):
    """m_il and the output size as the reference binary printed them for the same input."""
    z = _golden(name)
    meta = json.loads(str(z["meta"]))
    inp = tmp_path / "in.sgy"
    inp.write_bytes(z["input"].tobytes())
    cfg = dict(meta["config"])
    if meta["velocity_file"]:
        vp = tmp_path / meta["velocity_file"]
        vp.write_bytes(z["velocity"].tobytes())
        cfg["velocity"] = str(vp)
    lines = [f"input_data={inp}", f"output_data={tmp_path / 'out.sgy'}"]
    lines += [f"{k}={str(v).lower() if isinstance(v, bool) else v}" for k, v in cfg.items()]
    cp = tmp_path / "c.txt"
    cp.write_text("\n".join(lines) + "\n")
    plan = H.plan_config(str(cp))
    log = meta["stdout"]
    m = [ln for ln in log.splitlines() if ln.startswith("Buffer size: IL=")][0]
    assert int(m.split("IL=")[1].split()[0].lstrip("±")) == plan["m_il"]
    dims = [ln for ln in log.splitlines() if ln.startswith("Output dimensions:")][0]
    assert dims == f"Output dimensions: IL={plan['n_oi']}, XL={plan['n_ox']}"
