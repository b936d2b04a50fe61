"""Generate the committed golden fixtures by running the REFERENCE itself.

Needs the reference built from its own sources (`make -C oracle ref`, which reads the
reference tree).  For each case it writes a small seeded SEG-Y (and velocity file), runs the
reference's serial binary (oracle/_ref/poststackmig_serial) on a config.txt, and stores the
input bytes, the config and the reference's output bytes in tests/golden/<case>.npz.  It also
records the reference's own IBM<->IEEE conversions and Vrms cubes from its velocity providers.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from poststackmig3d_b200 import synth as S  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def _cases():
    rng = np.random.default_rng(7)
    cases = []

    # 1: diffractor, constant V, IEEE, padding both ways (the config-1 recipe, scaled down)
    d = S.diffractor_cube(19, 15, 100, 0.004, 25.0, 2000.0, 0.2, 20.0, 0.1, seed=11)
    cases.append(dict(name="diffractor_pad", data=d, il=np.arange(1, 20),
                      xl=np.arange(1, 16), dt_us=4000, fmt=5,
                      cfg=dict(inline_step=25.0, crossline_step=25.0, inline_padding=3,
                               crossline_padding=4, velocity="2000.0", angle_aperture=30.0,
                               amp_correction=True)))

    # 2: IBM samples, Vrms from a same-grid SEG-Y (direct copy path), unsorted traces
    n_il, n_xl, n_t = 13, 11, 96
    d = rng.standard_normal((n_il, n_xl, n_t)).astype(np.float32)
    vr = S.linear_vrms(n_il, n_xl, n_t, 0.004, 20.0, 1700.0, 2600.0, 0.1, 100.0)
    order = rng.permutation(n_il * n_xl)
    cases.append(dict(name="ibm_segy_vel", data=d, il=np.arange(101, 101 + n_il),
                      xl=np.arange(201, 201 + n_xl), dt_us=4000, fmt=1, order=order,
                      vel=dict(kind="segy", data=vr, il=np.arange(101, 101 + n_il),
                               xl=np.arange(201, 201 + n_xl), dt_us=4000, fmt=5),
                      cfg=dict(inline_step=20.0, crossline_step=20.0, inline_padding=2,
                               crossline_padding=0, angle_aperture=40.0,
                               amp_correction=True)))

    # 3: text-table velocity (IDW over all points), amplitude correction off
    n_il, n_xl, n_t = 11, 9, 80
    d = rng.standard_normal((n_il, n_xl, n_t)).astype(np.float32)
    table = "# IL XL TIME VEL\n" + "\n".join(
        f"{il} {xl} {t:.3f} {v:.1f}" for il, xl, t, v in
        [(1, 1, 0.0, 1800.0), (1, 9, 0.2, 2100.0), (11, 1, 0.1, 1950.0),
         (11, 9, 0.3, 2400.0), (6, 5, 0.15, 2000.0)]) + "\n"
    cases.append(dict(name="table_vel_noamp", data=d, il=np.arange(1, n_il + 1),
                      xl=np.arange(1, n_xl + 1), dt_us=4000, fmt=5,
                      vel=dict(kind="table", text=table),
                      cfg=dict(inline_step=25.0, crossline_step=30.0, inline_padding=0,
                               crossline_padding=2, angle_aperture=35.0,
                               amp_correction=False)))

    # 4: irregular labels (a missing inline label, crossline step 2, missing traces) and a
    #    coarser Vrms SEG-Y grid (inverse-distance path)
    n_il, n_xl, n_t = 7, 9, 72
    d = rng.standard_normal((n_il, n_xl, n_t)).astype(np.float32)
    il = np.array([5, 6, 7, 9, 10, 11, 12])
    xl = np.arange(10, 10 + 2 * n_xl, 2)
    vgrid = S.linear_vrms(4, 5, 36, 0.008, 50.0, 1800.0, 2500.0, 0.05, 200.0)
    cases.append(dict(name="irregular_idw", data=d, il=il, xl=xl, dt_us=4000, fmt=5,
                      skip=[(6, 14), (10, 10), (12, 26)],
                      vel=dict(kind="segy", data=vgrid, il=np.array([5, 7, 9, 12]),
                               xl=np.array([10, 13, 17, 21, 26]), dt_us=8000, fmt=1),
                      cfg=dict(inline_step=25.0, crossline_step=25.0, inline_padding=2,
                               crossline_padding=2, angle_aperture=45.0,
                               amp_correction=True)))

    # 5: unknown format code (3) -> read as IEEE with a warning; one crossline with padding
    n_il, n_xl, n_t = 9, 1, 64
    d = rng.standard_normal((n_il, n_xl, n_t)).astype(np.float32)
    cases.append(dict(name="fmt3_single_xl", data=d, il=np.arange(1, n_il + 1),
                      xl=np.array([7]), dt_us=2000, fmt=5, format_code=3,
                      cfg=dict(inline_step=25.0, crossline_step=25.0, inline_padding=1,
                               crossline_padding=3, velocity="1800", angle_aperture=60.0,
                               amp_correction=True)))
    return cases


def _run_case(c, tmp):
    inp = os.path.join(tmp, c["name"] + ".sgy")
    outp = os.path.join(tmp, c["name"] + "_out.sgy")
    S.write_segy(inp, c["data"], c["il"], c["xl"], c["dt_us"], c["fmt"], order=c.get("order"),
                 skip=c.get("skip"), format_code=c.get("format_code"), text=c["name"])
    cfg = dict(input_data=inp, output_data=outp)
    cfg.update(c["cfg"])
    vel_bytes = b""
    vel_name = ""
    if "vel" in c:
        v = c["vel"]
        if v["kind"] == "segy":
            vel_name = c["name"] + "_vel.sgy"
            vp = os.path.join(tmp, vel_name)
            S.write_segy(vp, v["data"], v["il"], v["xl"], v["dt_us"], v["fmt"], text="vrms")
        else:
            vel_name = c["name"] + "_vel.txt"
            vp = os.path.join(tmp, vel_name)
            with open(vp, "w") as f:
                f.write(v["text"])
        with open(vp, "rb") as f:
            vel_bytes = f.read()
        cfg["velocity"] = vp
    cfgp = os.path.join(tmp, c["name"] + ".txt")
    O.write_config(cfgp, **cfg, n_threads=1)
    r = O.run_ref_binary(cfgp, "serial")
    if r.returncode != 0:
        raise RuntimeError(f"reference failed on {c['name']}: {r.stderr}")
    with open(inp, "rb") as f:
        in_bytes = f.read()
    with open(outp, "rb") as f:
        out_bytes = f.read()
    cfg_store = {k: v for k, v in cfg.items() if k not in ("input_data", "output_data",
                                                           "velocity")}
    if "vel" not in c:
        cfg_store["velocity"] = c["cfg"]["velocity"]
    meta = dict(config=cfg_store, velocity_file=vel_name, stdout=r.stdout[-4000:])
    np.savez_compressed(os.path.join(OUT, c["name"] + ".npz"),
                        input=np.frombuffer(in_bytes, dtype=np.uint8),
                        output=np.frombuffer(out_bytes, dtype=np.uint8),
                        velocity=np.frombuffer(vel_bytes, dtype=np.uint8),
                        meta=np.array(json.dumps(meta)))
    return vp if "vel" in c else None


def _ibm_vectors():
    L = O.ref_lib("serial")
    rng = np.random.default_rng(3)
    floats = np.concatenate([
        np.array([0.0, -0.0, 1.0, -1.0, 0.5, 16.0, 1.0 / 16, 256.0, 0.1, -0.1, 3.14159265,
                  1e-5, -1e-5, 123456.789, 1e20, -1e-20, 5.877472e-39, 2.0 ** -130,
                  3.0e38], dtype=np.float32),
        rng.standard_normal(200).astype(np.float32) * np.float32(10.0) ** rng.integers(
            -8, 8, 200).astype(np.float32)]).astype(np.float32)
    enc = np.array([L.ref_ieee_to_ibm(float(f)) for f in floats], dtype=np.uint32)
    words = np.concatenate([
        np.array([0x00000000, 0x80000000, 0x41100000, 0xC1100000, 0x40800000, 0x42640000,
                  0x7FFFFFFF, 0xFFFFFFFF, 0x00000001, 0x00100000, 0x3F100000, 0x61100000,
                  0x21100000], dtype=np.uint32),
        rng.integers(0, 2 ** 32, 300, dtype=np.uint64).astype(np.uint32)])
    dec = np.array([L.ref_ibm_to_ieee(int(w)) for w in words], dtype=np.float32)
    np.savez_compressed(os.path.join(OUT, "ibm_vectors.npz"), floats=floats, ibm=enc,
                        words=words, decoded=dec)


def _velocity_vectors(tmp):
    """Vrms cubes from the reference's providers on small grids."""
    out = {}
    vr = S.linear_vrms(5, 6, 40, 0.004, 25.0, 1600.0, 2600.0, 0.1, 50.0)
    p = os.path.join(tmp, "vgrid.sgy")
    S.write_segy(p, vr, np.array([3, 5, 7, 9, 11]), np.array([2, 4, 6, 8, 10, 12]), 4000, 5)
    with open(p, "rb") as f:
        out["segy_bytes"] = np.frombuffer(f.read(), dtype=np.uint8)
    grids = {
        # exact grid, same dt/nt (direct copy)
        "exact": (np.array([3, 5, 7, 9, 11]), np.array([2, 4, 6, 8, 10, 12]), 40, 0.004),
        # exact grid, different dt (per-sample getVelocity time interpolation)
        "exact_dt": (np.array([3, 5, 7]), np.array([2, 4, 6]), 50, 0.003),
        # off-grid inlines/crosslines (2x2 inverse-distance), beyond the ends too
        "idw": (np.array([1, 4, 6, 12, 14]), np.array([1, 3, 5, 9, 13]), 30, 0.006),
    }
    for k, (il, xl, nt, dt) in grids.items():
        cube = np.zeros((len(il), len(xl), nt), dtype=np.float32)
        rc = O.ref_lib("serial").ref_velocity_cube(p.encode(), il.astype(np.int32), len(il),
                                                   xl.astype(np.int32), len(xl), nt, dt,
                                                   cube)
        assert rc == 0
        out[f"segy_{k}_il"] = il
        out[f"segy_{k}_xl"] = xl
        out[f"segy_{k}_meta"] = np.array([nt, dt])
        out[f"segy_{k}_cube"] = cube
    table = ("# comment\n1 1 0.0 1800\n1 10 0.5 2200.5\n10 1 0.25 2000\n"
             "10 10 1.0 3000\n5 5 0.4 2400\n5 5 0.4 2600\n")
    p = os.path.join(tmp, "vtable.txt")
    with open(p, "w") as f:
        f.write(table)
    out["table_text"] = np.array(table)
    il = np.array([1, 3, 5, 10, 12])
    xl = np.array([1, 5, 10])
    cube = np.zeros((len(il), len(xl), 25), dtype=np.float32)
    assert O.ref_lib("serial").ref_velocity_cube(p.encode(), il.astype(np.int32), len(il),
                                                 xl.astype(np.int32), len(xl), 25, 0.04,
                                                 cube) == 0
    out["table_il"] = il
    out["table_xl"] = xl
    out["table_cube"] = cube
    np.savez_compressed(os.path.join(OUT, "velocity_vectors.npz"), **out)


def main():
    if not O.ref_available():
        O.build()
    with tempfile.TemporaryDirectory() as tmp:
        for c in _cases():
            _run_case(c, tmp)
            print("wrote", c["name"])
        _velocity_vectors(tmp)
    _ibm_vectors()
    print("done")


if __name__ == "__main__":
    main()
