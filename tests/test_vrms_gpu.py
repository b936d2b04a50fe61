"""Vrms assembled on the GPU (psm_set_vrms_table / psm_set_vrms_grid) against the host
providers, bit for bit, and against the reference's own Vrms cubes (golden vectors made by
running the reference's providers; they differ from the host providers by 1-2 ulp only where
the reference's -ffast-math build reorders the inverse-distance sums)."""
import os

import numpy as np
import pytest

from poststackmig3d_b200 import Migrator, plan_geometry
from poststackmig3d_b200 import host as H

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def _migrator(il, xl, n_t, dt):
    g = plan_geometry(len(il), len(xl), int(n_t), float(dt), 25.0, 25.0, 30.0, 3000.0,
                      il_labels=il, xl_labels=xl)
    m = Migrator(0)
    m.set_geometry(g)
    return m


def _table_points(text):
    pts = []
    for line in text.splitlines():
        if not line or line[0] == "#":
            continue
        a, b, c, d = line.split()[:4]
        pts.append((int(a), int(b), float(c), float(d)))
    return pts


def test_table_vrms_matches_host_and_reference(tmp_path):
    v = _golden("velocity_vectors")
    t = tmp_path / "t.txt"
    t.write_text(str(v["table_text"]))
    il, xl = v["table_il"], v["table_xl"]
    host = H.velocity_cube(str(t), il, xl, 25, 0.04)
    with _migrator(il, xl, 25, 0.04) as m:
        m.set_vrms_table(_table_points(str(v["table_text"])), il, xl)
        got = m.get_vrms()
    assert np.array_equal(got, host)
    np.testing.assert_allclose(got, v["table_cube"], rtol=4e-7, atol=0)


def test_table_vrms_many_points(tmp_path):
    """A dense table (an exact hit, a point repeated, times off the sample grid)."""
    rng = np.random.default_rng(5)
    pts = [(int(a), int(b), float(c), float(np.float32(d))) for a, b, c, d in zip(
        rng.integers(1, 30, 300), rng.integers(1, 40, 300), rng.uniform(0, 0.4, 300),
        rng.uniform(1500, 3500, 300))]
    pts.append((5, 7, 0.008, 2100.0))   # exact hit at sample 4 of (5, 7)
    pts.append((5, 7, 0.008, 9999.0))   # the first hit wins
    t = tmp_path / "t.txt"
    t.write_text("# il xl t v\n" + "".join(f"{a} {b} {c!r} {d!r}\n" for a, b, c, d in pts))
    il = np.array([1, 5, 9, 17, 29], dtype=np.int32)
    xl = np.array([2, 7, 11, 38], dtype=np.int32)
    host = H.velocity_cube(str(t), il, xl, 120, 0.002)
    with _migrator(il, xl, 120, 0.002) as m:
        m.set_vrms_table(pts, il, xl)
        got = m.get_vrms()
    assert np.array_equal(got, host)
    assert got[1, 1, 4] == np.float32(2100.0)


@pytest.mark.parametrize("kind", ["exact", "exact_dt", "idw"])
def test_grid_vrms_matches_host_and_reference(tmp_path, kind):
    v = _golden("velocity_vectors")
    p = tmp_path / "v.sgy"
    p.write_bytes(v["segy_bytes"].tobytes())
    g_il, g_xl, grid, info = H.read_segy(str(p))
    nt, dt = v[f"segy_{kind}_meta"]
    il, xl = v[f"segy_{kind}_il"], v[f"segy_{kind}_xl"]
    host = H.velocity_cube(str(p), il, xl, int(nt), float(dt))
    with _migrator(il, xl, nt, dt) as m:
        m.set_vrms_grid(grid, g_il, g_xl, info["dt_seconds"], il, xl)
        got = m.get_vrms()
    assert np.array_equal(got, host), kind
    ref = v[f"segy_{kind}_cube"]
    if kind == "idw":
        np.testing.assert_allclose(got, ref, rtol=4e-7, atol=0)
    else:
        assert np.array_equal(got, ref)
