"""The forward kernel's per-sample pass bound search, restated in C (tests/pass_bound_search.c)
with the same FP32 operations: galloping out from an estimate of the boundary and then
bisecting returns the bound that a bisection of all of [0, md2] returns, from the kernel's
estimate and from any other start, in about a quarter of the evaluations.  On the GPU the
bound decides which terms the kernel keeps, so the term counts there equal the oracle's
(tests/test_forward_gpu.py); this covers many more (v, t0, dt, n_t, aperture) cases."""
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def test_galloping_search_finds_the_bisection_bound(tmp_path):
    exe = str(tmp_path / "pass_bound_search")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-o", exe,
                    os.path.join(HERE, "pass_bound_search.c"), "-lm"], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    m = re.match(r"cases (\d+) searched (\d+) mismatches (\d+) bisection ([\d.]+) "
                 r"gallop ([\d.]+)", r.stdout)
    assert m, r.stdout
    cases, searched, bad = int(m[1]), int(m[2]), int(m[3])
    bisect, gallop = float(m[4]), float(m[5])
    assert r.returncode == 0 and bad == 0, r.stdout
    assert cases == 360000 and searched > 50000
    assert gallop < 0.3 * bisect, (gallop, bisect)
