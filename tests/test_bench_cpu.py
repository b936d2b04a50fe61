"""bench.py's reference arm runs on the host cores (no GPU) and prints the JSON line the driver
reads: the reference's own kernel (oracle/_ref, or the oracle port where the reference was not
built) timed on a bounded sample of the workload, with its CPU-baseline and end-to-end keys.
Under torchrun only rank 0 works and prints; the other ranks exit 0 without work."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                          cwd=ROOT, env=e, capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_one_line():
    r = _bench("--impl", "reference", "--workload", "config1", "--steps", "2", "--warmup", "1",
               "--cpu-rows", "1")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "G/s" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["ms_per_step"] > 0
    assert d["config"]["workload"].startswith("config1")
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    r = _bench("--impl", "reference", "--workload", "config1", "--steps", "1", "--warmup", "0",
               "--cpu-rows", "1", env={"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
