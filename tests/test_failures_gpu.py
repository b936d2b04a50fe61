"""Failure detection without a GPU fault.

The reference has no error paths in its kernel (src/migration_kernel.cpp:17-383) and reports
host failures with a message and exit code 1 (src/main.cpp:438-441); here every failure comes
back as a status code, and the context stays usable afterwards.

* A bounded wait that runs out: with PSM_FAULT=stall_producer the forward kernel's producer
  warp leaves the first ring stage of each tile unfilled, so the consumers' wait on it ends
  after PSM_WAIT_LIMIT_MS of GPU time; the producer's own wait for the consumers ends the same
  way, and it lets its copies into the other stage land before the CTA exits.  The call
  returns PSM_ERR_DEVICE (the kernel's PSM_DEV_ERR_TIMEOUT flag), and the next call on the same
  device, without the knob, gives the right image.
* A device allocation that fails: PSM_FAULT=nomem:K fails the K-th allocation after the
  context is created; the call returns PSM_ERR_NOMEM, leaves the context without a geometry
  (PSM_ERR_STATE until the next successful psm_set_geometry), and the context then works.

Each knob is read when a context is created, so the tests run their contexts in child
processes (spawned, with the knob in their environment) and keep this process's context
clean."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys, time
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
from poststackmig3d_b200 import Migrator
from poststackmig3d_b200 import synth as S
from poststackmig3d_b200._lib import PsmError
from helpers import geometry_for

W = S.random_workload(91, 10, 12, 200, vel_kind="lateral", pad_il=1, pad_xl=1)
g = geometry_for(W)
out = {}
m = Migrator(0)
try:
    m.set_geometry(g)
    out["geometry"] = 0
except PsmError as e:
    out["geometry"] = e.code
    buf = np.empty((g.n_oi, g.n_ox, g.n_t), dtype=np.float32)
    out["forward_without_geometry"] = m._L.psm_forward(m._ctx, buf.ctypes.data)
    m.set_geometry(g)
m.set_traces(W.data)
m.set_vrms(W.vrms_cube())
t = time.time()
try:
    m.forward()
    out["forward"] = 0
except PsmError as e:
    out["forward"] = e.code
    out["message"] = str(e)
out["forward_s"] = time.time() - t
print(json.dumps(out))
m.close()
"""


def _child(env_extra):
    env = dict(os.environ)
    env.pop("PSM_FAULT", None)
    env.update(env_extra)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], capture_output=True, text=True,
                       env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def _reference_image():
    from poststackmig3d_b200 import Migrator
    from poststackmig3d_b200 import synth as S
    from helpers import geometry_for
    W = S.random_workload(91, 10, 12, 200, vel_kind="lateral", pad_il=1, pad_xl=1)
    with Migrator(0) as m:
        m.set_geometry(geometry_for(W))
        m.set_traces(W.data)
        m.set_vrms(W.vrms_cube())
        return m.forward()


def test_stalled_producer_times_out_and_the_device_stays_usable():
    before = _reference_image()
    out = _child({"PSM_FAULT": "stall_producer", "PSM_WAIT_LIMIT_MS": "50"})
    assert out["geometry"] == 0
    assert out["forward"] == -5, out  # PSM_ERR_DEVICE
    assert "device error flags 1" in out["message"], out  # PSM_DEV_ERR_TIMEOUT
    assert out["forward_s"] < 60.0
    # the same device migrates correctly right afterwards, in a fresh context and in this one
    assert _child({})["forward"] == 0
    assert (_reference_image() == before).all()


def test_failed_allocation_reports_nomem_and_the_context_recovers():
    out = _child({"PSM_FAULT": "nomem:2"})
    assert out["geometry"] == -4, out  # PSM_ERR_NOMEM from psm_set_geometry
    assert out["forward_without_geometry"] == -2, out  # PSM_ERR_STATE
    assert out["forward"] == 0, out  # after a successful psm_set_geometry
