"""Out-of-core forward (psm_forward_streamed): a cube held in host memory, migrated in
slabs through a small device budget, equals the resident-cube forward bit for bit."""
import numpy as np
import pytest

from poststackmig3d_b200 import Migrator
from poststackmig3d_b200 import synth as S
from poststackmig3d_b200.migration import plan_slabs, slab_bytes

from helpers import geometry_for, gpu_forward

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,pad_il,vel,precision", [(71, 2, "lateral", "f32"),
                                                       (72, 0, "linear", "f32"),
                                                       (73, 1, "lateral", "bf16")])
def test_streamed_forward_equals_resident(seed, pad_il, vel, precision):
    """Consecutive slabs keep their shared input inlines on the device (moved to the front of
    the buffers) and upload only the new ones; 16-bit storage moves its words and scales."""
    import dataclasses
    W = S.random_workload(seed, 24, 13, 260, vel_kind=vel, pad_il=pad_il, pad_xl=2,
                          d_il=150.0, angle=25.0)
    g = dataclasses.replace(geometry_for(W), precision=precision)
    whole, _, _ = gpu_forward(W, g)
    budget = int(1.1 * slab_bytes(g, min(g.n_il, 2 * (g.m_il + g.pad_il) + 1), 1))
    assert len(plan_slabs(g, budget)) > 1
    with Migrator(0) as m:
        img = m.forward_streamed(g, W.data, W.vrms_cube(), budget)
        # the kept inlines live only in the staged storage afterwards: no traces to read
        buf = np.empty(W.data.shape, dtype=np.float32)
        assert m._L.psm_get_traces(m._ctx, buf.ctypes.data) == -2  # PSM_ERR_STATE
    assert np.array_equal(img, whole)
