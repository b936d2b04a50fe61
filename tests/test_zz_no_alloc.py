"""psm_forward_noalloc: the forward migration for callers that cannot call cudaMalloc.

Such callers (an application or framework that owns every device byte through its own pool,
or a pipeline that must not pay cudaMalloc's implicit device synchronisation after set-up)
pass their own device buffers; the entry point's working memory is a fixed file-scope device
array.  This file is collected last so that, if it fails, a run that stops at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest

from poststackmig3d_b200 import Migrator, _lib
from poststackmig3d_b200 import synth as S
from poststackmig3d_b200._lib import PsmGeom

from helpers import geometry_for, rel_err


def _fn():
    f = _lib.cuda().psm_forward_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(PsmGeom), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    return f


def test_noalloc_rejects_bad_arguments_before_touching_a_device():
    W = S.random_workload(40, 5, 6, 50, vel_kind="const")
    g = geometry_for(W)
    gc = g.to_c()
    oc = np.ascontiguousarray(g.out_center, dtype=np.int32)
    f = _fn()
    assert f(ctypes.byref(gc), oc.ctypes.data, None, 16, 16, None) == -1  # PSM_ERR_ARG
    big = g.to_c()
    big.n_t = 20000  # beyond the stated 16384-sample limit of the scratch array
    assert f(ctypes.byref(big), None, 16, 16, 16, None) == -6  # PSM_ERR_UNSUPPORTED
    big = g.to_c()
    big.n_oi = 5000  # beyond 4096 output inlines
    assert f(ctypes.byref(big), None, 16, 16, 16, None) == -6


@pytest.mark.gpu
def test_noalloc_matches_forward_on_two_calls_in_a_row():
    """Both entry points run the same kernel on the same tables, so the images are equal bit
    for bit.  The cases run twice in a row (the array keeps the previous call's contents), the
    second round under a free-memory check: once the library's kernels are loaded, a call
    allocates no device memory."""
    import torch

    def pair_cube(data, ns):
        # (d[t], d[t+1] - d[t]) with d = 0 past the last sample, rows of ns pairs
        n_il, n_xl, n_t = data.shape
        d = torch.zeros((n_il, n_xl, ns + 1), dtype=torch.float32, device="cuda")
        d[..., :n_t] = torch.from_numpy(data).cuda()
        return torch.stack([d[..., :ns], d[..., 1:] - d[..., :ns]], dim=-1).contiguous()

    f = _fn()
    cases = [S.random_workload(41, 12, 15, 300, vel_kind="lateral", pad_il=2, pad_xl=3),
             S.random_workload(42, 9, 10, 130, vel_kind="linear", angle=50.0)]
    runs = []
    for k, W in enumerate(cases):
        g = geometry_for(W)
        with Migrator(0) as m:  # the existing entry point
            m.set_geometry(g)
            m.set_traces(W.data)
            m.set_vrms(W.vrms_cube())
            ref = m.forward()
        ns = (g.n_t + 7) & ~7
        img = torch.full((g.n_oi, g.n_ox, g.n_t), float("nan"), dtype=torch.float32,
                         device="cuda")
        # the first case passes NULL: the regular-label centres clamp(o - pad_il)
        oc = None if k == 0 else np.ascontiguousarray(g.out_center, dtype=np.int32)
        runs.append((g.to_c(), oc, pair_cube(W.data, ns),
                     torch.from_numpy(W.vrms_cube()).cuda(), img, ref))
    torch.cuda.synchronize()

    def call(gc, oc, pairs, vrms, img, ref):
        img.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = f(ctypes.byref(gc), None if oc is None else oc.ctypes.data, pairs.data_ptr(),
               vrms.data_ptr(), img.data_ptr(), None)
        assert rc == 0
        got = img.cpu().numpy()
        assert np.array_equal(got, ref), rel_err(got, ref)

    for r in runs:  # the first round loads the library's kernels on this device
        call(*r)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for r in runs:  # the second call of each case reuses what the previous calls left
        call(*r)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
