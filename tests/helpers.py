"""Shared test helpers: run the GPU operator and the oracle on the same workload."""
from __future__ import annotations

import numpy as np

import oracle as O
from poststackmig3d_b200 import Migrator, estimate_max_velocity, plan_geometry

# FP32 parity bar against the reference: 1e-4 relative RMS, and max error 1e-4 of the
# image peak.  Second bar (fp32_floor_ok): the GPU image's distance to the FP64 oracle of
# the same operator may be at most 3x the distance of the reference's own FP32 arithmetic
# (the oracle's FP32 restatement) to that FP64 oracle -- i.e. no worse than FP32 noise.
REL_RMS_TOL = 1e-4
MAX_REL_TOL = 1e-4
FP32_FLOOR_FACTOR = 3.0


def fp32_floor_ok(img, ref32, ref64):
    e_gpu = rel_err(img, ref64)[0]
    e_ref = rel_err(ref32, ref64)[0]
    return e_gpu <= FP32_FLOOR_FACTOR * e_ref + 1e-7, (e_gpu, e_ref)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.sqrt(np.mean(b * b)) or 1.0
    rms = np.sqrt(np.mean((a - b) ** 2)) / den
    mx = np.abs(a - b).max() / (np.abs(b).max() or 1.0)
    return float(rms), float(mx)


def geometry_for(W, il_labels=None, xl_labels=None):
    vr = W.vrms_cube()
    n_il, n_xl, n_t = W.data.shape
    return plan_geometry(n_il, n_xl, n_t, W.dt, W.d_il, W.d_xl, W.angle,
                         estimate_max_velocity(vr), W.pad_il, W.pad_xl, W.amp,
                         il_labels=il_labels, xl_labels=xl_labels)


def gpu_forward(W, g=None):
    g = g or geometry_for(W)
    with Migrator(0) as m:
        m.set_geometry(g)
        m.set_traces(W.data)
        m.set_vrms(W.vrms_cube())
        img = m.forward()
        n = m.count_terms()
    return img, n, g


def oracle_forward(W, g, flags=O.CONTRACT | O.AVX_ORDER, want64=False):
    return O.migrate_volume(W.data, W.vrms_cube(), g.out_center, g.n_ox, g.pad_il, g.pad_xl,
                            g.m_il, np.float32(g.dt_seconds), g.t0(), np.float32(g.tan2),
                            g.d_il, g.d_xl, g.amp, flags, 0, want64)


def dequantized(data, precision):
    """The fp32 samples that 16-bit storage represents (oracle.dequantized)."""
    return O.dequantized(data, precision)
