"""Python face of the migration operator (the reference's MigrationKernel seam).

* MigrationKernel.kirchhoff_kernel_3d_with_padding mirrors
  MigrationKernel::kirchhoffKernel3DWithPadding (include/migration_kernel.h:16-31) argument by
  argument and runs it on the GPU through psm_kirchhoff_inline.
* Migrator holds a whole cube resident in HBM (psm_ctx) and migrates every output inline in
  one launch; plan_geometry() derives its parameters the way src/main.cpp:124-217 does for a
  regular grid.
Everything here calls libpsm_cuda.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import PsmGeom, check

PRECISIONS = {"f32": 0, "bf16": 1, "f16": 2}


def _addr(a) -> int:
    """Host address of a C-contiguous float32 numpy array or CPU torch tensor."""
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if a.is_cuda:
            raise ValueError("host buffer expected")
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(type(a))


def _f32(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape != tuple(shape):
        a = a.reshape(shape)
    return a


# ----------------------------------------------------------------------------- geometry


def tan2_theta(angle_deg: float) -> float:
    """src/main.cpp:188-189: float(tan(angle * pi / 180)) squared in float."""
    t = np.float32(math.tan(angle_deg * math.pi / 180.0))
    return float(np.float32(t * t))


def max_aperture_il(max_v: float, n_t: int, dt_seconds: float, tan2: float,
                    inline_step: float) -> int:
    """src/main.cpp:197-201 (the float/double mix kept)."""
    max_t = (n_t - 1) * dt_seconds
    rad = np.float32(np.float32(np.float32(max_v) * np.float32(max_t)) / np.float32(2.0))
    rad = np.float32(rad * np.sqrt(np.float32(tan2), dtype=np.float32))
    return int(float(rad) / inline_step) + 1


def padded_labels(labels: Sequence[int], pad: int) -> np.ndarray:
    """src/main.cpp:144-172: extend by pad steps of labels[1]-labels[0] on both sides."""
    labels = np.asarray(labels, dtype=np.int64)
    if pad > 0 and len(labels) > 1:
        step = int(labels[1] - labels[0])
        return np.arange(labels[0] - pad * step, labels[-1] + pad * step + 1, step,
                         dtype=np.int64)
    return labels.copy()


def output_centers(in_labels: Sequence[int], out_labels: Sequence[int]) -> np.ndarray:
    """src/main.cpp:258-288: the real inline index each output inline migrates."""
    in_labels = np.asarray(in_labels, dtype=np.int64)
    res = np.empty(len(out_labels), dtype=np.int32)
    n = len(in_labels)
    for o, lab in enumerate(out_labels):
        hit = np.nonzero(in_labels == lab)[0]
        if len(hit):
            res[o] = hit[0]
        elif lab < in_labels[0]:
            res[o] = 0
        elif lab > in_labels[-1]:
            res[o] = n - 1
        else:
            res[o] = int(np.argmin(np.abs(in_labels - lab)))  # first minimum, as :278-284
    return res


@dataclasses.dataclass
class Geometry:
    n_il: int
    n_xl: int
    n_t: int
    dt_seconds: float
    d_il: float
    d_xl: float
    tan2: float
    m_il: int
    pad_il: int
    pad_xl: int
    n_oi: int
    n_ox: int
    out_center: np.ndarray
    amp: bool = True
    precision: str = "f32"
    compensated: bool = False
    compat_omp_pad: bool = False  # trailing padded crosslines as the reference's OpenMP build

    @property
    def dt(self) -> float:
        return float(np.float32(self.dt_seconds))

    def t0(self) -> np.ndarray:
        """src/main.cpp:214-217."""
        return np.array([np.float32(i * self.dt_seconds) for i in range(self.n_t)],
                        dtype=np.float32)

    def to_c(self) -> PsmGeom:
        return PsmGeom(self.n_il, self.n_xl, self.n_t, self.pad_il, self.pad_xl, self.n_oi,
                       self.n_ox, self.m_il, int(bool(self.amp)), PRECISIONS[self.precision],
                       np.float32(self.dt_seconds), self.d_il, self.d_xl, self.tan2,
                       self.dt_seconds, int(bool(self.compensated)),
                       int(bool(self.compat_omp_pad)))


def plan_geometry(n_il: int, n_xl: int, n_t: int, dt_seconds: float, d_il: float,
                  d_xl: float, angle: float, max_v: float, pad_il: int = 0, pad_xl: int = 0,
                  amp: bool = True, il_labels=None, xl_labels=None,
                  precision: str = "f32") -> Geometry:
    """Geometry of a migration as src/main.cpp:140-217 derives it.  max_v is the value of
    estimateMaxVelocity (main.cpp:22-64)."""
    il_labels = np.arange(1, n_il + 1) if il_labels is None else np.asarray(il_labels)
    xl_labels = np.arange(1, n_xl + 1) if xl_labels is None else np.asarray(xl_labels)
    out_il = padded_labels(il_labels, pad_il)
    out_xl = padded_labels(xl_labels, pad_xl)
    t2 = tan2_theta(angle)
    return Geometry(n_il, n_xl, n_t, dt_seconds, d_il, d_xl, t2,
                    max_aperture_il(max_v if max_v >= 100.0 else 3000.0, n_t, dt_seconds, t2,
                                    d_il),
                    pad_il, pad_xl, len(out_il), len(out_xl),
                    output_centers(il_labels, out_il), amp, precision)


# ----------------------------------------------------------------------------- slabs

Slab = tuple  # (o0, o1, i0, i1): output inlines [o0, o1) read input inlines [i0, i1)


def _slab_tuple(s) -> Slab:
    return (s.o0, s.o1, s.i0, s.i1)


def slab_bytes(g: Geometry, n_in: int, n_out: int) -> int:
    """Device bytes a slab of n_in input and n_out output inlines holds (psm_slab_bytes)."""
    gc = g.to_c()
    return int(_lib.cuda().psm_slab_bytes(ctypes.byref(gc), int(n_in), int(n_out)))


def plan_slabs(g: Geometry, max_device_bytes: int):
    """Consecutive slabs of output inlines of at most max_device_bytes each."""
    gc = g.to_c()
    oc = np.ascontiguousarray(g.out_center, dtype=np.int32)
    arr = (_lib.PsmSlab * max(g.n_oi, 1))()
    n = ctypes.c_int32()
    check(_lib.cuda().psm_plan_slabs(ctypes.byref(gc), oc.ctypes.data, int(max_device_bytes),
                                     arr, g.n_oi, ctypes.byref(n)), lambda: "psm_plan_slabs")
    return [_slab_tuple(arr[k]) for k in range(n.value)]


def split_slabs(g: Geometry, n_parts: int, weight=None):
    """n_parts consecutive slabs of about equal work (weight[o] per output inline)."""
    gc = g.to_c()
    oc = np.ascontiguousarray(g.out_center, dtype=np.int32)
    w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float64)
    arr = (_lib.PsmSlab * n_parts)()
    check(_lib.cuda().psm_split_slabs(ctypes.byref(gc), oc.ctypes.data,
                                      None if w is None else w.ctypes.data, int(n_parts), arr),
          lambda: "psm_split_slabs")
    return [_slab_tuple(arr[k]) for k in range(n_parts)]


def slab_geometry(g: Geometry, slab: Slab) -> Geometry:
    """The slab as a problem of its own (traces and Vrms from input inline slab[2] on)."""
    gc = g.to_c()
    oc = np.ascontiguousarray(g.out_center, dtype=np.int32)
    s = _lib.PsmSlab(*slab)
    loc = PsmGeom()
    lc = np.zeros(max(slab[1] - slab[0], 1), dtype=np.int32)
    check(_lib.cuda().psm_slab_geometry(ctypes.byref(gc), oc.ctypes.data, ctypes.byref(s),
                                        ctypes.byref(loc), lc.ctypes.data),
          lambda: "psm_slab_geometry")
    return dataclasses.replace(g, n_il=loc.n_il, n_oi=loc.n_oi, out_center=lc[:loc.n_oi])


def estimate_max_velocity(vrms: np.ndarray) -> float:
    """src/main.cpp:22-64 on a dense Vrms cube: max over (first, middle, last) inline x
    (first, middle, last) crossline at the last sample; below 100 m/s -> 3000."""
    n_il, n_xl, n_t = vrms.shape
    ils = [0] + ([n_il // 2, n_il - 1] if n_il > 1 else [])
    xls = [0] + ([n_xl // 2, n_xl - 1] if n_xl > 1 else [])
    mv = 0.0
    for i in ils:
        for x in xls:
            mv = max(mv, float(vrms[i, x, n_t - 1]))
    return mv if mv >= 100.0 else 3000.0


# ----------------------------------------------------------------------------- operator


def measure_limbs(device: int = 0) -> dict:
    """Measured throughput of the SM limbs the summation draws on (psm_measure_limbs): MUFU
    rsqrt, scalar and packed fp32 FMA, 8-byte shared loads and shared fp32 reductions, each
    per SM clock per SM, and the SM clock the probes ran at."""
    from ._lib import PsmLimbs
    out = PsmLimbs()
    check(_lib.cuda().psm_measure_limbs(device, ctypes.byref(out)))
    return out.as_dict()


class Migrator:
    """A cube resident on one GPU and its forward (migration) operator."""

    def __init__(self, device: int = 0):
        self._L = _lib.cuda()
        self._ctx = ctypes.c_void_p()
        check(self._L.psm_create(ctypes.byref(self._ctx), device), lambda: "psm_create")
        self.geom: Optional[Geometry] = None

    def _err(self):
        return self._L.psm_last_error(self._ctx).decode()

    def close(self):
        if self._ctx:
            self._L.psm_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_geometry(self, g: Geometry) -> None:
        oc = np.ascontiguousarray(g.out_center, dtype=np.int32)
        gc = g.to_c()
        self.geom = None  # as in the library: no geometry unless this call succeeds
        check(self._L.psm_set_geometry(self._ctx, ctypes.byref(gc), oc.ctypes.data),
              self._err)
        self.geom = g

    def set_traces(self, data) -> None:
        g = self.geom
        if isinstance(data, np.ndarray):
            data = _f32(data, (g.n_il, g.n_xl, g.n_t))
        check(self._L.psm_set_traces(self._ctx, _addr(data)), self._err)

    def forward_streamed(self, g: Geometry, traces, vrms, max_device_bytes: int) -> np.ndarray:
        """Migrate a host-resident cube in slabs of at most max_device_bytes of device memory
        (psm_forward_streamed); the ctx's geometry is the last slab's afterwards."""
        tr = _f32(traces, (g.n_il, g.n_xl, g.n_t))
        vr = _f32(vrms, (g.n_il, g.n_xl, g.n_t))
        img = np.empty((g.n_oi, g.n_ox, g.n_t), dtype=np.float32)
        gc = g.to_c()
        oc = np.ascontiguousarray(g.out_center, dtype=np.int32)
        check(self._L.psm_forward_streamed(self._ctx, ctypes.byref(gc), oc.ctypes.data,
                                           tr.ctypes.data, vr.ctypes.data, img.ctypes.data,
                                           int(max_device_bytes)), self._err)
        self.geom = None
        return img

    def set_vrms_table(self, points, il_labels, xl_labels) -> None:
        """Vrms from a text table's points [(il, xl, time_s, v), ...], assembled on the GPU."""
        pts = list(points)
        p_il = np.array([p[0] for p in pts], dtype=np.int32)
        p_xl = np.array([p[1] for p in pts], dtype=np.int32)
        p_t = np.array([p[2] for p in pts], dtype=np.float64)
        p_v = np.array([p[3] for p in pts], dtype=np.float32)
        il = np.ascontiguousarray(il_labels, dtype=np.int32)
        xl = np.ascontiguousarray(xl_labels, dtype=np.int32)
        check(self._L.psm_set_vrms_table(self._ctx, p_il.ctypes.data, p_xl.ctypes.data,
                                         p_t.ctypes.data, p_v.ctypes.data, len(pts),
                                         il.ctypes.data, xl.ctypes.data), self._err)

    def set_vrms_grid(self, grid, g_il, g_xl, g_dt: float, il_labels, xl_labels) -> None:
        """Vrms from a SEG-Y Vrms grid [g_nil][g_nxl][g_nt] (sorted labels), on the GPU."""
        gr = _f32(grid)
        gi = np.ascontiguousarray(g_il, dtype=np.int32)
        gx = np.ascontiguousarray(g_xl, dtype=np.int32)
        il = np.ascontiguousarray(il_labels, dtype=np.int32)
        xl = np.ascontiguousarray(xl_labels, dtype=np.int32)
        check(self._L.psm_set_vrms_grid(self._ctx, gr.ctypes.data, gi.ctypes.data, len(gi),
                                        gx.ctypes.data, len(gx), gr.shape[2], float(g_dt),
                                        il.ctypes.data, xl.ctypes.data), self._err)

    def get_vrms(self) -> np.ndarray:
        g = self.geom
        out = np.empty((g.n_il, g.n_xl, g.n_t), dtype=np.float32)
        check(self._L.psm_get_vrms(self._ctx, out.ctypes.data), self._err)
        return out

    def set_traces_segy(self, records, format: int, position) -> None:
        """Upload SEG-Y trace records (uint8 [n_records][240 + 4 n_t], as in the file after
        its 3600 header bytes) and decode them on the GPU into the resident cube; record r
        fills cube trace position[r] (il_index * n_xl + xl_index) or nothing (-1)."""
        rec = np.ascontiguousarray(records, dtype=np.uint8)
        n_t = self.geom.n_t
        n = rec.size // (240 + 4 * n_t)
        if rec.size != n * (240 + 4 * n_t):
            raise ValueError("records are not whole traces of 240 + 4 n_t bytes")
        pos = np.ascontiguousarray(position, dtype=np.int32)
        if pos.size != n:
            raise ValueError("one position per record")
        check(self._L.psm_set_traces_segy(self._ctx, rec.ctypes.data, n, int(format),
                                          pos.ctypes.data), self._err)

    def get_image_segy(self, format: int, source, il_label, xl_label) -> np.ndarray:
        """The image as output SEG-Y trace records (uint8 [n_oi * n_ox][240 + 4 n_t])."""
        g = self.geom
        out = np.empty((g.n_oi * g.n_ox, 240 + 4 * g.n_t), dtype=np.uint8)
        src = np.ascontiguousarray(source, dtype=np.int32)
        il = np.ascontiguousarray(il_label, dtype=np.int32)
        xl = np.ascontiguousarray(xl_label, dtype=np.int32)
        if src.size != g.n_oi * g.n_ox or il.size != g.n_oi or xl.size != g.n_ox:
            raise ValueError("source [n_oi * n_ox], il_label [n_oi], xl_label [n_ox]")
        check(self._L.psm_get_image_segy(self._ctx, out.ctypes.data, int(format),
                                         src.ctypes.data, il.ctypes.data, xl.ctypes.data),
              self._err)
        return out

    def get_traces(self) -> np.ndarray:
        g = self.geom
        out = np.empty((g.n_il, g.n_xl, g.n_t), dtype=np.float32)
        check(self._L.psm_get_traces(self._ctx, out.ctypes.data), self._err)
        return out

    def set_image(self, image) -> None:
        g = self.geom
        img = _f32(image, (g.n_oi, g.n_ox, g.n_t))
        check(self._L.psm_set_image(self._ctx, img.ctypes.data), self._err)

    def set_vrms(self, vrms) -> None:
        g = self.geom
        if isinstance(vrms, np.ndarray):
            vrms = _f32(vrms, (g.n_il, g.n_xl, g.n_t))
        check(self._L.psm_set_vrms(self._ctx, _addr(vrms)), self._err)

    def image_shape(self):
        g = self.geom
        return (g.n_oi, g.n_ox, g.n_t)

    def forward(self, out=None):
        """Migrate the resident cube; returns image [n_oi][n_ox][n_t] (host)."""
        if out is None:
            out = np.empty(self.image_shape(), dtype=np.float32)
        check(self._L.psm_forward(self._ctx, _addr(out)), self._err)
        return out

    def forward_host(self, traces, vrms, out=None):
        """Upload, migrate and download in one pipelined call (psm_forward_host): traces and
        vrms are host float32 [n_il][n_xl][n_t] (numpy or pinned CPU tensors)."""
        g = self.geom
        if out is None:
            out = np.empty(self.image_shape(), dtype=np.float32)
        if isinstance(traces, np.ndarray):
            traces = _f32(traces, (g.n_il, g.n_xl, g.n_t))
        if isinstance(vrms, np.ndarray):
            vrms = _f32(vrms, (g.n_il, g.n_xl, g.n_t))
        check(self._L.psm_forward_host(self._ctx, _addr(traces), _addr(vrms), _addr(out)),
              self._err)
        return out

    def forward_async(self) -> None:
        check(self._L.psm_forward_async(self._ctx), self._err)

    def synchronize(self) -> None:
        check(self._L.psm_synchronize(self._ctx), self._err)

    def get_image(self, out=None):
        if out is None:
            out = np.empty(self.image_shape(), dtype=np.float32)
        check(self._L.psm_get_image(self._ctx, _addr(out)), self._err)
        return out

    def image_device_ptr(self) -> int:
        p = ctypes.c_void_p()
        check(self._L.psm_image_device(self._ctx, ctypes.byref(p)), self._err)
        return p.value

    def stream_handle(self) -> int:
        p = ctypes.c_void_p()
        check(self._L.psm_stream(self._ctx, ctypes.byref(p)), self._err)
        return p.value or 0

    def count_terms(self) -> int:
        """Terms that pass every reference mask over the real input traces, all output
        inlines (padded ones included)."""
        n = ctypes.c_int64()
        check(self._L.psm_count_terms(self._ctx, ctypes.byref(n)), self._err)
        return int(n.value)

    def adjoint(self, image, out=None):
        """Adjoint of forward (demigration / spray): data [n_il][n_xl][n_t] = M^T image."""
        g = self.geom
        if isinstance(image, np.ndarray):
            image = _f32(image, self.image_shape())
        if out is None:
            out = np.empty((g.n_il, g.n_xl, g.n_t), dtype=np.float32)
        check(self._L.psm_adjoint(self._ctx, _addr(image), _addr(out)), self._err)
        return out

    def adjoint_async(self) -> None:
        """M^T of the ctx image into the ctx's trace cube, enqueued on the ctx stream
        (psm_adjoint_async); get_traces() reads the result."""
        check(self._L.psm_adjoint_async(self._ctx), self._err)

    def forward_device(self, d_data: int, d_image: int) -> None:
        """image = M data on device memory (addresses of fp32 arrays [n_il][n_xl][n_t] and
        [n_oi][n_ox][n_t], e.g. torch tensors' data_ptr()), enqueued on the ctx stream
        (psm_forward_device); synchronize() waits."""
        check(self._L.psm_forward_device(self._ctx, ctypes.c_void_p(d_data),
                                         ctypes.c_void_p(d_image)), self._err)

    def adjoint_device(self, d_image: int, d_data: int) -> None:
        """data = M^T image on device memory, enqueued on the ctx stream
        (psm_adjoint_device)."""
        check(self._L.psm_adjoint_device(self._ctx, ctypes.c_void_p(d_image),
                                         ctypes.c_void_p(d_data)), self._err)

    def lsm_cg(self, data, iters: int):
        """Least-squares migration: CG on min ||M^T m - data||^2 (FP32 operators, FP64
        inner products on the GPU).  Returns (image, data-residual norms [iters + 1])."""
        g = self.geom
        if isinstance(data, np.ndarray):
            data = _f32(data, (g.n_il, g.n_xl, g.n_t))
        img = np.empty(self.image_shape(), dtype=np.float32)
        hist = np.zeros(iters + 1, dtype=np.float64)
        check(self._L.psm_lsm_cg(self._ctx, _addr(data), img.ctypes.data, int(iters),
                                 hist.ctypes.data), self._err)
        return img, hist

    VARIANTS = {1: "scalar/g2", 2: "scalar/g4", 3: "packed/g2", 4: "packed/g4",
                5: "packed/g4/j16", 6: "scalar/g4/j16", 7: "packed/g8", 8: "scalar/g8",
                9: "packed/g4/o3", 10: "scalar/g4/o3", 11: "pairs/o3", 12: "pairs",
                13: "pairs/j4/o4"}

    def set_variant(self, variant: int) -> None:
        check(self._L.psm_set_variant(self._ctx, int(variant)), self._err)

    def variant(self) -> int:
        v = ctypes.c_int()
        check(self._L.psm_get_variant(self._ctx, ctypes.byref(v)), self._err)
        return v.value

    def autotune(self):
        """Time every forward variant once on the resident cube and keep the fastest.
        Returns (best variant, {variant: ms})."""
        ms = np.zeros(max(self.VARIANTS) + 1, dtype=np.float32)
        best = ctypes.c_int()
        check(self._L.psm_autotune(self._ctx, ms.ctypes.data, ctypes.byref(best)), self._err)
        return best.value, {v: float(ms[v]) for v in self.VARIANTS}

    def count_terms_rows(self) -> np.ndarray:
        out = np.zeros(self.geom.n_oi, dtype=np.int64)
        check(self._L.psm_count_terms_rows(self._ctx, out.ctypes.data), self._err)
        return out

    def count_terms_computed(self) -> int:
        """Terms the forward launch evaluates: count_terms without the padded output inlines
        that repeat an inline already migrated (the forward copies those rows; the reference
        migrates them again, main.cpp:258-288)."""
        rows = self.count_terms_rows()
        _, first = np.unique(np.asarray(self.geom.out_center), return_index=True)
        return int(rows[first].sum())


class Problem:
    """One problem of a batched launch: a cube, its Vrms and its geometry.

    vrms: a [n_il][n_xl][n_t] cube, a [n_t] trace used for every output point, or None with
    velocity set (a constant-velocity scan panel).  Problems given the same traces array
    share one device copy of it."""

    def __init__(self, geom: Geometry, traces, vrms=None, velocity: float = 0.0):
        self.geom = geom
        self.traces = _f32(traces, (geom.n_il, geom.n_xl, geom.n_t))
        if vrms is None:
            if not velocity > 0.0:
                raise ValueError("a constant-velocity problem needs velocity > 0")
            self.vrms, self.kind = None, 2
        else:
            v = _f32(vrms)
            if v.ndim == 1:
                if v.size != geom.n_t:
                    raise ValueError("a Vrms trace has n_t samples")
                self.vrms, self.kind = v, 1
            else:
                self.vrms, self.kind = _f32(v, (geom.n_il, geom.n_xl, geom.n_t)), 0
        self.velocity = float(velocity)
        self.out_center = np.ascontiguousarray(geom.out_center, dtype=np.int32)


class Batch:
    """Several problems (velocity-scan panels over one cube, sub-volumes with their own
    Vrms) migrated by ONE persistent launch replayed as a CUDA graph (include/psm.h,
    psm_batch_*).  The host arrays of the problems are kept referenced: reload() uploads
    them again."""

    PERSISTENT, PER_PROBLEM, ONE_GRID = 0, 1, 2
    DEPTH_FIRST, PROBLEM_ORDER = 0, 1
    ORDERS = {0: "depth-first", 1: "problem"}

    def __init__(self, migrator: "Migrator", problems):
        self._m = migrator
        self._L = migrator._L
        self.problems = list(problems)
        # a traces array shared by several problems must be the same object to share its
        # device copy; _f32 keeps float32 C-contiguous inputs as they are
        arr = (_lib.PsmProblem * len(self.problems))()
        for i, p in enumerate(self.problems):
            arr[i].geom = p.geom.to_c()
            arr[i].out_center = p.out_center.ctypes.data
            arr[i].traces = p.traces.ctypes.data
            arr[i].vrms = p.vrms.ctypes.data if p.vrms is not None else None
            arr[i].vrms_kind = p.kind
            arr[i].velocity = p.velocity
        self._arr = arr
        self._b = ctypes.c_void_p()
        check(self._L.psm_batch_create(migrator._ctx, arr, len(self.problems),
                                       ctypes.byref(self._b)), migrator._err)

    def close(self):
        if self._b:
            self._L.psm_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_mode(self, mode: int) -> None:
        check(self._L.psm_batch_set_mode(self._b, int(mode)), self._m._err)

    def set_variant(self, variant: int) -> None:
        check(self._L.psm_batch_set_variant(self._b, int(variant)), self._m._err)

    def variant(self) -> int:
        v = ctypes.c_int()
        check(self._L.psm_batch_get_variant(self._b, ctypes.byref(v)), self._m._err)
        return v.value

    def set_order(self, order: int) -> None:
        check(self._L.psm_batch_set_order(self._b, int(order)), self._m._err)

    def order(self) -> int:
        o = ctypes.c_int()
        check(self._L.psm_batch_get_order(self._b, ctypes.byref(o)), self._m._err)
        return o.value

    SCHEDULES = {0: "persistent/depth-first", 1: "persistent/problem", 2: "per-problem",
                 3: "one-grid/depth-first", 4: "one-grid/problem"}

    def mode(self) -> int:
        v = ctypes.c_int()
        check(self._L.psm_batch_get_mode(self._b, ctypes.byref(v)), self._m._err)
        return v.value

    def autotune(self):
        """Time every kernel variant on each schedule (SCHEDULES: persistent depth-first /
        problem order, per-problem launches, one grid depth-first / problem order); keep the
        fastest.  Returns (variant, order, mode, {(variant, schedule): ms})."""
        nv = max(Migrator.VARIANTS) + 1
        ms = np.zeros(5 * nv, dtype=np.float32)
        best, order, mode = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._L.psm_batch_autotune(self._b, ms.ctypes.data, ctypes.byref(best),
                                         ctypes.byref(order), ctypes.byref(mode)),
              self._m._err)
        return best.value, order.value, mode.value, {
            (v, sch): float(ms[sch * nv + v]) for sch in range(5) for v in Migrator.VARIANTS
            if ms[sch * nv + v] > 0}

    def reload(self) -> None:
        check(self._L.psm_batch_reload(self._b), self._m._err)

    def run_async(self) -> None:
        check(self._L.psm_batch_run_async(self._b), self._m._err)

    def synchronize(self) -> None:
        check(self._L.psm_batch_synchronize(self._b), self._m._err)

    def run(self) -> None:
        check(self._L.psm_batch_run(self._b), self._m._err)

    def image(self, i: int, out=None) -> np.ndarray:
        g = self.problems[i].geom
        shape = (g.n_oi, g.n_ox, g.n_t)
        if out is None:
            out = np.empty(shape, dtype=np.float32)
        check(self._L.psm_batch_get_image(self._b, int(i), _addr(out)), self._m._err)
        return out

    def image_device_ptr(self, i: int) -> int:
        p = ctypes.c_void_p()
        check(self._L.psm_batch_image_device(self._b, int(i), ctypes.byref(p)), self._m._err)
        return p.value

    def count_terms(self) -> int:
        n = ctypes.c_int64()
        check(self._L.psm_batch_count_terms(self._b, ctypes.byref(n)), self._m._err)
        return n.value


class MigrationKernel:
    """Mirror of the reference's static class MigrationKernel (include/migration_kernel.h)."""

    @staticmethod
    def kirchhoff_kernel_3d_with_padding(input_buffer, n_buf_il, n_buf_xl, n_t,
                                         velocity_slice, output_slice, il_pos_indices,
                                         xl_pos_indices, current_il_pos, current_xl_start,
                                         dt, t0_times, tan_theta_sq, inline_bin_size,
                                         crossline_bin_size, amp_correction):
        """kirchhoffKernel3DWithPadding on the GPU.  output_slice: float32 array
        [n_out_xl][n_t], fully overwritten in place (as the reference overwrites its
        vector<vector<float>>)."""
        L = _lib.cuda()
        buf = _f32(input_buffer).reshape(-1)
        vel = _f32(velocity_slice).reshape(-1)
        if buf.size != n_buf_il * n_buf_xl * n_t:
            raise ValueError("input_buffer size mismatch")
        if vel.size < n_buf_xl * n_t:
            raise ValueError("velocity_slice size mismatch")
        if not (isinstance(output_slice, np.ndarray) and output_slice.dtype == np.float32
                and output_slice.flags["C_CONTIGUOUS"]):
            raise TypeError("output_slice must be a C-contiguous float32 array")
        n_out_xl = output_slice.shape[0] if output_slice.ndim > 1 else (
            output_slice.size // max(n_t, 1))
        ilp = np.ascontiguousarray(il_pos_indices, dtype=np.int32)
        t0 = _f32(t0_times)
        if t0.size < n_t:
            raise ValueError("t0_times shorter than n_t")
        rc = L.psm_kirchhoff_inline(buf.ctypes.data, n_buf_il, n_buf_xl, n_t, vel.ctypes.data,
                                    output_slice.ctypes.data, n_out_xl, ilp.ctypes.data, None,
                                    int(current_il_pos), int(current_xl_start),
                                    np.float32(dt), t0.ctypes.data, np.float32(tan_theta_sq),
                                    np.float32(inline_bin_size),
                                    np.float32(crossline_bin_size), int(bool(amp_correction)))
        check(rc, lambda: L.psm_kirchhoff_inline_error().decode())
        return output_slice
