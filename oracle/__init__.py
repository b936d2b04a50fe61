"""TEST INFRASTRUCTURE ONLY: the CPU checker for the Kirchhoff summation path.

Python access to liboracle.so (our C restatement, oracle.c) and, when it has been built,
to the reference's own code compiled from its sources into oracle/_ref/.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import this package, and only to
check or time against; the product (poststackmig3d_b200) never imports it.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

CONTRACT = 1
F64 = 2
AVX_ORDER = 4

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")

_lib = None
_ref = {}


def build(reference: Optional[str] = None) -> None:
    """Compile liboracle.so, and the reference into _ref/ from its source tree: `reference`,
    else the PSM_REFERENCE_SRC environment variable (skipped when neither names a tree with
    src/)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    ref = reference or os.environ.get("PSM_REFERENCE_SRC")
    if ref and os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = ctypes.CDLL(path)
        L.oracle_kirchhoff_inline.restype = ctypes.c_int64
        L.oracle_kirchhoff_inline.argtypes = [
            _f32p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, _f32p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, _i32p, ctypes.c_int32,
            ctypes.c_int32, ctypes.c_float, _f32p, ctypes.c_float, ctypes.c_float,
            ctypes.c_float, ctypes.c_int, ctypes.c_int]
        L.oracle_migrate_volume.restype = None
        L.oracle_migrate_volume.argtypes = [
            _f32p, _f32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _i32p,
            ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
            ctypes.c_float, _f32p, ctypes.c_float, ctypes.c_float, ctypes.c_float,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
            _i64p]
        L.oracle_count_rows.restype = None
        L.oracle_count_rows.argtypes = [
            _f32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _i32p, ctypes.c_int32,
            ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
            ctypes.c_float, _f32p, ctypes.c_float, ctypes.c_float, ctypes.c_float,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64p]
        L.oracle_adjoint_volume.restype = None
        L.oracle_adjoint_volume.argtypes = [
            _f64p, _f32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _i32p,
            ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
            ctypes.c_float, _f32p, ctypes.c_float, ctypes.c_float, ctypes.c_float,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


# ----------------------------------------------------------------- driver-level geometry
# Restatements of src/main.cpp; they return plain numbers for the oracle's arguments.


def t0_times(n_t: int, dt_seconds: float) -> np.ndarray:
    """main.cpp:214-217: t0[i] = float(i * dt) with dt in double."""
    return np.array([np.float32(i * dt_seconds) for i in range(n_t)], dtype=np.float32)


def tan2_theta(angle_deg: float) -> np.float32:
    """main.cpp:188-189: float(tan(angle*pi/180)) squared in float."""
    t = np.float32(math.tan(angle_deg * math.pi / 180.0))
    return np.float32(t * t)


def max_aperture_il(max_v: float, n_t: int, dt_seconds: float, tan2: np.float32,
                    inline_step: float) -> int:
    """main.cpp:197-201."""
    max_t = (n_t - 1) * dt_seconds
    rad = np.float32(np.float32(np.float32(max_v) * np.float32(max_t)) / np.float32(2.0))
    rad = np.float32(rad * np.float32(np.sqrt(np.float32(tan2))))
    return int(float(rad) / inline_step) + 1


def output_centers(n_il: int, pad_il: int) -> np.ndarray:
    """Regular-label case of main.cpp:258-288: padded output inlines take the nearest real
    inline."""
    if pad_il > 0 and n_il > 1:
        o = np.arange(n_il + 2 * pad_il) - pad_il
    else:
        o = np.arange(n_il)
    return np.clip(o, 0, n_il - 1).astype(np.int32)


def migrate_volume(data, vrms, out_center, n_ox, pad_il, pad_xl, m_il, dt, t0, tan2, d_il,
                   d_xl, amp=True, flags=CONTRACT | AVX_ORDER, threads=0, want64=False):
    """Run oracle_migrate_volume; returns (image f32, image f64 or None, counts[2])."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    vrms = np.ascontiguousarray(vrms, dtype=np.float32)
    n_il, n_xl, n_t = data.shape
    out_center = np.ascontiguousarray(out_center, dtype=np.int32)
    n_oi = len(out_center)
    out = np.empty((n_oi, n_ox, n_t), dtype=np.float32)
    out64 = np.empty((n_oi, n_ox, n_t), dtype=np.float64) if want64 else None
    counts = np.zeros(2, dtype=np.int64)
    lib().oracle_migrate_volume(data, vrms, n_il, n_xl, n_t, out_center, n_oi, n_ox,
                                pad_il, pad_xl, m_il, np.float32(dt),
                                np.ascontiguousarray(t0, dtype=np.float32), np.float32(tan2),
                                np.float32(d_il), np.float32(d_xl), int(bool(amp)), flags,
                                threads, _ptr(out), _ptr(out64), counts)
    return out, out64, counts


def count_rows(vrms, out_center, r0, r1, n_ox, pad_il, pad_xl, m_il, dt, t0, tan2, d_il,
               d_xl, amp=True, flags=CONTRACT, threads=0):
    """Real-trace term counts of output rows [r0, r1)."""
    vrms = np.ascontiguousarray(vrms, dtype=np.float32)
    n_il, n_xl, n_t = vrms.shape
    out = np.zeros(r1 - r0, dtype=np.int64)
    lib().oracle_count_rows(vrms, n_il, n_xl, n_t,
                            np.ascontiguousarray(out_center, dtype=np.int32), r0, r1, n_ox,
                            pad_il, pad_xl, m_il, np.float32(dt),
                            np.ascontiguousarray(t0, dtype=np.float32), np.float32(tan2),
                            np.float32(d_il), np.float32(d_xl), int(bool(amp)), flags,
                            threads, out)
    return out


def adjoint_volume(image64, vrms, n_il, n_xl, out_center, pad_il, pad_xl, m_il, dt, t0,
                   tan2, d_il, d_xl, amp=True, flags=CONTRACT, threads=0):
    image64 = np.ascontiguousarray(image64, dtype=np.float64)
    n_oi, n_ox, n_t = image64.shape
    out = np.zeros((n_il, n_xl, n_t), dtype=np.float64)
    lib().oracle_adjoint_volume(image64, np.ascontiguousarray(vrms, dtype=np.float32), n_il,
                                n_xl, n_t, np.ascontiguousarray(out_center, dtype=np.int32),
                                n_oi, n_ox, pad_il, pad_xl, m_il, np.float32(dt),
                                np.ascontiguousarray(t0, dtype=np.float32), np.float32(tan2),
                                np.float32(d_il), np.float32(d_xl), int(bool(amp)), flags,
                                threads, out)
    return out


def kirchhoff_inline(buf, vel, n_out_xl, il_pos, cur_il_pos, cur_xl_start, dt, t0, tan2,
                     d_il, d_xl, amp=True, flags=CONTRACT | AVX_ORDER, want64=False):
    buf = np.ascontiguousarray(buf, dtype=np.float32)
    n_buf_il, n_buf_xl, n_t = buf.shape
    out = np.empty((n_out_xl, n_t), dtype=np.float32)
    out64 = np.empty((n_out_xl, n_t), dtype=np.float64) if want64 else None
    n = lib().oracle_kirchhoff_inline(
        buf, n_buf_il, n_buf_xl, n_t, np.ascontiguousarray(vel, dtype=np.float32),
        _ptr(out), _ptr(out64), n_out_xl, np.ascontiguousarray(il_pos, dtype=np.int32),
        cur_il_pos, cur_xl_start, np.float32(dt), np.ascontiguousarray(t0, dtype=np.float32),
        np.float32(tan2), np.float32(d_il), np.float32(d_xl), int(bool(amp)), flags)
    return out, out64, n


def dequantized(data, precision):
    """The fp32 samples that 16-bit storage represents: per trace scale = max |d| (1 for an
    all-zero trace), q = round-to-nearest-even(d / scale) in bf16 or fp16, d' = q * scale
    (fp32 product).  Mirrors the device quantisation so the FP64 oracle can be fed the same
    operator input."""
    d = np.ascontiguousarray(data, dtype=np.float32)
    m = np.abs(d).max(axis=-1, keepdims=True)
    scale = np.where(m > 0, m, np.float32(1.0)).astype(np.float32)
    x = (d / scale).astype(np.float32)
    if precision == "bf16":
        u = x.view(np.uint32).astype(np.uint64)
        u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
        q = u.astype(np.uint32).view(np.float32)
    elif precision == "f16":
        q = x.astype(np.float16).astype(np.float32)
    else:
        raise ValueError(precision)
    return (q * scale).astype(np.float32)


# ----------------------------------------------------------------- the reference itself


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_serial.so"))


def ref_lib(kind: str = "serial"):
    if kind not in _ref:
        L = ctypes.CDLL(os.path.join(REF_DIR, f"libref_{kind}.so"))
        L.ref_kirchhoff_inline.restype = None
        L.ref_kirchhoff_inline.argtypes = [
            _f32p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, _f32p, _f32p,
            ctypes.c_size_t, _i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, _f32p,
            ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int]
        L.ref_velocity_cube.restype = ctypes.c_int
        L.ref_velocity_cube.argtypes = [ctypes.c_char_p, _i32p, ctypes.c_int, _i32p,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_double, _f32p]
        L.ref_velocity_point.restype = ctypes.c_int
        L.ref_velocity_point.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32,
                                         ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_float)]
        L.ref_ibm_to_ieee.restype = ctypes.c_float
        L.ref_ibm_to_ieee.argtypes = [ctypes.c_uint32]
        L.ref_ieee_to_ibm.restype = ctypes.c_uint32
        L.ref_ieee_to_ibm.argtypes = [ctypes.c_float]
        _ref[kind] = L
    return _ref[kind]


def ref_binary(kind: str = "omp") -> str:
    return os.path.join(REF_DIR, f"poststackmig_{kind}")


def ref_kirchhoff_inline(buf, vel, n_out_xl, il_pos, cur_il_pos, cur_xl_start, dt, t0, tan2,
                         d_il, d_xl, amp=True, kind="serial"):
    buf = np.ascontiguousarray(buf, dtype=np.float32)
    n_buf_il, n_buf_xl, n_t = buf.shape
    out = np.empty((n_out_xl, n_t), dtype=np.float32)
    ref_lib(kind).ref_kirchhoff_inline(
        buf, n_buf_il, n_buf_xl, n_t, np.ascontiguousarray(vel, dtype=np.float32), out,
        n_out_xl, np.ascontiguousarray(il_pos, dtype=np.int32), cur_il_pos, cur_xl_start,
        np.float32(dt), np.ascontiguousarray(t0, dtype=np.float32), np.float32(tan2),
        np.float32(d_il), np.float32(d_xl), int(bool(amp)))
    return out


def reference_rows(data, vrms, out_center, rows, n_ox, pad_il, pad_xl, m_il, dt, t0, tan2,
                   d_il, d_xl, amp=True, kind="omp"):
    """Output rows `rows` of the whole-volume migration computed by the reference's own
    kirchhoffKernel3DWithPadding (libref_<kind>.so), each with the buffers its driver
    prepares: input inlines [c - m_il - pad_il, c + m_il + 1 + pad_il) clamped to the cube,
    crosslines padded with zero traces (prepareInputBufferWithPadding,
    src/migration_kernel.cpp:385-468), the centre inline's Vrms with v = 0 on padded
    crosslines (prepareVelocitySliceWithPadding, :470-511).  data and vrms [n_il][n_xl][n_t].
    Returns (image rows [len(rows)][n_ox][n_t] float32, seconds spent in the kernel)."""
    import time
    n_il, n_xl, n_t = data.shape
    out = np.empty((len(rows), n_ox, n_t), dtype=np.float32)
    secs = 0.0
    for k, r in enumerate(rows):
        c = int(out_center[r])
        rs, re = max(0, c - m_il), min(n_il, c + m_il + 1)
        il0, il1 = max(0, rs - pad_il), min(n_il, re + pad_il)
        nbx = n_xl + 2 * pad_xl
        if pad_xl:
            buf = np.zeros((il1 - il0, nbx, n_t), dtype=np.float32)
            buf[:, pad_xl:pad_xl + n_xl] = data[il0:il1]
            vel = np.zeros((nbx, n_t), dtype=np.float32)
            vel[pad_xl:pad_xl + n_xl] = vrms[c]
        else:
            buf = data[il0:il1]
            vel = vrms[c]
        il_pos = np.arange(il0, il1, dtype=np.int32)
        t = time.perf_counter()
        out[k] = ref_kirchhoff_inline(buf, vel, n_ox, il_pos, c - il0, 0, np.float32(dt), t0,
                                      np.float32(tan2), d_il, d_xl, amp, kind=kind)
        secs += time.perf_counter() - t
    return out, secs


def reference_rows_threaded(data, vrms, out_center, rows, n_ox, pad_il, pad_xl, m_il, dt, t0,
                            tan2, d_il, d_xl, amp=True, threads=1, xl_block=16):
    """reference_rows with the work spread over `threads` host threads the way the
    reference's driver spreads it (src/main.cpp:254-256): every thread runs the kernel alone on
    a piece of work it takes when it is free.  A piece here is one output inline's block of
    `xl_block` output crosslines, given to the reference's serial build as current_xl_start
    and a shorter output slice; the kernel computes every output crossline on its own
    (src/migration_kernel.cpp:75-375), so the rows equal the whole-inline calls.  (The
    kernel's own OpenMP loop splits one inline's crosslines statically, and the crosslines
    near the cube's edges hold fewer terms, which leaves threads idle.)  Returns (image rows
    [len(rows)][n_ox][n_t] float32, wall seconds of the kernel calls)."""
    import time
    from concurrent.futures import ThreadPoolExecutor
    n_il, n_xl, n_t = data.shape
    L = ref_lib("serial")
    out = np.zeros((len(rows), n_ox, n_t), dtype=np.float32)
    t0 = np.ascontiguousarray(t0, dtype=np.float32)
    jobs = []
    for r in rows:  # the buffers the driver prepares (reference_rows), outside the timing
        c = int(out_center[r])
        rs, re = max(0, c - m_il), min(n_il, c + m_il + 1)
        il0, il1 = max(0, rs - pad_il), min(n_il, re + pad_il)
        nbx = n_xl + 2 * pad_xl
        if pad_xl:
            buf = np.zeros((il1 - il0, nbx, n_t), dtype=np.float32)
            buf[:, pad_xl:pad_xl + n_xl] = data[il0:il1]
            vel = np.zeros((nbx, n_t), dtype=np.float32)
            vel[pad_xl:pad_xl + n_xl] = vrms[c]
        else:
            buf = np.ascontiguousarray(data[il0:il1], dtype=np.float32)
            vel = np.ascontiguousarray(vrms[c], dtype=np.float32)
        jobs.append((buf, vel, np.arange(il0, il1, dtype=np.int32), c - il0))
    units = [(k, x0, min(xl_block, n_ox - x0)) for x0 in range(0, n_ox, xl_block)
             for k in range(len(rows))]

    def run(u):
        k, x0, nb = u
        buf, vel, il_pos, cur = jobs[k]
        L.ref_kirchhoff_inline(buf, buf.shape[0], buf.shape[1], n_t, vel, out[k, x0:x0 + nb],
                               nb, il_pos, cur, x0, np.float32(dt), t0, np.float32(tan2),
                               np.float32(d_il), np.float32(d_xl), int(bool(amp)))

    with ThreadPoolExecutor(max_workers=max(1, int(threads))) as ex:
        t = time.perf_counter()
        list(ex.map(run, units))
        secs = time.perf_counter() - t
    return out, secs


def write_config(path: str, **kv) -> None:
    with open(path, "w") as f:
        for k, v in kv.items():
            if isinstance(v, bool):
                v = "true" if v else "false"
            f.write(f"{k}={v}\n")


def run_ref_binary(config_path: str, kind: str = "omp", threads: Optional[int] = None,
                   timeout: float = 3600.0) -> subprocess.CompletedProcess:
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    return subprocess.run([ref_binary(kind), config_path], capture_output=True, text=True,
                          env=env, timeout=timeout)
