"""Seeded synthetic post-stack cubes and a small numpy SEG-Y writer/reader.

These stand in for field data: every cube is generated from a fixed seed with the shapes,
sample rates, wavelets and velocity laws the migration workloads are quoted on (point
diffractors, dipping planes, Ricker wavelets, Gaussian noise, constant or linear Vrms with a
lateral Gaussian perturbation).  The SEG-Y layout written here is the one the reference
reads (src/segy_utils.cpp:39-111, 152-214): 3200 B text header, 400 B binary header with
dt@16, ns@20, format@24 (big-endian), 240 B trace headers with INLINE_3D@188 and
CROSSLINE_3D@192, samples as big-endian IEEE (format 5) or IBM (format 1) floats.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional, Sequence

import numpy as np

# --------------------------------------------------------------------------- IBM floats


def ieee_to_ibm_words(x: np.ndarray) -> np.ndarray:
    """IEEE float32 -> IBM System/360 single words (uint32), truncating the fraction.

    IBM single: sign bit, 7-bit base-16 exponent biased by 64, 24-bit fraction in [1/16, 1).
    Zero maps to 0.  Used only to write test inputs; the product's encoder lives in the C++
    host."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros(x.shape, dtype=np.uint32)
    nz = x != 0
    a = np.abs(x[nz])
    e = np.floor(np.log(a) / np.log(16.0)).astype(np.int64) + 1  # a = f * 16**e, f in [1/16,1)
    f = a / np.power(16.0, e)
    # guard the log() rounding at exact powers of 16
    hi = f >= 1.0
    e[hi] += 1
    f[hi] /= 16.0
    lo = f < 1.0 / 16.0
    e[lo] -= 1
    f[lo] *= 16.0
    frac = np.floor(f * 16777216.0).astype(np.uint64) & 0xFFFFFF
    sign = (x[nz] < 0).astype(np.uint64) << 31
    out[nz] = (sign | ((e + 64).astype(np.uint64) << 24) | frac).astype(np.uint32)
    return out


def ibm_words_to_ieee(w: np.ndarray) -> np.ndarray:
    """IBM single words (uint32) -> float32 by the IBM definition, value computed in FP64."""
    w = np.asarray(w, dtype=np.uint32).astype(np.uint64)
    sign = np.where((w >> 31) & 1, -1.0, 1.0)
    expo = ((w >> 24) & 0x7F).astype(np.int64) - 64
    frac = (w & 0xFFFFFF).astype(np.float64) / 16777216.0
    return (sign * np.ldexp(frac, 4 * expo)).astype(np.float32)


# --------------------------------------------------------------------------- SEG-Y


@dataclasses.dataclass
class SegyCube:
    data: np.ndarray  # [n_il][n_xl][n_t] float32
    il_labels: np.ndarray
    xl_labels: np.ndarray
    dt_us: int
    fmt: int


def write_segy(path: str, data: np.ndarray, il_labels: Sequence[int],
               xl_labels: Sequence[int], dt_us: int, fmt: int = 5,
               order: Optional[np.ndarray] = None, text: str = "synthetic",
               skip: Optional[Sequence[tuple]] = None, format_code: Optional[int] = None,
               header_fill: bool = True) -> None:
    """Write data[n_il][n_xl][n_t] as a SEG-Y file.

    order: optional permutation of the n_il*n_xl traces (tests the lookup table on unsorted
    files).  skip: (il_label, xl_label) pairs to leave out (irregular grids).
    format_code: value written at binary-header byte 24 (defaults to fmt); samples are
    encoded as IBM when fmt == 1, IEEE otherwise.  header_fill writes a few standard
    trace-header fields besides INLINE_3D/CROSSLINE_3D so header copying is observable."""
    data = np.asarray(data, dtype=np.float32)
    n_il, n_xl, n_t = data.shape
    il_labels = np.asarray(il_labels, dtype=np.int64)
    xl_labels = np.asarray(xl_labels, dtype=np.int64)
    assert len(il_labels) == n_il and len(xl_labels) == n_xl
    th = bytearray(3200)
    txt = ("C 1 " + text).encode("ascii")[:3200]
    th[: len(txt)] = txt
    bh = bytearray(400)
    bh[12:14] = (1).to_bytes(2, "big")  # traces per ensemble
    bh[16:18] = int(dt_us).to_bytes(2, "big")
    bh[20:22] = int(n_t).to_bytes(2, "big")
    bh[24:26] = int(fmt if format_code is None else format_code).to_bytes(2, "big")
    skip_set = set(tuple(int(v) for v in p) for p in (skip or []))
    ii, xx = np.meshgrid(np.arange(n_il), np.arange(n_xl), indexing="ij")
    ii = ii.ravel()
    xx = xx.ravel()
    if order is not None:
        ii = ii[order]
        xx = xx[order]
    keep = np.array([(int(il_labels[a]), int(xl_labels[b])) not in skip_set
                     for a, b in zip(ii, xx)], dtype=bool)
    ii = ii[keep]
    xx = xx[keep]
    n_tr = len(ii)
    hdr = np.zeros((n_tr, 240), dtype=np.uint8)

    def put32(col, vals):
        v = np.asarray(vals, dtype=">i4").view(np.uint8).reshape(-1, 4)
        hdr[:, col:col + 4] = v

    def put16(col, vals):
        v = np.asarray(vals, dtype=">i2").view(np.uint8).reshape(-1, 2)
        hdr[:, col:col + 2] = v

    put32(188, il_labels[ii])
    put32(192, xl_labels[xx])
    if header_fill:
        put32(0, np.arange(1, n_tr + 1))          # trace sequence number in line
        put32(8, il_labels[ii])                   # field record
        put32(20, np.arange(1, n_tr + 1) + 1000)  # CDP
        put32(180, (xx * 25 + 500000))            # CDP X
        put32(184, (ii * 25 + 6000000))           # CDP Y
        put16(114, np.full(n_tr, n_t))
        put16(116, np.full(n_tr, dt_us))
    traces = data[ii, xx, :]
    if fmt == 1:
        words = ieee_to_ibm_words(traces).astype(">u4")
    else:
        words = traces.astype(">f4")
    body = np.concatenate([hdr, words.view(np.uint8).reshape(n_tr, 4 * n_t)], axis=1)
    with open(path, "wb") as f:
        f.write(bytes(th))
        f.write(bytes(bh))
        f.write(body.tobytes())


def read_segy_raw(path: str):
    """Independent numpy reader: returns (text, binary, headers[n][240] u8, samples words
    [n][n_t] big-endian uint32)."""
    return read_segy_raw_bytes(np.fromfile(path, dtype=np.uint8).tobytes())


def read_segy_raw_bytes(buf: bytes):
    raw = np.frombuffer(buf, dtype=np.uint8)
    text = raw[:3200].tobytes()
    binary = raw[3200:3600].tobytes()
    n_t = int.from_bytes(binary[20:22], "big")
    tr = 240 + 4 * n_t
    n = (len(raw) - 3600) // tr
    body = raw[3600:3600 + n * tr].reshape(n, tr)
    hdrs = body[:, :240]
    words = body[:, 240:].copy().view(">u4").reshape(n, n_t)
    return text, binary, hdrs, words


def decode_samples(words: np.ndarray, fmt: int) -> np.ndarray:
    if fmt == 1:
        return ibm_words_to_ieee(words.astype(np.uint32))
    return words.astype(">u4").view(">f4").astype(np.float32)


def header_i32(hdrs: np.ndarray, col: int) -> np.ndarray:
    return hdrs[:, col:col + 4].copy().view(">i4").ravel().astype(np.int64)


# --------------------------------------------------------------------------- wavelets


def ricker(t: np.ndarray, f: float) -> np.ndarray:
    """Unit-peak Ricker (1 - 2a) e^{-a}, a = (pi f t)^2."""
    a = (np.pi * f * t) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


def _add_event(cube: np.ndarray, t_event: np.ndarray, amp: np.ndarray, f: float, dt: float,
               half_width_s: float) -> None:
    """Add amp * ricker(t - t_event) per trace over a +-half_width window."""
    n_t = cube.shape[-1]
    hw = int(math.ceil(half_width_s / dt))
    flat = cube.reshape(-1, n_t)
    te = t_event.reshape(-1)
    am = np.broadcast_to(amp, te.shape).reshape(-1)
    c = np.rint(te / dt).astype(np.int64)
    for off in range(-hw, hw + 1):
        idx = c + off
        ok = (idx >= 0) & (idx < n_t)
        if not ok.any():
            continue
        rows = np.nonzero(ok)[0]
        tt = idx[ok] * dt - te[ok]
        # each row appears once per offset, so plain fancy-index accumulation is exact
        flat[rows, idx[ok]] += (am[ok] * ricker(tt, f)).astype(np.float32)


# --------------------------------------------------------------------------- workloads


@dataclasses.dataclass
class Workload:
    """A migration job on a regular grid: cube, Vrms cube and the config-file parameters."""
    name: str
    data: np.ndarray            # [n_il][n_xl][n_t] float32
    vrms: Optional[np.ndarray]  # [n_il][n_xl][n_t] float32 or None (constant velocity)
    velocity: float             # constant velocity when vrms is None
    dt: float                   # seconds
    d_il: float
    d_xl: float
    angle: float                # degrees
    amp: bool
    pad_il: int
    pad_xl: int
    il_labels: np.ndarray
    xl_labels: np.ndarray

    @property
    def shape(self):
        return self.data.shape

    def vrms_cube(self) -> np.ndarray:
        if self.vrms is not None:
            return self.vrms
        return np.full(self.data.shape, np.float32(self.velocity), dtype=np.float32)


def write_run(directory: str, W: "Workload", output: str = "out.sgy", fmt: int = 5,
              **extra) -> str:
    """Write workload W as the input of one poststackmig run in `directory`: the traces as a
    SEG-Y file (labels W.il_labels / W.xl_labels, sample format fmt), a Vrms SEG-Y on the same
    grid when W has a Vrms cube (else the constant velocity), and config.txt with the
    reference's keys (src/config_parser.cpp; output_data = directory/output).  extra adds or
    overrides keys (n_threads, ...).  Returns the config path."""
    import os
    dt_us = int(round(W.dt * 1e6))
    inp = os.path.join(directory, "input.sgy")
    write_segy(inp, W.data, W.il_labels, W.xl_labels, dt_us, fmt)
    if W.vrms is not None:
        vel = os.path.join(directory, "vrms.sgy")
        write_segy(vel, W.vrms, W.il_labels, W.xl_labels, dt_us, 5, text="vrms")
    else:
        vel = repr(float(W.velocity))
    kv = dict(input_data=inp, output_data=os.path.join(directory, output),
              inline_step=float(W.d_il), crossline_step=float(W.d_xl), velocity=vel,
              inline_padding=int(W.pad_il), crossline_padding=int(W.pad_xl),
              angle_aperture=float(W.angle), amp_correction=bool(W.amp))
    kv.update(extra)
    cfg = os.path.join(directory, "config.txt")
    with open(cfg, "w") as f:
        for k, v in kv.items():
            f.write(f"{k}={str(v).lower() if isinstance(v, bool) else v}\n")
    return cfg


def diffractor_cube(n_il=101, n_xl=101, n_t=501, dt=0.002, d=25.0, v=2000.0, t_apex=0.5,
                    f=25.0, noise=0.1, seed=1) -> np.ndarray:
    """One point diffractor at the cube centre: unit-peak Ricker placed on
    t = sqrt(t_apex^2 + 4 r^2 / v^2), plus N(0, noise^2)."""
    rng = np.random.default_rng(seed)
    il = (np.arange(n_il) - (n_il - 1) / 2.0) * d
    xl = (np.arange(n_xl) - (n_xl - 1) / 2.0) * d
    r2 = il[:, None] ** 2 + xl[None, :] ** 2
    th = np.sqrt(t_apex ** 2 + 4.0 * r2 / v ** 2)
    t = np.arange(n_t) * dt
    cube = ricker(t[None, None, :] - th[:, :, None], f).astype(np.float32)
    if noise > 0:
        cube += rng.normal(0.0, noise, size=cube.shape).astype(np.float32)
    return cube


def workload_config1(seed: int = 1, n: int = 101, n_t: int = 501, pad: int = 30) -> Workload:
    """Plain FP32 migration, CPU-runnable: 101x101 traces, 501 samples at 2 ms, 25 m bins,
    one diffractor at t0 = 0.5 s, V = 2000 m/s, 30 deg, amp on, padding 30 each side."""
    data = diffractor_cube(n, n, n_t, 0.002, 25.0, 2000.0, 0.5, 25.0, 0.1, seed)
    return Workload("config1", data, None, 2000.0, 0.002, 25.0, 25.0, 30.0, True, pad, pad,
                    np.arange(1, n + 1), np.arange(1, n + 1))


def linear_vrms(n_il, n_xl, n_t, dt, d, v0=1500.0, v1=3500.0, lateral=0.05,
                sigma=2000.0) -> np.ndarray:
    """Vrms(t) rising linearly v0 -> v1 over the record, times (1 + lateral * G(x, y)) with
    G a unit Gaussian bump of width sigma (m) at the cube centre."""
    t = np.arange(n_t) * dt
    vt = v0 + (v1 - v0) * t / max(t[-1], dt)
    il = (np.arange(n_il) - (n_il - 1) / 2.0) * d
    xl = (np.arange(n_xl) - (n_xl - 1) / 2.0) * d
    g = np.exp(-(il[:, None] ** 2 + xl[None, :] ** 2) / (2.0 * sigma ** 2))
    return ((1.0 + lateral * g)[:, :, None] * vt[None, None, :]).astype(np.float32)


def reflectivity_cube(vrms: np.ndarray, dt: float, d: float, n_diff: int, n_planes: int,
                      f: float, noise_frac: float, seed: int,
                      max_dip_deg: float = 30.0) -> np.ndarray:
    """Seeded point diffractors + dipping planes (+-1 amplitudes) with a Ricker of peak
    frequency f, modelled with t = sqrt(t0^2 + 4 r^2 / v^2) (v = Vrms at the scatterer),
    plus Gaussian noise at noise_frac of the peak amplitude."""
    rng = np.random.default_rng(seed)
    n_il, n_xl, n_t = vrms.shape
    cube = np.zeros((n_il, n_xl, n_t), dtype=np.float32)
    il = np.arange(n_il) * d
    xl = np.arange(n_xl) * d
    t_max = (n_t - 1) * dt
    for _ in range(n_diff):
        ci = rng.uniform(0.1, 0.9) * il[-1]
        cx = rng.uniform(0.1, 0.9) * xl[-1]
        t0 = rng.uniform(0.15, 0.85) * t_max
        a = rng.choice([-1.0, 1.0]) * rng.uniform(0.5, 1.0)
        iv = min(int(ci / d), n_il - 1)
        xv = min(int(cx / d), n_xl - 1)
        v = float(vrms[iv, xv, min(int(t0 / dt), n_t - 1)])
        r2 = (il[:, None] - ci) ** 2 + (xl[None, :] - cx) ** 2
        th = np.sqrt(t0 ** 2 + 4.0 * r2 / v ** 2)
        _add_event(cube, th, np.float32(a), f, dt, 1.5 / f)
    for _ in range(n_planes):
        t0 = rng.uniform(0.2, 0.8) * t_max
        dip = np.deg2rad(rng.uniform(0.0, max_dip_deg))
        az = rng.uniform(0.0, 2.0 * np.pi)
        a = rng.choice([-1.0, 1.0])
        vm = float(vrms.mean())
        slope = 2.0 * np.sin(dip) / vm  # s/m, zero-offset time dip
        x = il[:, None] - il[-1] / 2.0
        y = xl[None, :] - xl[-1] / 2.0
        tp = t0 + slope * (np.cos(az) * x + np.sin(az) * y)
        _add_event(cube, tp, np.float32(a), f, dt, 1.5 / f)
    peak = float(np.abs(cube).max()) or 1.0
    if noise_frac > 0:
        cube += rng.normal(0.0, noise_frac * peak, size=cube.shape).astype(np.float32)
    return cube


def workload_config2(seed: int = 2, n: int = 401, n_t: int = 1001,
                     n_diff: int = 60, n_planes: int = 5) -> Workload:
    """Production size: 401x401 traces, 1001 samples at 2 ms, 25 m bins, Vrms 1500->3500 m/s
    with a 5% lateral Gaussian bump (sigma 2 km), 60 diffractors + 5 dipping planes, 30 Hz
    Ricker, 5% noise, 45 deg aperture, amp on, no padding."""
    vrms = linear_vrms(n, n, n_t, 0.002, 25.0)
    data = reflectivity_cube(vrms, 0.002, 25.0, n_diff, n_planes, 30.0, 0.05, seed)
    return Workload("config2", data, vrms, 0.0, 0.002, 25.0, 25.0, 45.0, True, 0, 0,
                    np.arange(1, n + 1), np.arange(1, n + 1))


def random_workload(seed: int, n_il: int, n_xl: int, n_t: int, *, dt=0.004, d_il=25.0,
                    d_xl=20.0, angle=35.0, amp=True, pad_il=0, pad_xl=0,
                    vel_kind="linear") -> Workload:
    """Small seeded case for parity tests: random reflectivity traces and a Vrms cube that
    is constant, linear in time, or laterally varying."""
    rng = np.random.default_rng(seed)
    data = rng.standard_normal((n_il, n_xl, n_t)).astype(np.float32)
    t = np.arange(n_t) * dt
    if vel_kind == "const":
        vr = None
        vel = 2200.0
    else:
        vt = 1600.0 + 900.0 * t / max(t[-1], dt)
        vr = np.broadcast_to(vt, (n_il, n_xl, n_t)).astype(np.float32).copy()
        if vel_kind == "lateral":
            vr *= (1.0 + 0.1 * rng.random((n_il, n_xl, 1))).astype(np.float32)
        vel = 0.0
    return Workload(f"random{seed}", data, vr, vel, dt, d_il, d_xl, angle, amp, pad_il,
                    pad_xl, np.arange(10, 10 + n_il), np.arange(100, 100 + 2 * n_xl, 2))


def workload_config4(seed: int = 4, n: int = 201, n_t: int = 751, n_panels: int = 32,
                     n_sub: int = 8):
    """Batched form: n_panels constant-velocity scan panels 1800 + 50 k m/s (k < 32, so
    1800..3350) over one n x n x n_t cube (2 ms, 25 m bins, 20 diffractors + 3 dipping planes
    modelled with Vrms 1800 -> 3400 m/s, 25 Hz Ricker, 5% noise), 30 deg aperture, amp on;
    plus n_sub sub-volumes of 64-256 traces per axis and 401-1001 samples, each with its own
    linear Vrms(t) (10 diffractors + 1 plane, 25 Hz, 5% noise).

    Returns (panels, subvolumes): panels is a list of Workloads sharing one data array (the
    velocity field differs), subvolumes a list of Workloads with Vrms cubes."""
    vmod = linear_vrms(n, n, n_t, 0.002, 25.0, 1800.0, 3400.0, lateral=0.0)
    data = reflectivity_cube(vmod, 0.002, 25.0, 20, 3, 25.0, 0.05, seed)
    labels = np.arange(1, n + 1)
    panels = [Workload(f"config4_panel{k}", data, None, 1800.0 + 50.0 * k, 0.002, 25.0, 25.0,
                       30.0, True, 0, 0, labels, labels) for k in range(n_panels)]
    rng = np.random.default_rng(seed + 1000)
    subs = []
    for k in range(n_sub):
        ni, nx = (int(v) for v in rng.integers(64, 257, 2))
        nt = int(rng.integers(401, 1002))
        v0 = float(rng.uniform(1500.0, 2000.0))
        v1 = float(rng.uniform(2500.0, 3500.0))
        vr = linear_vrms(ni, nx, nt, 0.002, 25.0, v0, v1, lateral=0.0)
        d = reflectivity_cube(vr, 0.002, 25.0, 10, 1, 25.0, 0.05, seed + 1 + k)
        subs.append(Workload(f"config4_sub{k}", d, vr, 0.0, 0.002, 25.0, 25.0, 30.0, True, 0,
                             0, np.arange(1, ni + 1), np.arange(1, nx + 1)))
    return panels, subs
