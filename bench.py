#!/usr/bin/env python
"""Benchmark of the B200 Kirchhoff post-stack 3D time migration.

One step = one forward migration (diffraction summation) of the whole resident cube of the
production workload: 401x401 traces x 1001 samples at 2 ms, 25 m bins, Vrms 1500->3500 m/s
with a 5% lateral Gaussian perturbation, 45 deg aperture, amplitude correction on (seeded
synthetic data, poststackmig3d_b200.synth.workload_config2).

metric: summed input samples/s (G/s) = (output sample, input trace) terms that pass every
mask of the reference, counted exactly by psm_count_terms, per second.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

--impl reference times the reference's own CPU implementation of the path
(MigrationKernel::kirchhoffKernel3DWithPadding compiled from its sources into oracle/_ref,
on all host cores, each running the kernel alone on blocks of output crosslines as the
reference's driver runs it on inlines) on a bounded sample of output inlines of the same
workload.
Multi-GPU (torchrun): independent replicas, one per GPU, no collective on the data path
(weak scaling); value = all ranks' terms / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import dataclasses
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("summed input samples/s (G/s) on 1 B200, mixed/batched vs plain FP32 at stated "
          "rel err")
UNIT = "G/s"
# Algorithmic needs of one term (an output sample and an input trace that pass the masks) on
# the SM limbs: one load of the staged sample pair (both interpolation operands: 8 bytes in
# fp32 storage, 4 in 16-bit storage), one rsqrt (travel time and weight; mirrored pairs share
# it between two traces, so half), and the fp32 lane operations of t^2, s, floor, frac, the
# interpolation and the weighted accumulate (7; 4.5 with pairs, which add the two traces'
# samples and interpolate once).  Peak terms/s = min over limbs of (measured rate per clock
# per SM / need per term) x SMs x SM clock; the limbs come from psm_measure_limbs.
FP32_OPS_PER_TERM = {False: 7.0, True: 4.5}
N_SM = 148


def limb_roofline(limbs, sm_mhz, achieved_gterms, paired, elem_bytes):
    """Roofline of the summation over the measured limbs: {bound, peak (Gterm/s), per-limb
    peaks and needs}."""
    n_sm = int(limbs.get("n_sm") or N_SM)
    per = {
        "lds": (limbs["lds64_bytes_per_clk_sm"], float(elem_bytes), "B"),
        "mufu": (limbs["rsqrt_per_clk_sm"], 0.5 if paired else 1.0, "rsqrt"),
        "fp32": (max(limbs["ffma_per_clk_sm"], limbs["ffma2_per_clk_sm"]),
                 FP32_OPS_PER_TERM[bool(paired)], "lane-ops"),
    }
    peaks = {}
    for k, (rate, need, unit) in per.items():
        tpc = rate / need  # terms per clock per SM
        peaks[k] = {"rate_per_clk_sm": rate, "need_per_term": need, "unit": unit,
                    "terms_per_clk_sm": tpc,
                    "peak_gterms": tpc * n_sm * sm_mhz * 1e6 / 1e9}
    bound = min(peaks, key=lambda k: peaks[k]["peak_gterms"])
    peak = peaks[bound]["peak_gterms"]
    for k in peaks:
        peaks[k]["frac"] = achieved_gterms / peaks[k]["peak_gterms"]
    return bound, peak, peaks


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload",
                   choices=["config2", "config2_201", "config1", "config4", "config5",
                            "config2_io"],
                   default="config2",
                   help="config4 runs the batched form (32 velocity panels + 8 sub-volumes in "
                        "one persistent launch); config5 least-squares migration; config2_io "
                        "the GPU SEG-Y codec, GPU Vrms assembly and slab streaming on config 2")
    p.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    p.add_argument("--shard", action="store_true",
                   help="N>1: one migration split over the ranks in slabs of output inlines "
                        "(each rank holds its slab's input inlines; strong scaling) instead "
                        "of N replicas of the whole migration (weak scaling)")
    p.add_argument("--variant", type=int, default=0,
                   help="forward kernel variant (0: autotune)")
    p.add_argument("--cpu-rows", type=int, default=2,
                   help="output inlines in the bounded CPU sample")
    p.add_argument("--no-cpu-baseline", action="store_true",
                   help="skip the CPU legs (reference kernel sample, parity rows, binaries)")
    p.add_argument("--no-binary-baseline", action="store_true",
                   help="skip the whole-binary config-1 timings")
    p.add_argument("--storage", choices=["f32", "bf16", "f16"], default="f32",
                   help="trace storage in HBM (16-bit: per-trace fp32 scale, fp32 sums)")
    p.add_argument("--compensated", action="store_true",
                   help="compensated (Kahan) summation over the aperture")
    p.add_argument("--panels", type=int, default=32, help="config4: velocity panels")
    p.add_argument("--subvolumes", type=int, default=8, help="config4: sub-volumes")
    p.add_argument("--order", type=int, default=-1,
                   help="config4 tile order (0 depth-first, 1 problem; -1: autotune)")
    return p.parse_args()


def workload(name):
    from poststackmig3d_b200 import synth as S
    if name == "config2":
        return S.workload_config2()
    if name == "config2_201":  # same recipe on 201x201 traces: the profiling case
        return S.workload_config2(n=201)
    return S.workload_config1()


def geometry(W):
    from poststackmig3d_b200 import estimate_max_velocity, plan_geometry
    n_il, n_xl, n_t = W.data.shape
    return plan_geometry(n_il, n_xl, n_t, W.dt, W.d_il, W.d_xl, W.angle,
                         estimate_max_velocity(W.vrms_cube()), W.pad_il, W.pad_xl, W.amp)


def config_dict(W, g, extra=None):
    d = {"workload": f"{W.name}: {g.n_il}x{g.n_xl} traces x {g.n_t} samples, "
                     f"dt {g.dt_seconds * 1e3:.0f} ms, {W.d_il:.0f} m bins, "
                     f"{W.angle:.0f} deg aperture, amp {'on' if W.amp else 'off'}, "
                     f"pad {W.pad_il}/{W.pad_xl}",
         "traces": [g.n_il, g.n_xl], "samples": g.n_t, "image": [g.n_oi, g.n_ox, g.n_t],
         "m_il": g.m_il, "storage": g.precision, "compensated": bool(g.compensated),
         "l2": "inputs larger than L2 (cube 644 MB, Vrms 644 MB)"}
    if extra:
        d.update(extra)
    return d


# --------------------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock, power and throttle reasons."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str):
        self.rows = []
        self.proc = None
        self.t = None
        self.device_id = device_id

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", self.device_id], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.t:
            self.t.join(timeout=5)

    def summary(self):
        sm = []
        mx = []
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
            except ValueError:
                continue
            for n, v in zip(names, r[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def profile_traffic():
    """DRAM bytes per forward launch from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "fwd_kernel_config2_201.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":")[1].split()[0])
            except (IndexError, ValueError):
                return None
    return None


# --------------------------------------------------------------------------- CPU arm


def cpu_reference_sample(W, g, rows, threads):
    """Time the reference's own kirchhoffKernel3DWithPadding (oracle/_ref) on output inlines
    `rows`, with the buffers its driver would prepare (prepareInputBufferWithPadding /
    prepareVelocitySliceWithPadding), on all host threads the way its driver uses them
    (src/main.cpp:254-256: each thread runs the kernel alone on the next piece of work), a
    piece being one inline's block of 16 output crosslines (oracle.reference_rows_threaded).
    Falls back to the oracle port when the reference was not built.  Returns (terms,
    seconds, kind, rows of the image)."""
    import oracle as O
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    t0 = g.t0()
    vr = W.vrms_cube()
    kind = "reference" if O.ref_available() else "port"
    cnt = O.count_rows(vr, g.out_center, 0, g.n_oi, g.n_ox, g.pad_il, g.pad_xl, g.m_il,
                       np.float32(g.dt_seconds), t0, np.float32(g.tan2), g.d_il, g.d_xl,
                       g.amp, threads=threads) if len(rows) > 8 else None
    terms = 0
    for r in rows:
        terms += int(cnt[r]) if cnt is not None else int(O.count_rows(
            vr, g.out_center, r, r + 1, g.n_ox, g.pad_il, g.pad_xl, g.m_il,
            np.float32(g.dt_seconds), t0, np.float32(g.tan2), g.d_il, g.d_xl, g.amp,
            threads=threads)[0])
    if kind == "reference":
        out, secs = O.reference_rows_threaded(W.data, vr, g.out_center, rows, g.n_ox,
                                              g.pad_il, g.pad_xl, g.m_il, g.dt_seconds, t0,
                                              g.tan2, g.d_il, g.d_xl, g.amp, threads=threads,
                                              xl_block=16)
    else:
        out = np.empty((len(rows), g.n_ox, g.n_t), dtype=np.float32)
        secs = 0.0
        for k, r in enumerate(rows):
            sub = np.ascontiguousarray(g.out_center[r:r + 1])
            t = time.perf_counter()
            out[k] = O.migrate_volume(W.data, vr, sub, g.n_ox, g.pad_il, g.pad_xl, g.m_il,
                                      np.float32(g.dt_seconds), t0, np.float32(g.tan2),
                                      g.d_il, g.d_xl, g.amp, threads=threads)[0][0]
            secs += time.perf_counter() - t
    return terms, secs, kind, out


def _err(a, b):
    """Relative RMS error of a against b, and max error relative to b's peak."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = float(np.sqrt(np.mean(b * b))) or 1.0
    return {"rel_rms": float(np.sqrt(np.mean((a - b) ** 2)) / den),
            "max_rel": float(np.abs(a - b).max() / (np.abs(b).max() or 1.0))}


def parity_block(W, g, image, rows, ref_rows, threads):
    """Error of the GPU image on output rows `rows` against the reference's own kernel
    (ref_rows, FP32) and against the FP64 oracle of the same operator (fed the dequantised
    samples for 16-bit storage): relative RMS and max error over the rows, max relative to the
    peak of the rows."""
    import oracle as O

    err = _err
    got = image[rows]
    data = W.data if g.precision == "f32" else O.dequantized(W.data, g.precision)
    sub = np.ascontiguousarray(g.out_center[rows])
    t = time.perf_counter()
    r32, r64, _ = O.migrate_volume(data, W.vrms_cube(), sub, g.n_ox, g.pad_il, g.pad_xl,
                                   g.m_il, np.float32(g.dt_seconds), g.t0(),
                                   np.float32(g.tan2), g.d_il, g.d_xl, g.amp,
                                   O.CONTRACT | O.F64, threads, True)
    out = {"rows": [int(r) for r in rows],
           "vs_fp64": err(got, r64),
           "reference_fp32_vs_fp64": err(ref_rows, r64) if ref_rows is not None else None,
           "vs_reference": err(got, ref_rows) if ref_rows is not None else None,
           "reference": "kirchhoffKernel3DWithPadding compiled from the reference's sources "
                        "(oracle/_ref, serial build on every host thread), same rows and "
                        "buffers",
           "fp64": "FP64 oracle of the same operator (oracle/oracle.c, masks in the "
                   "reference's FP32 arithmetic)" + (", fed the dequantised samples"
                                                    if g.precision != "f32" else ""),
           "oracle_s": time.perf_counter() - t}
    return out


def binary_baseline(threads):
    """Whole-program wall time on config 1 (101x101x501, pad 30/30): the reference's OpenMP
    binary (oracle/_ref/poststackmig_omp, compiled from its sources) with n_threads = all host
    threads and with n_threads = 1 (src/main.cpp:94-97, :423-430), and this repository's
    poststackmig binary on the same SEG-Y and config.  G/s = real-trace terms / wall."""
    import tempfile

    import oracle as O
    from poststackmig3d_b200 import host as H
    from poststackmig3d_b200 import synth as S
    if not os.path.exists(O.ref_binary("omp")):
        return None
    W = S.workload_config1()
    g = geometry(W)
    terms = int(O.count_rows(W.vrms_cube(), g.out_center, 0, g.n_oi, g.n_ox, g.pad_il,
                             g.pad_xl, g.m_il, np.float32(g.dt_seconds), g.t0(),
                             np.float32(g.tan2), g.d_il, g.d_xl, g.amp,
                             threads=threads).sum())
    res = {"workload": "config1: 101x101 traces x 501 samples, pad 30/30, one SEG-Y run "
                       "(read, migrate, write)", "terms": terms}
    with tempfile.TemporaryDirectory() as d:
        for key, th in (("reference_omp_all_threads", threads), ("reference_omp_1_thread", 1)):
            cfg = S.write_run(d, W, output=f"{key}.sgy", n_threads=th)
            t = time.perf_counter()
            r = O.run_ref_binary(cfg, "omp", threads=th, timeout=1800)
            wall = time.perf_counter() - t
            if r.returncode != 0:
                return None
            res[key] = {"wall_s": wall, "G/s": terms / wall / 1e9, "threads": th}
        cfg = S.write_run(d, W, output="ours.sgy")
        H.run_binary(cfg, timeout=600)  # first run pays the module load
        t = time.perf_counter()
        r = H.run_binary(cfg, timeout=600)
        wall = time.perf_counter() - t
        if r.returncode == 0:
            res["poststackmig_b200"] = {"wall_s": wall, "G/s": terms / wall / 1e9}
    return res


def sample_rows(g, k):
    mid = g.n_oi // 2
    return [min(g.n_oi - 1, mid + i) for i in range(k)]


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    W = workload(args.workload)
    g = geometry(W)
    rows = sample_rows(g, args.cpu_rows)
    vals = []
    kind = "reference"
    for i in range(args.warmup + args.steps):
        terms, secs, kind, _ = cpu_reference_sample(W, g, rows, threads)
        if i >= args.warmup:
            vals.append((terms, secs))
    terms = sum(v[0] for v in vals)
    secs = sum(v[1] for v in vals)
    value = terms / secs / 1e9
    sample = (f"{len(rows)} central output inlines of {W.name} per step "
              f"(rows {rows[0]}..{rows[-1]}, {terms // max(len(vals), 1)} terms/step), in "
              f"blocks of 16 output crosslines taken by {threads} host threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": secs / max(len(vals), 1) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": config_dict(W, g),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------- GPU arm


def run_ours(args):
    import torch
    from poststackmig3d_b200 import Migrator

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    W = workload(args.workload)
    g = dataclasses.replace(geometry(W), precision=args.storage,
                            compensated=bool(args.compensated))
    data, vrms = W.data, W.vrms_cube()
    gl, slab = g, None
    if args.shard:  # this rank's slab of output inlines and the input inlines it reads
        from poststackmig3d_b200.migration import slab_geometry, split_slabs
        c = np.asarray(g.out_center)
        i0 = np.maximum(0, c - g.m_il - g.pad_il)
        i1 = np.minimum(g.n_il, c + g.m_il + 1 + g.pad_il)
        slab = split_slabs(g, world, (i1 - i0).astype(np.float64))[rank]  # work ~ buffer
        gl = slab_geometry(g, slab)
        data = np.ascontiguousarray(data[slab[2]:slab[3]])
        vrms = np.ascontiguousarray(vrms[slab[2]:slab[3]])
    m = Migrator(local)
    m.set_geometry(gl)
    m.set_traces(data)
    m.set_vrms(vrms)
    # G/s counts the terms the launch evaluates; padded output inlines that repeat an edge
    # inline are copies (the reference migrates them again; their terms are reported apart)
    n_terms_all = m.count_terms()
    n_terms = n_terms_local = m.count_terms_computed()
    if dist and args.shard:  # the whole migration's terms
        t = torch.tensor([n_terms_all, n_terms], dtype=torch.int64, device="cuda")
        dist.all_reduce(t)
        n_terms_all, n_terms = int(t[0].item()), int(t[1].item())
    job_scale = 1 if args.shard else world  # replicas: every rank migrates the whole cube
    stream = torch.cuda.ExternalStream(m.stream_handle())
    tuned = None
    if args.variant:
        m.set_variant(args.variant)
    else:  # project autotuner: one timed launch per kernel variant, keep the fastest
        best, ms_v = m.autotune()
        tuned = {Migrator.VARIANTS[v]: round(t, 3) for v, t in ms_v.items()}

    from poststackmig3d_b200.migration import measure_limbs
    limbs = measure_limbs(local)

    for _ in range(max(args.warmup, 0)):
        m.forward_async()
    m.synchronize()

    props = torch.cuda.get_device_properties(local)
    uuid = str(getattr(props, "uuid", ""))
    dev_id = ("GPU-" + uuid) if uuid and not uuid.startswith("GPU-") else (uuid or str(local))
    clk = ClockSampler(dev_id)

    # ---- device-resident throughput: K forward launches between two events
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk.start()
    time.sleep(0.25)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        m.forward_async()
    ev1.record(stream)
    m.synchronize()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    clk.stop()
    if dist:
        dist.barrier()
    ms_max = ms
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = job_scale * n_terms / (ms_max * 1e-3) / 1e9

    # ---- end to end through the public API: pinned host inputs -> image on the host
    e2e = None
    if not args.no_e2e:
        h_data = torch.from_numpy(data).pin_memory()
        h_vrms = torch.from_numpy(vrms).pin_memory()
        h_img = torch.empty(m.image_shape(), dtype=torch.float32).pin_memory()
        e2e_steps = max(1, min(args.steps, 3))
        m.forward_host(h_data, h_vrms, h_img)  # one pipelined call: upload, migrate, download
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            m.forward_host(h_data, h_vrms, h_img)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1) / e2e_steps
        if dist:
            t = torch.tensor([e2e_ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": job_scale * n_terms / (e2e_ms * 1e-3) / 1e9, "unit": UNIT,
               "ms_per_step": e2e_ms,
               "h2d_bytes_per_step": int(h_data.numel() * 4 + h_vrms.numel() * 4),
               "d2h_bytes_per_step": int(h_img.numel() * 4),
               "call": "psm_forward_host on pinned host buffers (traces, Vrms in; image out)"}

    clocks = clk.summary()
    sm_mhz = clocks["sm_mhz"] or limbs["sm_clock_mhz"]
    achieved = n_terms_local / (ms * 1e-3) / 1e9  # this GPU's launch
    paired = "pairs" in Migrator.VARIANTS[m.variant()]
    bound, peak, limb_peaks = limb_roofline(limbs, sm_mhz, achieved, paired,
                                            8 if g.precision == "f32" else 4)
    comp_bytes = (2 * g.n_il * g.n_xl * g.n_t + g.n_oi * g.n_ox * g.n_t) * 4
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        hbm_peak = float(peaks["hbm_gbs"])
        hbm_src = "measured"
    except Exception:
        hbm_peak, hbm_src = 6650.0, "fallback"
    hbm_ach = comp_bytes / (ms * 1e-3) / 1e9
    roofline = {
        "bound": bound, "achieved": achieved, "peak": peak, "unit": "Gterm/s",
        "frac": achieved / peak,
        "traffic": profile_traffic() if g.precision == "f32" and not g.compensated else None,
        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the forward "
                          "kernel on the 201x201 crop, scaled by term count "
                          "(profiles/fwd_kernel_config2_201.md)",
        "peak_basis": f"measured limbs (psm_measure_limbs) x {limbs['n_sm']} SMs x median SM "
                      f"clock {sm_mhz:.0f} MHz under load; binding limb {bound}",
        "limbs": limb_peaks,
        "hbm": {"achieved": hbm_ach, "peak": hbm_peak, "unit": "GB/s",
                "frac": hbm_ach / hbm_peak, "peak_source": hbm_src,
                "algorithmic_bytes_per_launch": comp_bytes},
    }

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rows = sample_rows(g, args.cpu_rows)
        terms, secs, kind, ref_rows = cpu_reference_sample(W, g, rows, threads)
        cpu = {"value": terms / secs / 1e9, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"{len(rows)} central output inlines of {W.name} "
                         f"({terms} terms, {secs:.1f} s), in blocks of 16 output "
                         f"crosslines taken by {threads} host threads"}
        if kind == "reference":
            image = m.get_image()
            parity = parity_block(W, g, image, rows, ref_rows, threads)
        if not args.no_binary_baseline:
            cpu["binary"] = binary_baseline(threads)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
                "higher_is_better": True, "scaling": "strong" if args.shard else "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                "config": config_dict(W, g, {"n_terms": n_terms,
                                             "n_terms_copied_rows": n_terms_all - n_terms,
                                             "parallelism": (f"output-inline slabs x{world}"
                                                             if args.shard else
                                                             f"replicas x{world}"),
                                             "variant": Migrator.VARIANTS[m.variant()],
                                             "autotune_ms": tuned}),
                "roofline": roofline, "parity": parity, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": args.steps, "clocks": clocks}
        print(json.dumps(line), flush=True)
    m.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_lsm(args):
    """Least-squares migration on 201x201 traces x 1001 samples (dt 2 ms, 25 m bins, V = 2000
    m/s, 30 deg, amp on): data modelled by the adjoint operator from a sparse reflectivity
    (2% nonzero, Laplace amplitudes) plus 5% Gaussian noise, then 10 CGLS iterations with
    FP32 operators and FP64 inner products on the GPU."""
    import torch
    from poststackmig3d_b200 import Migrator, plan_geometry
    n, n_t = 201, 1001
    g = plan_geometry(n, n, n_t, 0.002, 25.0, 25.0, 30.0, 2000.0, 0, 0, True)
    rng = np.random.default_rng(5)
    vr = np.full((n, n, n_t), 2000.0, dtype=np.float32)
    mtrue = np.zeros((g.n_oi, g.n_ox, n_t), dtype=np.float32)
    mask = rng.random(mtrue.shape) < 0.02
    mtrue[mask] = rng.laplace(0.0, 1.0, int(mask.sum())).astype(np.float32)
    m = Migrator(0)
    m.set_geometry(g)
    m.set_vrms(vr)
    d = m.adjoint(mtrue)
    d += (0.05 * np.abs(d).max() * rng.standard_normal(d.shape)).astype(np.float32)
    # dot-product test of the operator pair on seeded random vectors, with the plain and with
    # the compensated forward; the error is also given relative to ||M d|| ||m||, which does
    # not depend on how nearly orthogonal the two random vectors happen to be
    d1 = rng.standard_normal(d.shape).astype(np.float32)
    m1 = rng.standard_normal(mtrue.shape).astype(np.float32)
    m.set_traces(d1)
    Md = m.forward()
    MTm = m.adjoint(m1)
    rhs = float(np.sum(d1.astype(np.float64) * MTm))
    lhs = float(np.sum(Md.astype(np.float64) * m1))
    norms = float(np.linalg.norm(Md.astype(np.float64)) * np.linalg.norm(m1.astype(np.float64)))
    gk = dataclasses.replace(g, compensated=True)
    m.set_geometry(gk)
    m.set_vrms(vr)
    m.set_traces(d1)
    lhs_k = float(np.sum(m.forward().astype(np.float64) * m1))
    m.set_geometry(g)
    m.set_vrms(vr)
    dot = {"plain_forward": abs(lhs - rhs) / max(abs(lhs), abs(rhs)),
           "compensated_forward": abs(lhs_k - rhs) / max(abs(lhs_k), abs(rhs)),
           "plain_vs_norms": abs(lhs - rhs) / norms,
           "compensated_vs_norms": abs(lhs_k - rhs) / norms,
           "cos": lhs / norms}
    # the two operators on device memory (CUDA events on the library's stream): the adjoint
    # of the resident image, the forward of the resident traces
    from poststackmig3d_b200.migration import measure_limbs
    stream = torch.cuda.ExternalStream(m.stream_handle())
    n_terms = m.count_terms()

    def kernel_ms(fn, reps=3):
        fn()
        m.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        m.synchronize()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    m.set_traces(d1)
    fwd_ms = kernel_ms(m.forward_async)
    m.set_image(m1)
    adj_ms = kernel_ms(m.adjoint_async)
    limbs = measure_limbs(0)
    iters = 10
    props = torch.cuda.get_device_properties(0)
    uuid = str(getattr(props, "uuid", ""))
    clk = ClockSampler(("GPU-" + uuid) if uuid and not uuid.startswith("GPU-") else (uuid or "0"))
    torch.cuda.synchronize()
    clk.start()
    time.sleep(0.25)
    # the call uploads the data, runs the initial forward (s = M r) and downloads the image
    # around its iterations: time it with 0 iterations too (the faster of two calls, after
    # an untimed one), and report the difference
    m.lsm_cg(d, 0)
    secs0 = float("inf")
    for _ in range(2):
        t = time.perf_counter()
        m.lsm_cg(d, 0)
        secs0 = min(secs0, time.perf_counter() - t)
    t = time.perf_counter()
    img, hist = m.lsm_cg(d, iters)
    secs = time.perf_counter() - t
    clk.stop()
    m.close()
    line = {"metric": "least-squares migration, 10 CG iterations",
            "value": (secs - secs0) / iters * 1e3,
            "unit": "ms/iteration", "n_gpus": 1, "steps": iters, "warmup": 1,
            "ms_per_step": (secs - secs0) / iters * 1e3,
            "call_ms": secs * 1e3, "call_ms_0_iterations": secs0 * 1e3,
            "higher_is_better": False,
            "config": {"workload": "config5: 201x201 traces x 1001 samples, V 2000 m/s, "
                                   "30 deg, 2% Laplace reflectivity, 5% noise",
                       "iterations": iters},
            "relative_residual": float(hist[-1] / hist[0]),
            "residual_history": [float(h / hist[0]) for h in hist],
            "dot_product_rel_err": dot["plain_forward"],
            "dot_product": dot,
            "operators": {
                "terms_per_application": n_terms, "forward_ms": fwd_ms, "adjoint_ms": adj_ms,
                "adjoint_gterm_s": n_terms / (adj_ms * 1e-3) / 1e9,
                "adjoint_roofline": {
                    "bound": "shared fp32 atomics (one per term: a mirrored pair of traces "
                             "shares one window)",
                    "achieved": n_terms / (adj_ms * 1e-3) / 1e9,
                    "peak": limbs["atom_per_clk_sm"] * limbs["n_sm"] * limbs["sm_clock_mhz"]
                            * 1e6 / 1e9,
                    "unit": "Gterm/s",
                    "peak_basis": "psm_measure_limbs atom_per_clk_sm x SMs x probe clock"}},
            "adjoint_accumulation": os.environ.get("PSM_ADJ_ACCUM", "f32"),
            "dtype": "f32 operators, f64 CG scalars", "data": "synthetic (seeded)",
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def run_batch(args):
    """Config 4: 32 constant-velocity scan panels (1800..3350 m/s) over one 201x201x751 cube
    and 8 uneven sub-volumes with their own linear Vrms(t), migrated by one persistent launch
    replayed as a CUDA graph (autotuned kernel variant).  The same problems run as one grid
    launch each are timed beside it."""
    import torch
    from poststackmig3d_b200 import Batch, Migrator, Problem, estimate_max_velocity
    from poststackmig3d_b200 import plan_geometry
    from poststackmig3d_b200 import synth as S

    panels, subs = S.workload_config4(n_panels=args.panels, n_sub=args.subvolumes)
    probs = []
    cube = np.ascontiguousarray(panels[0].data)
    for W in panels:
        g = plan_geometry(*cube.shape, W.dt, W.d_il, W.d_xl, W.angle, W.velocity, 0, 0, W.amp)
        g = dataclasses.replace(g, precision=args.storage, compensated=bool(args.compensated))
        probs.append(Problem(g, cube, velocity=W.velocity))
    for W in subs:
        vr = W.vrms_cube()
        g = plan_geometry(*W.data.shape, W.dt, W.d_il, W.d_xl, W.angle,
                          estimate_max_velocity(vr), 0, 0, W.amp)
        g = dataclasses.replace(g, precision=args.storage, compensated=bool(args.compensated))
        probs.append(Problem(g, W.data, np.ascontiguousarray(vr[0, 0])))
    m = Migrator(0)
    b = Batch(m, probs)
    n_terms = b.count_terms()
    stream = torch.cuda.ExternalStream(m.stream_handle())
    tuned = None
    if args.variant:
        b.set_variant(args.variant)
        b.set_order(max(args.order, 0))
    else:
        best, order, mode, ms_v = b.autotune()
        tuned = {f"{Migrator.VARIANTS[v]}/{Batch.SCHEDULES[sch]}": round(t, 3)
                 for (v, sch), t in ms_v.items()}
        if args.order >= 0:
            b.set_order(args.order)
    chosen_mode = b.mode()

    def timed(steps):
        for _ in range(max(args.warmup, 0)):
            b.run_async()
        b.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            b.run_async()
        e1.record(stream)
        b.synchronize()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    props = torch.cuda.get_device_properties(0)
    uuid = str(getattr(props, "uuid", ""))
    clk = ClockSampler(("GPU-" + uuid) if uuid and not uuid.startswith("GPU-") else (uuid or "0"))
    b.set_mode(Batch.PER_PROBLEM)
    ms_sep = timed(max(1, min(args.steps, 3)))
    b.set_mode(Batch.PERSISTENT)
    ms_pers = timed(max(1, min(args.steps, 3)))
    b.set_mode(Batch.ONE_GRID)
    ms_grid = timed(max(1, min(args.steps, 3)))
    b.set_mode(chosen_mode)
    torch.cuda.synchronize()
    clk.start()
    time.sleep(0.25)
    ms = timed(args.steps)
    clk.stop()
    value = n_terms / (ms * 1e-3) / 1e9

    e2e = None
    if not args.no_e2e:
        imgs = [torch.empty((p.geom.n_oi, p.geom.n_ox, p.geom.n_t),
                            dtype=torch.float32).pin_memory() for p in probs]
        steps = max(1, min(args.steps, 3))

        def e2e_step():
            b.reload()
            b.run()
            for i, im in enumerate(imgs):
                b.image(i, im)

        e2e_step()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1) / steps
        h2d = cube.nbytes + sum(W.data.nbytes + 4 * W.data.shape[2] for W in subs)
        e2e = {"value": n_terms / (e2e_ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": e2e_ms,
               "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(sum(im.numel() * 4 for im in imgs)),
               "host_inputs": "pageable numpy arrays (the Problem arrays)"}

    clocks = clk.summary()
    from poststackmig3d_b200.migration import measure_limbs
    limbs = measure_limbs(0)

    # parity of sampled rows: the slowest and fastest panels and the first sub-volume,
    # against the reference's kernel (constant or linear Vrms, as the problem has) and the
    # FP64 oracle; 16-bit storage is compared with the oracle fed the dequantised samples
    parity = None
    if not args.no_cpu_baseline:
        import oracle as O
        threads = os.cpu_count() or 1
        b.run()
        checks = []
        for k in (0, len(panels) - 1, len(panels)):
            if k >= len(probs):
                continue
            p = probs[k]
            W = panels[k] if k < len(panels) else subs[k - len(panels)]
            gk = p.geom
            row = [gk.n_oi // 2]
            vr = W.vrms_cube()
            img = b.image(k)[row]
            data = W.data if args.storage == "f32" else O.dequantized(W.data, args.storage)
            sub = np.ascontiguousarray(np.asarray(gk.out_center)[row])
            _, r64, _ = O.migrate_volume(data, vr, sub, gk.n_ox, 0, 0, gk.m_il,
                                         np.float32(gk.dt_seconds), gk.t0(),
                                         np.float32(gk.tan2), gk.d_il, gk.d_xl, gk.amp,
                                         O.CONTRACT | O.F64, threads, True)
            e = {"problem": k, "row": row[0], "vs_fp64": _err(img, r64)}
            if O.ref_available():
                ref, _ = O.reference_rows(W.data, vr, gk.out_center, row, gk.n_ox, 0, 0,
                                          gk.m_il, gk.dt_seconds, gk.t0(), gk.tan2, gk.d_il,
                                          gk.d_xl, gk.amp)
                e["vs_reference"] = _err(img, ref)
            checks.append(e)
        parity = {"checks": checks,
                  "reference": "kirchhoffKernel3DWithPadding compiled from the reference's "
                               "sources (oracle/_ref, OpenMP build)",
                  "fp64": "FP64 oracle of the same operator" + (
                      ", fed the dequantised samples" if args.storage != "f32" else "")}
    sm_mhz = clocks["sm_mhz"] or limbs["sm_clock_mhz"]
    bound, peak, limb_peaks = limb_roofline(limbs, sm_mhz, value,
                                            "pairs" in Migrator.VARIANTS[b.variant()],
                                            8 if args.storage == "f32" else 4)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": f"config4: {len(panels)} constant-velocity panels 1800 + 50 k "
                                   f"m/s over 201x201x751 (2 ms, 25 m, 30 deg, amp on) + "
                                   f"{len(subs)} sub-volumes 64-256 traces per axis, "
                                   f"401-1001 samples, own linear Vrms",
                       "problems": len(probs), "n_terms": n_terms,
                       "storage": args.storage, "compensated": bool(args.compensated),
                       "launch": {0: "one persistent launch per step",
                                  1: "one grid launch per problem",
                                  2: "one grid launch over every problem's tiles"}[chosen_mode]
                                 + ", replayed as a CUDA graph (autotuned schedule)",
                       "variant": Migrator.VARIANTS[b.variant()],
                       "tile_order": Batch.ORDERS[b.order()], "autotune_ms": tuned,
                       "per_problem_graph_ms": ms_sep, "persistent_graph_ms": ms_pers,
                       "one_grid_graph_ms": ms_grid,
                       "l2": "inputs larger than L2 (panel cube 121 MB, images 3.9 GB)"},
            "roofline": {"bound": bound, "achieved": value, "peak": peak, "unit": "Gterm/s",
                         "frac": value / peak, "traffic": None, "limbs": limb_peaks,
                         "peak_basis": f"measured limbs (psm_measure_limbs) x "
                                       f"{limbs['n_sm']} SMs x median SM clock "
                                       f"{sm_mhz:.0f} MHz under load"},
            "parity": parity, "cpu_baseline": None, "e2e": e2e, "gpu_launches": args.steps,
            "clocks": clocks}
    print(json.dumps(line), flush=True)
    b.close()
    m.close()
    return 0


def run_io(args):
    """The data formats either side of the summation, on config 2 (401x401 traces x 1001
    samples), each through the public API from host buffers (wall clock around the call):
    SEG-Y trace records decoded and image records encoded on the GPU (IEEE big-endian,
    format 5), the Vrms cube assembled on the GPU from a coarser SEG-Y grid (time
    interpolation) and from a text table of points, and the forward migration streamed in
    inline slabs under a device-memory budget of 70% of the resident footprint (4 slabs; an
    output inline's buffer alone spans about 74% of config 2's inlines).  Each is run
    once untimed first; the decoded cube and the streamed image are checked against the
    resident ones."""
    import torch
    from poststackmig3d_b200 import Migrator
    from poststackmig3d_b200.migration import plan_slabs, slab_bytes
    W = workload("config2")
    g = geometry(W)
    n_il, n_xl, n_t = W.data.shape
    vr = W.vrms_cube()
    rec_bytes = 240 + 4 * n_t
    rec = np.zeros((n_il * n_xl, rec_bytes), dtype=np.uint8)
    rec[:, 240:] = W.data.reshape(-1, n_t).astype(">f4").view(np.uint8)
    pos = np.arange(n_il * n_xl, dtype=np.int32)
    m = Migrator(0)
    m.set_geometry(g)

    def timed(f):
        f()
        torch.cuda.synchronize()
        t = time.perf_counter()
        out = f()
        torch.cuda.synchronize()
        return time.perf_counter() - t, out

    t_dec, _ = timed(lambda: m.set_traces_segy(rec, 5, pos))
    decoded_ok = bool(np.array_equal(m.get_traces(), W.data))
    m.set_vrms(vr)
    image = m.forward()
    src = np.arange(g.n_oi * g.n_ox, dtype=np.int32)
    il_lab = np.asarray(W.il_labels, dtype=np.int32)
    xl_lab = np.asarray(W.xl_labels, dtype=np.int32)
    t_enc, out = timed(lambda: m.get_image_segy(5, src, il_lab, xl_lab))
    encoded_ok = bool(np.array_equal(out[:, 240:].view(">f4").astype(np.float32),
                                     image.reshape(-1, n_t)))
    # Vrms: a SEG-Y grid at 4 ms on the same traces (time interpolation), and a table
    grid = np.ascontiguousarray(vr[:, :, ::2])
    t_grid, _ = timed(lambda: m.set_vrms_grid(grid, il_lab, xl_lab, 0.004, il_lab, xl_lab))
    pts = [(int(i), int(x), float(tt), 1500.0 + 1000.0 * tt)
           for i in (1, 201, 401) for x in (1, 201, 401) for tt in (0.0, 0.4, 0.8, 1.2, 1.6, 2.0)]
    t_table, _ = timed(lambda: m.set_vrms_table(pts, il_lab, xl_lab))
    m.set_vrms(vr)
    # slab streaming under 70% of the resident device footprint
    budget = int(0.70 * slab_bytes(g, g.n_il, g.n_oi))
    n_slabs = len(plan_slabs(g, budget))
    t_str, streamed = timed(lambda: m.forward_streamed(g, W.data, vr, budget))
    streamed_ok = bool(np.array_equal(streamed, image))
    m.close()
    samples = n_il * n_xl * n_t
    n_terms = 1104876190176
    line = {"metric": "config 2 formats and streaming through the public API (host buffers)",
            "workload": "config2_io: 401x401 traces x 1001 samples",
            "segy_decode": {"GB/s": rec.nbytes / t_dec / 1e9, "ms": t_dec * 1e3,
                            "format": 5, "bytes": rec.nbytes, "equal": decoded_ok},
            "segy_encode": {"GB/s": out.nbytes / t_enc / 1e9, "ms": t_enc * 1e3,
                            "format": 5, "bytes": out.nbytes, "equal": encoded_ok},
            "vrms_grid": {"Gsamples/s": samples / t_grid / 1e9, "ms": t_grid * 1e3,
                          "grid": "4 ms, same traces (time interpolation)"},
            "vrms_table": {"Gsamples/s": samples / t_table / 1e9, "ms": t_table * 1e3,
                           "points": len(pts)},
            "forward_streamed": {"G/s": n_terms / t_str / 1e9, "ms": t_str * 1e3,
                                 "slabs": n_slabs, "device_budget_bytes": budget,
                                 "equal_to_resident": streamed_ok},
            "data": "synthetic (seeded)"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "config5":
        return run_lsm(args)
    if args.workload == "config4":
        return run_batch(args)
    if args.workload == "config2_io":
        return run_io(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
