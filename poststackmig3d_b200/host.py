"""Python binding of libpsm_host.so (include/psm_host.h): config.txt parsing, SEG-Y reading
with the INLINE_3D/CROSSLINE_3D lookup, IBM/IEEE conversion, Vrms providers, the migration
plan and the whole config-driven run (src/main.cpp of the reference)."""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from ._lib import LIB_DIR, PsmError, cuda

_host = None
_P = ctypes.c_void_p


class PsmConfig(ctypes.Structure):
    _fields_ = [("input_data", ctypes.c_char * 1024), ("output_data", ctypes.c_char * 1024),
                ("inline_step", ctypes.c_double), ("crossline_step", ctypes.c_double),
                ("inline_padding", ctypes.c_int32), ("crossline_padding", ctypes.c_int32),
                ("velocity", ctypes.c_char * 1024), ("angle_aperture", ctypes.c_double),
                ("amp_correction", ctypes.c_int32), ("n_threads", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("compensated", ctypes.c_int32),
                ("device", ctypes.c_int32), ("compat_omp_pad", ctypes.c_int32)]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = v.decode() if isinstance(v, bytes) else v
        d["amp_correction"] = bool(d["amp_correction"])
        d["compensated"] = bool(d["compensated"])
        d["compat_omp_pad"] = bool(d["compat_omp_pad"])
        return d


class PsmSegyInfo(ctypes.Structure):
    _fields_ = [("num_traces", ctypes.c_int64), ("num_samples", ctypes.c_int32),
                ("dt_us", ctypes.c_int32), ("dt_seconds", ctypes.c_double),
                ("format", ctypes.c_int32), ("n_il", ctypes.c_int32),
                ("n_xl", ctypes.c_int32), ("n_mapped", ctypes.c_int64)]


class PsmPlan(ctypes.Structure):
    _fields_ = [("n_il", ctypes.c_int32), ("n_xl", ctypes.c_int32), ("n_t", ctypes.c_int32),
                ("n_oi", ctypes.c_int32), ("n_ox", ctypes.c_int32), ("m_il", ctypes.c_int32),
                ("max_v", ctypes.c_float), ("tan2_theta", ctypes.c_float),
                ("dt_seconds", ctypes.c_double)]


_ERR = ctypes.c_char_p
_HOST_SYMBOLS = [
    ("psm_config_load", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(PsmConfig), _P,
                                       ctypes.c_size_t]),
    ("psm_segy_scan", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(PsmSegyInfo), _P,
                                     ctypes.c_size_t]),
    ("psm_segy_read_cube", ctypes.c_int, [ctypes.c_char_p, _P, _P, _P, _P, ctypes.c_size_t]),
    ("psm_ibm_to_ieee", ctypes.c_float, [ctypes.c_uint32]),
    ("psm_ieee_to_ibm", ctypes.c_uint32, [ctypes.c_float]),
    ("psm_velocity_cube", ctypes.c_int, [ctypes.c_char_p, _P, ctypes.c_int32, _P,
                                         ctypes.c_int32, ctypes.c_int32, ctypes.c_double, _P,
                                         _P, ctypes.c_size_t]),
    ("psm_velocity_point", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                          ctypes.POINTER(ctypes.c_float), _P,
                                          ctypes.c_size_t]),
    ("psm_plan_config", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(PsmPlan), _P,
                                       ctypes.c_size_t]),
    ("psm_run_config", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _P, ctypes.c_size_t]),
]


def host_lib_path() -> str:
    return os.path.join(LIB_DIR, "libpsm_host.so")


def host() -> ctypes.CDLL:
    global _host
    if _host is None:
        cuda()  # dependency, loaded first so the rpath lookup is not needed
        path = host_lib_path()
        if not os.path.exists(path):
            raise ImportError(f"{path} is not built; run python -m poststackmig3d_b200.build")
        L = ctypes.CDLL(path)
        for name, res, args in _HOST_SYMBOLS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _host = L
    return _host


def _call(fn, *args):
    err = ctypes.create_string_buffer(2048)
    rc = fn(*args, err, len(err))
    if rc != 0:
        raise PsmError(rc, err.value.decode(errors="replace"))


def load_config(path: str) -> dict:
    c = PsmConfig()
    _call(host().psm_config_load, path.encode(), ctypes.byref(c))
    return c.as_dict()


def segy_info(path: str) -> dict:
    i = PsmSegyInfo()
    _call(host().psm_segy_scan, path.encode(), ctypes.byref(i))
    return {n: getattr(i, n) for n, _ in i._fields_}


def read_segy(path: str):
    """(il_labels, xl_labels, cube[n_il][n_xl][ns], info)."""
    info = segy_info(path)
    il = np.zeros(info["n_il"], dtype=np.int32)
    xl = np.zeros(info["n_xl"], dtype=np.int32)
    cube = np.zeros((info["n_il"], info["n_xl"], info["num_samples"]), dtype=np.float32)
    _call(host().psm_segy_read_cube, path.encode(), il.ctypes.data, xl.ctypes.data,
          cube.ctypes.data)
    return il, xl, cube, info


def ibm_to_ieee(words) -> np.ndarray:
    L = host()
    return np.array([L.psm_ibm_to_ieee(int(w)) for w in np.asarray(words).ravel()],
                    dtype=np.float32)


def ieee_to_ibm(values) -> np.ndarray:
    L = host()
    return np.array([L.psm_ieee_to_ibm(float(v)) for v in np.asarray(values, np.float32).ravel()],
                    dtype=np.uint32)


def velocity_cube(param: str, il_labels, xl_labels, n_t: int, dt: float) -> np.ndarray:
    il = np.ascontiguousarray(il_labels, dtype=np.int32)
    xl = np.ascontiguousarray(xl_labels, dtype=np.int32)
    out = np.zeros((len(il), len(xl), n_t), dtype=np.float32)
    _call(host().psm_velocity_cube, param.encode(), il.ctypes.data, len(il), xl.ctypes.data,
          len(xl), n_t, dt, out.ctypes.data)
    return out


def velocity_point(param: str, il: int, xl: int, t_idx: int, dt: float, n_t: int) -> float:
    v = ctypes.c_float()
    _call(host().psm_velocity_point, param.encode(), il, xl, t_idx, dt, n_t, ctypes.byref(v))
    return float(v.value)


def plan_config(path: str) -> dict:
    p = PsmPlan()
    _call(host().psm_plan_config, path.encode(), ctypes.byref(p))
    return {n: getattr(p, n) for n, _ in p._fields_}


def run_config(path: str, verbose: bool = True) -> None:
    """The whole poststackmig run of a config.txt (GPU migration)."""
    _call(host().psm_run_config, path.encode(), int(bool(verbose)))


def binary_path() -> str:
    return os.path.join(os.path.dirname(LIB_DIR), "bin", "poststackmig")


def run_binary(config_path: str, timeout: Optional[float] = None):
    import subprocess
    return subprocess.run([binary_path(), config_path], capture_output=True, text=True,
                          timeout=timeout)
