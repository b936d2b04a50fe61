"""ctypes binding of the in-tree native libraries.

The product path is native only: loading fails loudly (ImportError / RuntimeError) when
libpsm_cuda.so has not been built; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(PKG, "lib")

PSM_OK = 0
STATUS = {0: "PSM_OK", -1: "PSM_ERR_ARG", -2: "PSM_ERR_STATE", -3: "PSM_ERR_CUDA",
          -4: "PSM_ERR_NOMEM", -5: "PSM_ERR_DEVICE", -6: "PSM_ERR_UNSUPPORTED"}


class PsmGeom(ctypes.Structure):
    """Mirror of psm_geom (include/psm.h)."""
    _fields_ = [("n_il", ctypes.c_int32), ("n_xl", ctypes.c_int32), ("n_t", ctypes.c_int32),
                ("pad_il", ctypes.c_int32), ("pad_xl", ctypes.c_int32),
                ("n_oi", ctypes.c_int32), ("n_ox", ctypes.c_int32), ("m_il", ctypes.c_int32),
                ("amp_correction", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("dt", ctypes.c_float), ("d_il", ctypes.c_float), ("d_xl", ctypes.c_float),
                ("tan2_theta", ctypes.c_float), ("dt_seconds", ctypes.c_double),
                ("compensated", ctypes.c_int32), ("compat_omp_pad", ctypes.c_int32)]


class PsmProblem(ctypes.Structure):
    """Mirror of psm_problem (include/psm.h)."""
    _fields_ = [("geom", PsmGeom), ("out_center", ctypes.c_void_p),
                ("traces", ctypes.c_void_p), ("vrms", ctypes.c_void_p),
                ("vrms_kind", ctypes.c_int32), ("velocity", ctypes.c_float)]


class PsmSlab(ctypes.Structure):
    """Mirror of psm_slab (include/psm.h)."""
    _fields_ = [("o0", ctypes.c_int32), ("o1", ctypes.c_int32), ("i0", ctypes.c_int32),
                ("i1", ctypes.c_int32)]


class PsmLimbs(ctypes.Structure):
    """Mirror of psm_limbs (include/psm.h)."""
    _fields_ = [("sm_clock_mhz", ctypes.c_double), ("n_sm", ctypes.c_int32),
                ("rsqrt_per_clk_sm", ctypes.c_double), ("ffma_per_clk_sm", ctypes.c_double),
                ("ffma2_per_clk_sm", ctypes.c_double),
                ("lds64_bytes_per_clk_sm", ctypes.c_double),
                ("lds64_slope_bytes_per_clk_sm", ctypes.c_double),
                ("atom_per_clk_sm", ctypes.c_double),
                ("atom_slope_per_clk_sm", ctypes.c_double),
                ("red_per_clk_sm", ctypes.c_double), ("red_slope_per_clk_sm", ctypes.c_double),
                ("atom_u32_per_clk_sm", ctypes.c_double),
                ("atom_u32_slope_per_clk_sm", ctypes.c_double),
                ("atom_u64_per_clk_sm", ctypes.c_double),
                ("atom_u64_slope_per_clk_sm", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class PsmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


_cuda = None

# (name, restype, argtypes) of every symbol include/psm.h declares
_P = ctypes.c_void_p
_CUDA_SYMBOLS = [
    ("psm_version", ctypes.c_char_p, []),
    ("psm_device_count", ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    ("psm_create", ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int]),
    ("psm_destroy", ctypes.c_int, [_P]),
    ("psm_last_error", ctypes.c_char_p, [_P]),
    ("psm_set_geometry", ctypes.c_int, [_P, ctypes.POINTER(PsmGeom), _P]),
    ("psm_set_traces", ctypes.c_int, [_P, _P]),
    ("psm_set_vrms", ctypes.c_int, [_P, _P]),
    ("psm_forward", ctypes.c_int, [_P, _P]),
    ("psm_forward_async", ctypes.c_int, [_P]),
    ("psm_forward_host", ctypes.c_int, [_P, _P, _P, _P]),
    ("psm_synchronize", ctypes.c_int, [_P]),
    ("psm_image_device", ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    ("psm_get_image", ctypes.c_int, [_P, _P]),
    ("psm_stream", ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    ("psm_count_terms", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int64)]),
    ("psm_count_terms_rows", ctypes.c_int, [_P, _P]),
    ("psm_slab_bytes", ctypes.c_int64, [ctypes.POINTER(PsmGeom), ctypes.c_int32,
                                        ctypes.c_int32]),
    ("psm_plan_slabs", ctypes.c_int, [ctypes.POINTER(PsmGeom), _P, ctypes.c_int64, _P,
                                      ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    ("psm_split_slabs", ctypes.c_int, [ctypes.POINTER(PsmGeom), _P, _P, ctypes.c_int32, _P]),
    ("psm_slab_geometry", ctypes.c_int, [ctypes.POINTER(PsmGeom), _P, _P,
                                         ctypes.POINTER(PsmGeom), _P]),
    ("psm_forward_streamed", ctypes.c_int, [_P, ctypes.POINTER(PsmGeom), _P, _P, _P, _P,
                                            ctypes.c_int64]),
    ("psm_set_vrms_table", ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int32, _P, _P]),
    ("psm_set_vrms_grid", ctypes.c_int, [_P, _P, _P, ctypes.c_int32, _P, ctypes.c_int32,
                                         ctypes.c_int32, ctypes.c_double, _P, _P]),
    ("psm_get_vrms", ctypes.c_int, [_P, _P]),
    ("psm_set_traces_segy", ctypes.c_int, [_P, _P, ctypes.c_int64, ctypes.c_int32, _P]),
    ("psm_get_image_segy", ctypes.c_int, [_P, _P, ctypes.c_int32, _P, _P, _P]),
    ("psm_get_traces", ctypes.c_int, [_P, _P]),
    ("psm_set_image", ctypes.c_int, [_P, _P]),
    ("psm_adjoint", ctypes.c_int, [_P, _P, _P]),
    ("psm_adjoint_async", ctypes.c_int, [_P]),
    ("psm_forward_device", ctypes.c_int, [_P, _P, _P]),
    ("psm_adjoint_device", ctypes.c_int, [_P, _P, _P]),
    ("psm_lsm_cg", ctypes.c_int, [_P, _P, _P, ctypes.c_int, _P]),
    ("psm_set_variant", ctypes.c_int, [_P, ctypes.c_int]),
    ("psm_get_variant", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    ("psm_autotune", ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_int)]),
    ("psm_batch_create", ctypes.c_int, [_P, ctypes.POINTER(PsmProblem), ctypes.c_int,
                                        ctypes.POINTER(_P)]),
    ("psm_batch_destroy", ctypes.c_int, [_P]),
    ("psm_batch_reload", ctypes.c_int, [_P]),
    ("psm_batch_set_mode", ctypes.c_int, [_P, ctypes.c_int]),
    ("psm_batch_set_variant", ctypes.c_int, [_P, ctypes.c_int]),
    ("psm_batch_get_variant", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    ("psm_batch_set_order", ctypes.c_int, [_P, ctypes.c_int]),
    ("psm_batch_get_order", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    ("psm_batch_autotune", ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int)]),
    ("psm_batch_get_mode", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    ("psm_batch_run_async", ctypes.c_int, [_P]),
    ("psm_batch_synchronize", ctypes.c_int, [_P]),
    ("psm_batch_run", ctypes.c_int, [_P]),
    ("psm_batch_image_device", ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(_P)]),
    ("psm_batch_get_image", ctypes.c_int, [_P, ctypes.c_int, _P]),
    ("psm_batch_count_terms", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int64)]),
    ("psm_kirchhoff_inline", ctypes.c_int,
     [_P, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, _P, _P, ctypes.c_size_t, _P, _P,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_float, _P, ctypes.c_float, ctypes.c_float,
      ctypes.c_float, ctypes.c_int]),
    ("psm_kirchhoff_inline_error", ctypes.c_char_p, []),
    ("psm_measure_limbs", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(PsmLimbs)]),
]


def cuda_lib_path() -> str:
    return os.path.join(LIB_DIR, "libpsm_cuda.so")


def cuda() -> ctypes.CDLL:
    """Load libpsm_cuda.so (raises if it is missing: build with
    `python -m poststackmig3d_b200.build`)."""
    global _cuda
    if _cuda is None:
        path = cuda_lib_path()
        if not os.path.exists(path):
            raise ImportError(f"{path} is not built; run python -m poststackmig3d_b200.build")
        L = ctypes.CDLL(path)
        for name, res, args in _CUDA_SYMBOLS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _cuda = L
    return _cuda


def check(code: int, msg_fn=None) -> None:
    if code != PSM_OK:
        raise PsmError(code, msg_fn() if msg_fn else "")
