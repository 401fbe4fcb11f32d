"""ctypes binding of libngpu.so (include/ngpu.h).

The library is loaded from this package directory only; if it is missing the
import fails loudly -- there is no CPU fallback for the simulation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libngpu.so"

NGPU_FP32 = 0
NGPU_FP64 = 1
NGPU_LAYOUT_LANE_INSTANCE = 0
NGPU_LAYOUT_WARP_INSTANCE = 1
MECHSET_TTPC = 0
MECHSET_MAINEN = 1


class NgpuError(RuntimeError):
    """A libngpu call returned a non-zero status."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed ({code}): {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m neurogpu_b200._build` "
                "(the CUDA extension is required; there is no CPU path)")
        L = C.CDLL(str(LIB_PATH))
        P, I32, I64, F32, D = C.c_void_p, C.c_int32, C.c_int64, C.c_float, C.c_double
        sig = {
            "ngpu_last_error": (C.c_char_p, []),
            "ngpu_abi_version": (C.c_int, []),
            "ngpu_mechset_info": (C.c_int, [I32, P, P]),
            "ngpu_model_create": (C.c_int, [I32, P, P, P, P, P, I32, I32, P, P]),
            "ngpu_model_destroy": (C.c_int, [P]),
            "ngpu_model_layout": (C.c_int, [P, P, P, P, P, P]),
            "ngpu_model_partition": (C.c_int, [P, I32, P, P, P, P, P]),
            "ngpu_model_nodes": (C.c_int, [P, P, P, P, P]),
            "ngpu_device_count": (C.c_int, [P]),
            "ngpu_set_device": (C.c_int, [I32]),
            "ngpu_model_arrays": (C.c_int, [P, P, P, P, P]),
            "ngpu_model_split_info": (C.c_int, [P, I32, P, P, P, I32, P, P, I32, P, P]),
            "ngpu_run": (C.c_int, [P, I32, P, I32, I32, P, P, I32, F32, I32, P, F32, I32, P]),
            "ngpu_sim_create": (C.c_int, [P, I32, I32, I32, P]),
            "ngpu_sim_create_ex": (C.c_int, [P, I32, I32, I32, I32, P]),
            "ngpu_sim_create_shaped": (C.c_int, [P, I32, I32, I32, I32, I32, P]),
            "ngpu_sim_create_layout": (C.c_int, [P, I32, I32, I32, I32, I32, I32, P]),
            "ngpu_sim_layout": (C.c_int, [P, P, P, P]),
            "ngpu_batch_create": (C.c_int, [P, I32, P]),
            "ngpu_batch_destroy": (C.c_int, [P]),
            "ngpu_batch_init": (C.c_int, [P, F32, P]),
            "ngpu_batch_advance": (C.c_int, [P, I32, I32, P]),
            "ngpu_batch_run_graph": (C.c_int, [P, F32, I32, I32, P]),
            "ngpu_gemm_bf16_tn": (C.c_int, [P, P, I32, I32, I32, I32, I32, I32, I32, P, P, P, I32, I32, P, P, P]),
            "ngpu_gemm_error": (C.c_int, [P]),
            "ngpu_sim_destroy": (C.c_int, [P]),
            "ngpu_sim_set_params": (C.c_int, [P, P, I32]),
            "ngpu_sim_set_stimulus": (C.c_int, [P, I32, P, P, I32, F32, I32]),
            "ngpu_sim_set_recording": (C.c_int, [P, I32, P, I32]),
            "ngpu_sim_init": (C.c_int, [P, F32, P]),
            "ngpu_sim_advance": (C.c_int, [P, I32, I32, P]),
            "ngpu_sim_n_samples": (C.c_int, [P]),
            "ngpu_sim_get_trace": (C.c_int, [P, P, I32, P]),
            "ngpu_sim_check": (C.c_int, [P, P, P]),
            "ngpu_sim_trace_device": (C.c_int, [P, P, P]),
            "ngpu_sim_classes": (C.c_int, [P, P]),
            "ngpu_sim_param_folds": (C.c_int, [P, P]),
            "ngpu_sim_param_rows": (C.c_int, [P, P, P]),
            "ngpu_trace_features": (C.c_int, [P, I64, I64, I32, I32, C.c_double, C.c_double, C.c_double, F32, P, P]),
            "ngpu_sim_features": (C.c_int, [P, I32, C.c_double, C.c_double, C.c_double, F32, P, P]),
            "ngpu_dvdt_peaks_scratch_bytes": (I64, [I32, I32]),
            "ngpu_trace_dvdt_peaks": (C.c_int, [P, I64, I64, I32, I32, D, D, I32, P, I64, P, P]),
            "ngpu_sim_dvdt_peaks": (C.c_int, [P, I32, D, D, I32, P, I64, P, P]),
            "ngpu_jit_build": (C.c_int, [I32, I32, P, I32, I32, I32, P]),
            "ngpu_mechset_define": (C.c_int, [C.c_char_p, C.c_char_p, I32, P, P, P, I32, P, P]),
            "ngpu_jit_log": (C.c_char_p, []),
            "ngpu_launch_count": (I64, [I32]),
            "ngpu_run_static": (C.c_int, [P, I32, P, I32, I32, P, P, I32, F32, I32, P, F32, P, P]),
            "ngpu_ga_offspring": (C.c_int, [P, P, P, I32, I32, I32, D, D, D, D, D, D, C.c_uint64, C.c_uint64,
                                            P, P]),
            "ngpu_ga_select_truncation": (C.c_int, [P, I32, I32, P, P]),
            "ngpu_ga_select_nsga2": (C.c_int, [P, I32, I32, I32, P, P, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(fn: str, rc: int) -> None:
    if rc != 0:
        msg = lib().ngpu_last_error().decode(errors="replace")
        raise NgpuError(fn, rc, msg)


def ptr(a: np.ndarray | None) -> C.c_void_p | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to libngpu must be C-contiguous"
    return C.c_void_p(a.ctypes.data)


def exported_symbols() -> list[str]:
    """Names of the C-ABI entry points declared in include/ngpu.h."""
    hdr = (_HERE.parent / "include" / "ngpu.h").read_text()
    import re
    return sorted(set(re.findall(r"\b(ngpu_[a-z0-9_]+)\s*\(", hdr)))
