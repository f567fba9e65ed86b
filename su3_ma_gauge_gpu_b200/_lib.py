"""ctypes binding of ``libgfix.so`` (the C ABI declared in ``include/gfix.h``).

The shared library is built in-tree by ``su3_ma_gauge_gpu_b200.build``.  There is
no fallback: if the library is missing or fails to load, :func:`lib` raises, so
nothing in this package can silently run on the CPU.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libgfix.so"

GF_OK = 0
GF_ERR_INVALID = 1
GF_ERR_CUDA = 2
GF_ERR_TIMEOUT = 3
GF_ERR_NOMEM = 4
GF_ERR_UNSUPPORTED = 5

GF_LANDAU, GF_COULOMB, GF_MAG, GF_U1XU1 = 0, 1, 2, 3
GF_FP32, GF_FP64 = 0, 1
GF_MAX, GF_AVERAGE = 0, 1
GF_FILE_PLAIN, GF_FILE_HEADERONLY, GF_FILE_VOGT, GF_FILE_ILDG, GF_FILE_QCDSTAG = 0, 1, 2, 3, 4
GF_LAYOUT_GPU, GF_LAYOUT_TIMESLICE = 0, 1

_c_int, _c_float, _c_double = ctypes.c_int, ctypes.c_float, ctypes.c_double
_vp = ctypes.c_void_p
_i32p = ctypes.POINTER(ctypes.c_int32)
_dp = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes); the single source for the Python side of the ABI
SIGNATURES = {
    "gf_last_error_string": (ctypes.c_char_p, []),
    "gf_version": (ctypes.c_char_p, []),
    "gf_binary_arch": (_c_int, [ctypes.POINTER(_c_int)]),
    "gf_or_step": (_c_int, [_c_int, _c_int, _vp, _vp, _i32p, _c_int, _c_float, _vp]),
    "gf_micro_step": (_c_int, [_c_int, _c_int, _vp, _vp, _i32p, _c_int, _vp]),
    "gf_sa_step": (_c_int, [_c_int, _c_int, _vp, _vp, _i32p, _c_int, _c_float, _c_int, _c_int, _vp]),
    "gf_sr_step": (_c_int, [_c_int, _c_int, _vp, _vp, _i32p, _c_int, _c_float, _c_int, _c_int, _vp]),
    "gf_random_trafo": (_c_int, [_c_int, _c_int, _vp, _vp, _i32p, _c_int, _c_int, _c_int, _vp]),
    "gf_step_slices": (_c_int, [_c_int, _c_int, _c_int, _vp, _i32p, _c_int, _c_float, _c_int, _c_int, _c_int, _c_int,
                                _vp]),
    "gf_step_slices_at": (_c_int, [_c_int, _c_int, _c_int, _vp, _i32p, _c_int, _c_float, _c_int, _c_int, _c_int,
                                   _c_int, ctypes.c_longlong, _vp]),
    "gf_quality_per_site": (_c_int, [_c_int, _c_int, _vp, _i32p, _vp, _vp, _vp]),
    "gf_quality_prefactor_gff": (_c_double, [_c_int]),
    "gf_quality_prefactor_a": (_c_double, [_c_int]),
    "gf_project_su3": (_c_int, [_c_int, _vp, _i32p, _vp]),
    "gf_set_hot": (_c_int, [_c_int, _vp, _i32p, _c_int, _c_int, _vp]),
    "gf_stats_create": (_c_int, [_c_int, _c_int, _i32p, _c_int, ctypes.POINTER(_vp)]),
    "gf_stats_generate": (_c_int, [_vp, _vp, _vp, _dp, _dp]),
    "gf_stats_destroy": (_c_int, [_vp]),
    "gf_quality_noalloc": (_c_int, [_c_int, _c_int, _vp, _i32p, _c_int, _vp, _dp, _dp]),
    "gf_file_read": (_c_int, [ctypes.c_char_p, _c_int, _c_int, _i32p, _c_int, _c_int, _vp, _c_int, _vp]),
    "gf_file_write": (_c_int, [ctypes.c_char_p, _c_int, _c_int, _i32p, _c_int, _c_int, _vp, _c_int, ctypes.c_char_p,
                               _c_int, _vp]),
}



class CtxParams(ctypes.Structure):
    """gf_ctx_params of include/gfix.h."""

    _fields_ = [("gauge", ctypes.c_int), ("ninstances", ctypes.c_int), ("sizes", _i32p), ("mixed", ctypes.c_int),
                ("stream", ctypes.c_void_p)]


class Schedule(ctypes.Structure):
    """gf_schedule of include/gfix.h (the reference's ProgramOptions knobs)."""

    _fields_ = [("random_trafo", ctypes.c_int), ("seed", ctypes.c_uint32), ("rng_counter", ctypes.c_uint32),
                ("sa_steps", ctypes.c_int), ("sa_min", ctypes.c_float), ("sa_max", ctypes.c_float),
                ("sa_geometric", ctypes.c_int), ("micro_updates", ctypes.c_int), ("or_max_iter", ctypes.c_int),
                ("or_parameter", ctypes.c_float), ("precision", ctypes.c_double), ("switch_theta", ctypes.c_double),
                ("check_precision", ctypes.c_int), ("reproject", ctypes.c_int), ("use_graphs", ctypes.c_int),
                ("autotune", ctypes.c_int), ("micro_every", ctypes.c_int), ("sa_mode", ctypes.c_int),
                ("sa_repeat", ctypes.c_int), ("sa_slow_lo", ctypes.c_double), ("sa_slow_hi", ctypes.c_double),
                ("sa_slow_factor", ctypes.c_float), ("sr_max_iter", ctypes.c_int), ("sr_parameter", ctypes.c_float),
                ("sr_stop_theta", ctypes.c_double), ("stall_checks", ctypes.c_int),
                ("fold", ctypes.c_int), ("trace_checks", ctypes.c_int), ("fold_exit", ctypes.c_double),
                ("rng_streams", ctypes.c_int), ("persistent", ctypes.c_int), ("wait_budget_us", ctypes.c_int),
                ("wait_test_missing", ctypes.c_int)]


class Report(ctypes.Structure):
    """gf_report of include/gfix.h."""

    _fields_ = [("gff", ctypes.c_double), ("theta", ctypes.c_double), ("or_sweeps", ctypes.c_int),
                ("or_sweeps_fp64", ctypes.c_int), ("sa_sweeps", ctypes.c_int), ("converged", ctypes.c_int),
                ("chunks", ctypes.c_int), ("sr_sweeps", ctypes.c_int)]


SIGNATURES.update({
    "gf_create": (_c_int, [ctypes.POINTER(CtxParams), ctypes.POINTER(_vp)]),
    "gf_destroy": (_c_int, [_vp]),
    "gf_import": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int]),
    "gf_export": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int]),
    "gf_export_slices": (_c_int, [_vp, ctypes.POINTER(_c_int), _c_int, _vp, _c_int]),
    "gf_sweeps": (_c_int, [_vp, _c_int, _c_int, _c_float, _c_int, _c_int]),
    "gf_quality_all": (_c_int, [_vp, _dp, _dp]),
    "gf_reunitarize": (_c_int, [_vp]),
    "gf_set_storage": (_c_int, [_vp, _c_int]),
    "gf_fix": (_c_int, [_vp, ctypes.POINTER(Schedule), ctypes.POINTER(Report)]),
    "gf_kernel_launches": (_c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "gf_trace": (_c_int, [_vp, _c_int, _dp, _c_int, ctypes.POINTER(_c_int)]),
    "gf_autotune": (_c_int, [_vp, ctypes.POINTER(_c_int), ctypes.POINTER(_c_int)]),
    "gf_set_pass_shape": (_c_int, [_vp, _c_int, _c_int, _c_int]),
    "gf_set_pass_order": (_c_int, [_vp, _c_int, _c_int, _c_int]),
    "gf_set_pass_stages": (_c_int, [_vp, _c_int, _c_int]),
    "gf_instances": (_c_int, [_vp]),
})

_LIB = None


class GaugeFixError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status: int, func: str, message: str):
        super().__init__(f"{func} failed with status {status}: {message}")
        self.status = status


def lib() -> ctypes.CDLL:
    """Load libgfix.so (once) and attach the argument types."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m su3_ma_gauge_gpu_b200.build` "
                "(this package has no CPU fallback)")
        h = ctypes.CDLL(os.fspath(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = h
    return _LIB


def check(status: int, func: str) -> None:
    """Raise GaugeFixError for a non-zero status, with gf_last_error_string()."""
    if status != GF_OK:
        msg = lib().gf_last_error_string().decode(errors="replace")
        raise GaugeFixError(status, func, msg)


def size_arg(size) -> ctypes.Array:
    """(Nt, Nx, Ny, Nz) -> int32[4] for the C ABI."""
    if len(size) != 4:
        raise ValueError("size must have 4 entries (Nt, Nx, Ny, Nz)")
    return (ctypes.c_int32 * 4)(*[int(s) for s in size])
