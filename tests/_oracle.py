"""ctypes access to the CPU oracle (oracle/liborc.so) and to the reference-pin
libraries (oracle/_ref/libref_pin_{f64,f32}.so) for the tests.

Test infrastructure only: the oracle is the checker, never the thing measured.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
ORACLE_SO = ORACLE_DIR / "liborc.so"
REF_DIR = ORACLE_DIR / "_ref"

LANDAU, COULOMB, MAG, U1XU1 = 0, 1, 2, 3
OR, MICRO, SA, SR, RANDOM = 0, 1, 2, 3, 4
GAUGES = {"landau": LANDAU, "coulomb": COULOMB, "mag": MAG, "u1xu1": U1XU1}
ALGOS = {"or": OR, "micro": MICRO, "sa": SA, "sr": SR, "random": RANDOM}

_P = ctypes.c_void_p
_u32 = ctypes.c_uint32


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def _size(size):
    return np.ascontiguousarray(size, dtype=np.int32)


_ORC = None


def oracle() -> ctypes.CDLL:
    """Load (building with make if needed) the C oracle."""
    global _ORC
    if _ORC is None:
        if not ORACLE_SO.exists():
            subprocess.run(["make", "-C", str(ORACLE_DIR), "liborc.so"], check=True, capture_output=True)
        _ORC = ctypes.CDLL(str(ORACLE_SO))
    return _ORC


def ref_pin(prec: str):
    """The reference's own site-update code compiled for the host, or None if not built."""
    p = REF_DIR / f"libref_pin_{prec}.so"
    return ctypes.CDLL(str(p)) if p.exists() else None


def volume(size) -> int:
    return int(np.prod(size))


def field_zeros(size, dtype=np.float64):
    return np.zeros(volume(size) * 72, dtype=dtype)


def sfx(a) -> str:
    return "f64" if a.dtype == np.float64 else "f32"


def set_hot(size, seed, counter, dtype=np.float64, nthreads=8):
    U = field_zeros(size, dtype)
    getattr(oracle(), "orc_set_hot_" + sfx(U))(_ptr(U), _ptr(_size(size)), _u32(seed), _u32(counter), nthreads)
    return U


def step(U, size, gauge, algo, parity, param=0.0, seed=0, counter=0, Udw=None, nthreads=8):
    """One parity pass in place (Udw: slice t-1 for Coulomb)."""
    getattr(oracle(), "orc_step_" + sfx(U))(_ptr(U), _ptr(Udw), _ptr(_size(size)), gauge, algo, parity,
                                            ctypes.c_float(param), _u32(seed), _u32(counter), nthreads)


def step_slices(U, size, gauge, algo, parity, t_begin, t_end, param=0.0, seed=0, counter=0, nthreads=8,
                rng_site_offset=0):
    """One parity pass over the sites of timeslices [t_begin, t_end) only, in place; site h draws
    its random numbers as site h + rng_site_offset."""
    half = volume(size) // size[0] // 2
    getattr(oracle(), "orc_step_range_at_" + sfx(U))(_ptr(U), None, _ptr(_size(size)), gauge, algo, parity,
                                                     ctypes.c_float(param), _u32(seed), _u32(counter),
                                                     ctypes.c_int64(t_begin * half), ctypes.c_int64(t_end * half),
                                                     ctypes.c_int64(rng_site_offset), nthreads)


def quality(U, size, gauge, stop_max=0, per_site=False, nthreads=8):
    V = volume(size)
    g, a = ctypes.c_double(), ctypes.c_double()
    gs = np.zeros(V) if per_site else None
    as_ = np.zeros(V) if per_site else None
    getattr(oracle(), "orc_quality_" + sfx(U))(_ptr(U), _ptr(_size(size)), gauge, stop_max, ctypes.byref(g),
                                               ctypes.byref(a), _ptr(gs), _ptr(as_), nthreads)
    if per_site:
        return g.value, a.value, gs, as_
    return g.value, a.value


def project(U, size, nthreads=8):
    getattr(oracle(), "orc_project_" + sfx(U))(_ptr(U), _ptr(_size(size)), nthreads)


class Schedule(ctypes.Structure):
    _fields_ = [("random_trafo", ctypes.c_int), ("sa_steps", ctypes.c_int), ("sa_min", ctypes.c_float),
                ("sa_max", ctypes.c_float), ("micro_updates", ctypes.c_int), ("or_max_iter", ctypes.c_int),
                ("or_parameter", ctypes.c_float), ("precision", ctypes.c_float),
                ("check_precision", ctypes.c_int), ("reproject", ctypes.c_int), ("seed", ctypes.c_uint32)]


class Result(ctypes.Structure):
    _fields_ = [("gff", ctypes.c_double), ("theta", ctypes.c_double), ("or_iterations", ctypes.c_int)]


def fix(U, size, gauge, sched: Schedule, counter=0, nthreads=8):
    c = _u32(counter)
    r = Result()
    getattr(oracle(), "orc_fix_" + sfx(U))(_ptr(U), _ptr(_size(size)), gauge, ctypes.byref(sched), ctypes.byref(c),
                                           ctypes.byref(r), nthreads)
    return r, c.value


class AppSchedule(ctypes.Structure):
    """orc_app_schedule of oracle/gf_oracle.h: the apps' per-copy loop for every gauge."""

    _fields_ = [("random_trafo", ctypes.c_int), ("sa_steps", ctypes.c_int), ("sa_min", ctypes.c_float),
                ("sa_max", ctypes.c_float), ("micro_updates", ctypes.c_int), ("sa_mode", ctypes.c_int),
                ("sa_repeat", ctypes.c_int), ("sa_slow_lo", ctypes.c_double), ("sa_slow_hi", ctypes.c_double),
                ("sa_slow_factor", ctypes.c_float), ("sr_max_iter", ctypes.c_int), ("sr_parameter", ctypes.c_float),
                ("sr_stop_theta", ctypes.c_double), ("or_max_iter", ctypes.c_int), ("or_parameter", ctypes.c_float),
                ("precision", ctypes.c_float), ("check_precision", ctypes.c_int), ("reproject", ctypes.c_int),
                ("seed", ctypes.c_uint32)]


class AppResult(ctypes.Structure):
    _fields_ = [("gff", ctypes.c_double), ("theta", ctypes.c_double), ("or_iterations", ctypes.c_int),
                ("sa_sweeps", ctypes.c_int), ("sr_iterations", ctypes.c_int)]


def app_schedule(**kw) -> AppSchedule:
    """An AppSchedule with the apps' defaults (apps/program_options/ProgramOptions.hxx:223-266)."""
    base = dict(random_trafo=0, sa_steps=0, sa_min=0.01, sa_max=0.4, micro_updates=0, sa_mode=0, sa_repeat=1,
                sa_slow_lo=0.0, sa_slow_hi=0.0, sa_slow_factor=1.0, sr_max_iter=0, sr_parameter=1.7,
                sr_stop_theta=1e-6, or_max_iter=1000, or_parameter=1.7, precision=1e-7, check_precision=100,
                reproject=100, seed=1)
    base.update(kw)
    return AppSchedule(**base)


def fix_app(U, size, gauge, sched: AppSchedule, counter=0, Udw=None, nthreads=8):
    """orc_fix_app in place on U (and Udw for Coulomb); returns (AppResult, counter after)."""
    c = _u32(counter)
    r = AppResult()
    getattr(oracle(), "orc_fix_app_" + sfx(U))(_ptr(U), _ptr(Udw), _ptr(_size(size)), gauge, ctypes.byref(sched),
                                               ctypes.byref(c), ctypes.byref(r), nthreads)
    return r, c.value


def fix_coulomb(U, size, sched: AppSchedule, counter=0, nthreads=8):
    """orc_fix_coulomb in place on the GpuPatternTimeslice array U; returns ([AppResult] per slice, counter)."""
    c = _u32(counter)
    res = (AppResult * int(size[0]))()
    getattr(oracle(), "orc_fix_coulomb_" + sfx(U))(_ptr(U), _ptr(_size(size)), ctypes.byref(sched), ctypes.byref(c),
                                                   res, nthreads)
    return list(res), c.value


# ---- the reference's own code on the host (oracle/_ref) ----------------------------------------
def ref_step(U, size, gauge, algo, parity, param=0.0, seed=0, counter=0, Udw=None):
    lib = ref_pin(sfx(U))
    rc = getattr(lib, "ref_step_" + sfx(U))(_ptr(U), _ptr(Udw), _ptr(_size(size)), gauge, algo, parity,
                                             ctypes.c_float(param), _u32(seed), _u32(counter))
    assert rc == 0


def ref_quality_sites(U, size, gauge):
    lib = ref_pin(sfx(U))
    V = volume(size)
    g = np.zeros(V)
    a = np.zeros(V)
    getattr(lib, "ref_quality_sites_" + sfx(U))(_ptr(U), _ptr(_size(size)), gauge, _ptr(g), _ptr(a))
    return g, a


def ref_project(U, size):
    getattr(ref_pin(sfx(U)), "ref_project_" + sfx(U))(_ptr(U), _ptr(_size(size)))


def ref_set_hot(size, seed, counter, dtype=np.float64):
    U = field_zeros(size, dtype)
    getattr(ref_pin(sfx(U)), "ref_set_hot_" + sfx(U))(_ptr(U), _ptr(_size(size)), _u32(seed), _u32(counter))
    return U


# ---- the reference's own CUDA kernels (oracle/_ref/libref_gpu_*.so, built by oracle/Makefile) -----
def refgpu(name: str):
    """Load oracle/_ref/<name> (the reference's kernels for one compile-time extent and precision,
    behind oracle/ref_gpu.cu's C entry points), or None if it was not built."""
    p = REF_DIR / name
    if not p.exists():
        return None
    lib = ctypes.CDLL(str(p))
    lib.refgpu_step.argtypes = [ctypes.c_int, ctypes.c_int, _P, _P, _P, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                ctypes.c_int]
    lib.refgpu_quality.argtypes = [ctypes.c_int, _P, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double)]
    lib.refgpu_project.argtypes = [ctypes.c_int, _P]
    if hasattr(lib, "refgpu_or_loop"):
        lib.refgpu_or_loop.argtypes = [ctypes.c_int, _P, _P, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_float)]
    return lib


def refgpu_config(lib):
    size = (ctypes.c_int * 4)()
    es = lib.refgpu_config(size)
    return tuple(size), es


def refgpu_neighbours(lib, size, timeslice=False) -> np.ndarray:
    """The reference's neighbour table (host array of int32) for the library's extents."""
    V = volume(size) if not timeslice else volume(size[1:])
    nn = np.zeros(8 * V, np.int32)
    lib.refgpu_neighbour_table(int(timeslice), nn.ctypes.data_as(_P))
    return nn


def refgpu_or_loop(lib, gauge, U_ptr, nn_ptr, omega=1.7, precision=1e-12, check=20, reproject=100,
                   max_iter=20000):
    """The apps' overrelaxation loop (apps/LandauGaugeFixingSU3_4D.cu:244-271) on the reference's
    kernels, in place on the device array at U_ptr; precision is passed as a float, as the apps
    hold it.  Returns (functional, theta, sweeps, milliseconds) of the last check."""
    g, a = ctypes.c_double(), ctypes.c_double()
    n, ms = ctypes.c_int(), ctypes.c_float()
    rc = lib.refgpu_or_loop(gauge, U_ptr, nn_ptr, ctypes.c_float(omega), ctypes.c_float(precision), check, reproject,
                            max_iter, ctypes.byref(g), ctypes.byref(a), ctypes.byref(n), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"refgpu_or_loop failed: {rc}")
    return g.value, a.value, n.value, ms.value


# ---- layout helpers (reference GpuPattern) -----------------------------------------------------
def links(U, size):
    """GpuPattern array -> complex array [mu][V][3][3]."""
    V = volume(size)
    a = U.reshape(4, 3, 3, 2, V).astype(np.float64)
    return np.transpose(a[..., 0, :] + 1j * a[..., 1, :], (0, 3, 1, 2))


def rows01_maxdiff(A, B, size):
    """max |A - B| over the stored rows 0,1 (what the sweep reads and writes)."""
    V = volume(size)
    a = A.reshape(4, 3, 3, 2, V)[:, :2].astype(np.float64)
    b = B.reshape(4, 3, 3, 2, V)[:, :2].astype(np.float64)
    return float(np.abs(a - b).max())
