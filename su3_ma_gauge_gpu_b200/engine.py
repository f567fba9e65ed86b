"""Batched, mixed-precision gauge fixing: the context-level C ABI from Python.

:class:`GaugeFixer` holds one or more lattices (gauge copies, uneven extents)
and runs the reference driver's per-copy schedule
(apps/LandauGaugeFixingSU3_4D.cu:185-271: random trafo, SA + micro, OR with
reprojection and checks) on all of them at once.  With ``mixed=True`` the bulk
sweeps run in FP32 until theta < ``switch_theta``, then each instance moves to
FP64 storage (reunitarised in FP64) for the polish to theta < ``precision``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, fields

import numpy as np

from . import _lib
from ._lib import check, lib

ALGOS = {"or": 0, "micro": 1, "sa": 2, "sr": 3, "random": 4}
GAUGES = {"landau": _lib.GF_LANDAU, "coulomb": _lib.GF_COULOMB, "mag": _lib.GF_MAG, "u1xu1": _lib.GF_U1XU1}


@dataclass
class Schedule:
    """Fields of gf_schedule; defaults are the reference's ProgramOptions defaults
    (apps/program_options/ProgramOptions.hxx:223-266) except where noted."""

    random_trafo: int = 0
    seed: int = 1
    rng_counter: int = 0
    sa_steps: int = 0
    sa_min: float = 0.01
    sa_max: float = 0.4
    sa_geometric: int = 0
    micro_updates: int = 3
    or_max_iter: int = 1000
    or_parameter: float = 1.7
    precision: float = 1e-7
    switch_theta: float = 1e-9
    check_precision: int = 100
    reproject: int = 100
    use_graphs: int = 1
    autotune: int = 1
    micro_every: int = 1
    sa_mode: int = 0
    sa_repeat: int = 1
    sa_slow_lo: float = 0.0
    sa_slow_hi: float = 0.0
    sa_slow_factor: float = 1.0
    sr_max_iter: int = 0
    sr_parameter: float = 1.7
    sr_stop_theta: float = 1e-6
    stall_checks: int = 5  # not in the reference (no mixed precision there); 0 turns it off
    fold: int = 1          # refine contexts: iterative refinement below switch_theta (0: FP64 sweeps)
    trace_checks: int = 0  # > 0: keep that many OR checks per instance for GaugeFixer.trace()
    fold_exit: float = 4.0  # fold mode: FP64 sweeps once the master's theta < fold_exit * precision
    rng_streams: int = 0    # 1: one Philox stream through the instances, as the apps draw it (no SR)
    persistent: int = 0     # 1: one cooperative launch per check chunk (plain FP64, mixed=True, Coulomb)
    wait_budget_us: int = 0  # persistent: bound of every grid-barrier wait (0: one second)
    wait_test_missing: int = 0  # persistent: arrivals that never come (tests of the bounded wait only)

    @classmethod
    def mag_app(cls, **kw) -> "Schedule":
        """The MAG app's schedule (apps/MAGaugeFixingSU3_4D.cu:222-333): SA do-while with 5 SA +
        micro sweeps per temperature and step/15 for T in [0.7, 0.88], then SR, then OR."""
        base = dict(sa_mode=2, sa_repeat=5, sa_slow_lo=0.7, sa_slow_hi=0.88, sa_slow_factor=15.0,
                    sr_max_iter=1000, sr_parameter=1.7, sr_stop_theta=1e-6)
        base.update(kw)
        return cls(**base)

    @classmethod
    def u1xu1_app(cls, **kw) -> "Schedule":
        """The U1xU1 app's SA do-while: step/15 for T in [2, 2.7]."""
        base = dict(sa_mode=2, sa_repeat=1, sa_slow_lo=2.0, sa_slow_hi=2.7, sa_slow_factor=15.0)
        base.update(kw)
        return cls(**base)

    def to_c(self) -> _lib.Schedule:
        s = _lib.Schedule()
        for f in fields(self):
            setattr(s, f.name, getattr(self, f.name))
        return s


@dataclass
class Report:
    gff: float
    theta: float
    or_sweeps: int
    or_sweeps_fp64: int
    sa_sweeps: int
    converged: bool
    chunks: int
    sr_sweeps: int = 0


def _real(a) -> int:
    dt = str(getattr(a, "dtype", ""))
    if "float64" in dt:
        return _lib.GF_FP64
    if "float32" in dt:
        return _lib.GF_FP32
    raise TypeError(f"unsupported field dtype {dt}")


class GaugeFixer:
    """A gf_ctx: ``sizes`` is a list of lattices (Nt, Nx, Ny, Nz).

    For gauge="coulomb" every lattice is fixed as Nt independent timeslices (instances);
    load/store take the lattice index and the GpuPatternTimeslice array of all its slices,
    reports and quality() are per timeslice."""

    def __init__(self, sizes, gauge="landau", mixed=True, stream=None):
        """mixed: False (FP64 only), True (FP32 storage, then FP64), or "refine" (FP64 master,
        FP32 working copy with the accumulated gauge transformation W applied to the master at
        the switch: the FP32 phase never moves the field off its gauge orbit; for Coulomb the W of a
        timeslice is the one it keeps in its temporal planes)."""
        self.sizes = [tuple(int(v) for v in s) for s in sizes]
        self.gauge = GAUGES[gauge] if isinstance(gauge, str) else int(gauge)
        arr = (ctypes.c_int32 * (4 * len(self.sizes)))(*[v for s in self.sizes for v in s])
        self._keep = arr
        mode = 2 if mixed in ("refine", 2) else (1 if mixed else 0)
        p = _lib.CtxParams(self.gauge, len(self.sizes), ctypes.cast(arr, ctypes.POINTER(ctypes.c_int32)),
                           mode, stream.cuda_stream if stream is not None else None)
        h = ctypes.c_void_p()
        check(lib().gf_create(ctypes.byref(p), ctypes.byref(h)), "gf_create")
        self._h = h
        self.mixed = mixed

    @property
    def ninstances(self) -> int:
        return lib().gf_instances(self._h)

    def load(self, i: int, U) -> None:
        """Import instance i from a GpuPattern array: CUDA tensor, or numpy array (host)."""
        if isinstance(U, np.ndarray):
            U = np.ascontiguousarray(U)
            check(lib().gf_import(self._h, i, _real(U), U.ctypes.data, 1), "gf_import")
        else:
            check(lib().gf_import(self._h, i, _real(U), U.data_ptr(), 0), "gf_import")

    def store(self, i: int, U) -> None:
        """Export instance i (reunitarised, row 2 rebuilt) into a GpuPattern array."""
        if isinstance(U, np.ndarray):
            assert U.flags.c_contiguous
            check(lib().gf_export(self._h, i, _real(U), U.ctypes.data, 1), "gf_export")
        else:
            check(lib().gf_export(self._h, i, _real(U), U.data_ptr(), 0), "gf_export")

    def store_slices(self, copy_of_slice, U) -> None:
        """Coulomb gauge copies: export the lattice whose timeslice t comes from copy copy_of_slice[t]."""
        tab = (ctypes.c_int * len(copy_of_slice))(*[int(a) for a in copy_of_slice])
        if isinstance(U, np.ndarray):
            assert U.flags.c_contiguous
            check(lib().gf_export_slices(self._h, tab, _real(U), U.ctypes.data, 1), "gf_export_slices")
        else:
            check(lib().gf_export_slices(self._h, tab, _real(U), U.data_ptr(), 0), "gf_export_slices")

    def sweeps(self, algo: str, n: int, param: float = 0.0, seed: int = 0, rng_counter: int = 0) -> None:
        check(lib().gf_sweeps(self._h, ALGOS[algo], n, param, seed, rng_counter), "gf_sweeps")

    def quality(self):
        n = self.ninstances
        g = (ctypes.c_double * n)()
        a = (ctypes.c_double * n)()
        check(lib().gf_quality_all(self._h, g, a), "gf_quality_all")
        return np.array(g[:]), np.array(a[:])

    def reunitarize(self) -> None:
        check(lib().gf_reunitarize(self._h), "gf_reunitarize")

    def to_fp64(self) -> None:
        check(lib().gf_set_storage(self._h, _lib.GF_FP64), "gf_set_storage")

    def fix(self, schedule: Schedule | None = None) -> list[Report]:
        s = (schedule or Schedule()).to_c()
        reps = (_lib.Report * self.ninstances)()
        check(lib().gf_fix(self._h, ctypes.byref(s), reps), "gf_fix")
        return [Report(r.gff, r.theta, r.or_sweeps, r.or_sweeps_fp64, r.sa_sweeps, bool(r.converged), r.chunks,
                       r.sr_sweeps) for r in reps]

    def trace(self, i: int) -> np.ndarray:
        """OR checks of instance i in the last fix with trace_checks > 0: rows (sweeps, precision
        of the check: 0 FP32 / 1 FP64 / 4 FP64 master after a fold, functional, theta)."""
        n = ctypes.c_int()
        check(lib().gf_trace(self._h, i, None, 0, ctypes.byref(n)), "gf_trace")
        m = n.value
        buf = np.zeros(4 * max(m, 1))
        if m:
            check(lib().gf_trace(self._h, i, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), m, ctypes.byref(n)),
                  "gf_trace")
        return buf[:4 * min(m, n.value)].reshape(-1, 4)

    def autotune(self):
        """Time the OR-pass launch shapes and keep the fastest; returns (fp32, fp64) choices."""
        a, b = ctypes.c_int(), ctypes.c_int()
        check(lib().gf_autotune(self._h, ctypes.byref(a), ctypes.byref(b)), "gf_autotune")
        return a.value, b.value

    def set_pass_shape(self, real: str, variant: int, warps: int = 4) -> None:
        r = _lib.GF_FP64 if real in ("fp64", "double") else _lib.GF_FP32
        check(lib().gf_set_pass_shape(self._h, r, variant, warps), "gf_set_pass_shape")

    def set_pass_order(self, real: str, alternate: bool, capped: bool = False) -> None:
        """Persistent passes: walk odd-parity passes backwards (L2 reuse between passes); capped:
        fewer registers for more resident warps."""
        r = _lib.GF_FP64 if real in ("fp64", "double") else _lib.GF_FP32
        check(lib().gf_set_pass_order(self._h, r, int(bool(alternate)), int(bool(capped))), "gf_set_pass_order")

    def set_pass_stages(self, real: str, stages: int) -> None:
        """Pipelined pass with 4 warps per block: cp.async stages per warp (2, or 3: two tiles in flight)."""
        r = _lib.GF_FP64 if real in ("fp64", "double") else _lib.GF_FP32
        check(lib().gf_set_pass_stages(self._h, r, stages), "gf_set_pass_stages")

    def kernel_launches(self) -> int:
        n = ctypes.c_longlong()
        check(lib().gf_kernel_launches(self._h, ctypes.byref(n)), "gf_kernel_launches")
        return n.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().gf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
