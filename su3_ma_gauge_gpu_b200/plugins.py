"""Python mirror of the reference's gauge-fixing plugin interface.

cuLGT drives its sweeps through classes of static launch wrappers:
``LandauKernelsSU3``, ``CoulombKernelsSU3``, ``MAGKernelsSU3``, ``U1xU1KernelsSU3``
(gaugefixing/*KernelsSU3.hxx), ``CommonKernelsSU3`` (CommonKernelsSU3.hxx) and
``GaugeFixingStats`` (GaugeFixingStats.hxx).  This module keeps those names,
method names, argument order and meaning on top of the C ABI, so a driver
written against the reference reads the same.  Differences, all forced by the
reference's compile-time configuration: the lattice extents and precision are
given to the constructor (the reference bakes them in with ``-D_X_ -D_T_`` and
``-DDOUBLEPRECISION``); the launch geometry ``(a, b)`` and the neighbour table
``nnt`` are accepted and ignored (neighbours are computed on the fly).

Fields are CUDA tensors (or raw device pointers) in the reference GpuPattern
layout, ``V*4*3*3*2`` reals.  Every call goes to ``libgfix.so``; failures raise
:class:`~su3_ma_gauge_gpu_b200._lib.GaugeFixError`.
"""
from __future__ import annotations

import ctypes

from . import _lib
from ._lib import check, lib, size_arg


def _real_code(precision) -> int:
    if precision in ("double", "float64", "fp64", _lib.GF_FP64):
        return _lib.GF_FP64
    if precision in ("float", "float32", "fp32", _lib.GF_FP32):
        return _lib.GF_FP32
    raise ValueError(f"unknown precision {precision!r}")


def device_ptr(x, real: int | None = None) -> int:
    """Device address of a CUDA tensor (checked dtype/contiguity) or an int pointer."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if not getattr(x, "is_cuda", False):
        raise TypeError("field must be a CUDA tensor or a device pointer")
    if not x.is_contiguous():
        raise ValueError("field tensor must be contiguous")
    if real is not None:
        want = "torch.float64" if real == _lib.GF_FP64 else "torch.float32"
        if str(x.dtype) != want:
            raise TypeError(f"field dtype {x.dtype} does not match precision {want}")
    return x.data_ptr()


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


class _GaugeKernels:
    """Shared implementation of the four gauge plugins (LandauKernelsSU3.hxx:55-106)."""

    GAUGE = _lib.GF_LANDAU
    Ndim = 4
    Nc = 3

    def __init__(self, size, precision="double", stream=None):
        self.size = tuple(int(s) for s in size)
        self.real = _real_code(precision)
        self.stream = stream
        self._size = size_arg(self.size)

    def initCacheConfig(self):
        """No-op: the L1/shared split is chosen by the sm_100a kernels themselves."""

    def _step(self, fn, U, Udw, parity, *extra):
        f = getattr(lib(), fn)
        st = f(self.GAUGE, self.real, device_ptr(U, self.real), device_ptr(Udw, self.real), self._size,
               int(bool(parity)), *extra, _stream_ptr(self.stream))
        check(st, fn)

    def orStep(self, a, b, U, nnt, parity, orParameter):
        self._step("gf_or_step", U, None, parity, ctypes.c_float(orParameter))

    def microStep(self, a, b, U, nnt, parity):
        self._step("gf_micro_step", U, None, parity)

    def saStep(self, a, b, U, nnt, parity, temperature, rngSeed, rngCounter):
        self._step("gf_sa_step", U, None, parity, ctypes.c_float(temperature), int(rngSeed), int(rngCounter))

    def randomTrafo(self, a, b, U, nnt, parity, rngSeed, rngCounter):
        self._step("gf_random_trafo", U, None, parity, int(rngSeed), int(rngCounter))

    def generateGaugeQualityPerSite(self, a, b, U, dGff, dA):
        st = lib().gf_quality_per_site(self.GAUGE, self.real, device_ptr(U, self.real), self._size,
                                       device_ptr(dGff), device_ptr(dA), _stream_ptr(self.stream))
        check(st, "gf_quality_per_site")

    def getGaugeQualityPrefactorA(self):
        return lib().gf_quality_prefactor_a(self.GAUGE)

    def getGaugeQualityPrefactorGff(self):
        return lib().gf_quality_prefactor_gff(self.GAUGE)

    def restoreThirdLine(self, a, b, U, nnt):
        check(lib().gf_project_su3(self.real, device_ptr(U, self.real), self._size, _stream_ptr(self.stream)),
              "gf_project_su3")


class LandauKernelsSU3(_GaugeKernels):
    """gaugefixing/LandauKernelsSU3.hxx:55-106."""

    GAUGE = _lib.GF_LANDAU


class U1xU1KernelsSU3(_GaugeKernels):
    """gaugefixing/U1xU1KernelsSU3.hxx:55-106."""

    GAUGE = _lib.GF_U1XU1


class MAGKernelsSU3(_GaugeKernels):
    """gaugefixing/MAGKernelsSU3.hxx:57-111 (adds srStep)."""

    GAUGE = _lib.GF_MAG

    def srStep(self, a, b, U, nnt, parity, srParameter, rngSeed, rngCounter):
        self._step("gf_sr_step", U, None, parity, ctypes.c_float(srParameter), int(rngSeed), int(rngCounter))


class CoulombKernelsSU3(_GaugeKernels):
    """gaugefixing/CoulombKernelsSU3.hxx:53-101: one timeslice ``UtUp`` plus slice t-1 ``UtDw``.

    ``size`` is the timeslice lattice ``(1, Nx, Ny, Nz)`` (the reference's SIZE_TIMESLICE).
    """

    GAUGE = _lib.GF_COULOMB

    def orStep(self, a, b, UtUp, UtDw, nnt, parity, orParameter):
        self._step("gf_or_step", UtUp, UtDw, parity, ctypes.c_float(orParameter))

    def microStep(self, a, b, UtUp, UtDw, nnt, parity):
        self._step("gf_micro_step", UtUp, UtDw, parity)

    def saStep(self, a, b, UtUp, UtDw, nnt, parity, temperature, rngSeed, rngCounter):
        self._step("gf_sa_step", UtUp, UtDw, parity, ctypes.c_float(temperature), int(rngSeed), int(rngCounter))

    def randomTrafo(self, a, b, UtUp, UtDw, nnt, parity, rngSeed, rngCounter):
        self._step("gf_random_trafo", UtUp, UtDw, parity, int(rngSeed), int(rngCounter))


class CommonKernelsSU3:
    """gaugefixing/CommonKernelsSU3.hxx:38-61 (projectSU3, setHot)."""

    def __init__(self, size, precision="double", stream=None):
        self.size = tuple(int(s) for s in size)
        self.real = _real_code(precision)
        self.stream = stream
        self._size = size_arg(self.size)

    def initCacheConfig(self):
        """No-op (see _GaugeKernels.initCacheConfig)."""

    def projectSU3(self, a, b, U, ptrToDeviceSize=None):
        check(lib().gf_project_su3(self.real, device_ptr(U, self.real), self._size, _stream_ptr(self.stream)),
              "gf_project_su3")

    def setHot(self, a, b, U, ptrToDeviceSize, rngSeed, rngCounter):
        check(lib().gf_set_hot(self.real, device_ptr(U, self.real), self._size, int(rngSeed), int(rngCounter),
                               _stream_ptr(self.stream)), "gf_set_hot")


class GaugeFixingStats:
    """gaugefixing/GaugeFixingStats.hxx:55-232: functional and theta of a field.

    ``GaugeFixingStats(U, size, GType, ma)`` mirrors the template
    ``GaugeFixingStats<Ndim, Nc, GType, ma>(U, size)``; ``GType`` is one of the
    plugin classes above (only its gauge is used) and ``ma`` is ``"AVERAGE"`` or
    ``"MAX"``.
    """

    def __init__(self, U, size, GType=LandauKernelsSU3, ma="AVERAGE", precision="double", stream=None):
        self.U = U
        self.real = _real_code(precision)
        self.stream = stream
        stop = _lib.GF_AVERAGE if ma in ("AVERAGE", _lib.GF_AVERAGE) else _lib.GF_MAX
        h = ctypes.c_void_p()
        check(lib().gf_stats_create(GType.GAUGE, self.real, size_arg(size), stop, ctypes.byref(h)),
              "gf_stats_create")
        self._h = h
        self.currentGff = 0.0
        self.currentA = 0.0

    def setPointer(self, U):
        self.U = U

    def generateGaugeQuality(self):
        g, a = ctypes.c_double(), ctypes.c_double()
        check(lib().gf_stats_generate(self._h, device_ptr(self.U, self.real), _stream_ptr(self.stream),
                                      ctypes.byref(g), ctypes.byref(a)), "gf_stats_generate")
        self.currentGff, self.currentA = g.value, a.value

    def getCurrentGff(self):
        return self.currentGff

    def getCurrentA(self):
        return self.currentA

    def close(self):
        if getattr(self, "_h", None):
            lib().gf_stats_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
