"""Configuration files: the reference's LinkFile and app readers over gf_file_read / gf_file_write.

The reference loads a configuration with ``LinkFile<FileType, Standard, Gpu, Site>(reinterpret)``
(lattice/LinkFile.hxx:57-67) for the PLAIN, HEADERONLY and VOGT file types, and with the free
functions ``readILDG`` / ``writeILDG`` (apps/ildg.cpp) and ``readQCDSTAG`` / ``writeQCDSTAG``
(apps/qcdstag.cpp) for the other two; the drivers pick one by the ``fType`` option
(apps/LandauGaugeFixingSU3_4D.cu:119-160).  This module keeps those names and argument meanings.
The transcoding runs on the GPU (one pass over the payload) instead of element by element on the
host.  Fields are CUDA tensors or host numpy arrays in the GpuPattern layout, or in the
GpuPatternTimeslice layout (``layout="timeslice"``) the Coulomb drivers use
(``LinkFile<FileType, Standard, GpuPatternTimeslice, Site>``, ``readILDG_timeslice``,
``readQCDSTAG_timeslice``); the extents are passed explicitly where the reference takes them from
its compile-time constants.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib, size_arg
from .plugins import _real_code, _stream_ptr

PLAIN, HEADERONLY, VOGT, ILDG, QCDSTAG = (_lib.GF_FILE_PLAIN, _lib.GF_FILE_HEADERONLY, _lib.GF_FILE_VOGT,
                                          _lib.GF_FILE_ILDG, _lib.GF_FILE_QCDSTAG)
# filetypes/filetype_typedefs.h: how the reals on file are read (STANDARD = as the build's Real)
STANDARD, DOUBLE, FLOAT = "STANDARD", "DOUBLE", "FLOAT"

_FORMATS = {"PLAIN": PLAIN, "HEADERONLY": HEADERONLY, "VOGT": VOGT, "ILDG": ILDG, "QCDSTAG": QCDSTAG}
_LAYOUTS = {"gpu": _lib.GF_LAYOUT_GPU, "timeslice": _lib.GF_LAYOUT_TIMESLICE}


def _layout_code(layout) -> int:
    if layout in _LAYOUTS:
        return _LAYOUTS[layout]
    if layout in _LAYOUTS.values():
        return int(layout)
    raise ValueError(f"unknown layout {layout!r} (gpu or timeslice)")


def _format_code(ftype) -> int:
    if isinstance(ftype, str):
        try:
            return _FORMATS[ftype.upper()]
        except KeyError:
            raise ValueError(f"unknown file type {ftype!r}") from None
    if ftype in _FORMATS.values():
        return int(ftype)
    raise ValueError(f"unknown file type {ftype!r}")


def _field(U, real: int, writable: bool):
    """(pointer, on_device) of a CUDA tensor or a C-contiguous numpy array of the right dtype."""
    want = np.float64 if real == _lib.GF_FP64 else np.float32
    if getattr(U, "is_cuda", False):
        if not U.is_contiguous() or U.element_size() != np.dtype(want).itemsize or not U.is_floating_point():
            raise TypeError("field tensor must be contiguous and of the requested precision")
        return U.data_ptr(), 1
    if not isinstance(U, np.ndarray) or U.dtype != want or not U.flags.c_contiguous:
        raise TypeError(f"field must be a CUDA tensor or a C-contiguous numpy array of {np.dtype(want)}")
    if writable and not U.flags.writeable:
        raise ValueError("field array is read-only")
    return U.ctypes.data, 0


def _check_len(U, size):
    n = 72 * int(np.prod(size))
    got = U.numel() if hasattr(U, "numel") else U.size
    if got != n:
        raise ValueError(f"field has {got} reals, the lattice needs {n}")


def read_config(path, ftype, size, U, precision="double", reinterpret=STANDARD, stream=None, layout="gpu"):
    """Load a configuration of file type ``ftype`` into U (GpuPattern or GpuPatternTimeslice order)."""
    real = _real_code(precision)
    file_real = real if reinterpret == STANDARD else _real_code("double" if reinterpret == DOUBLE else "float")
    _check_len(U, size)
    ptr, on_dev = _field(U, real, True)
    check(lib().gf_file_read(str(path).encode(), _format_code(ftype), file_real, size_arg(size), real,
                             _layout_code(layout), ctypes.c_void_p(ptr), on_dev, _stream_ptr(stream)), "gf_file_read")


def write_config(path, ftype, size, U, precision="double", reinterpret=STANDARD, template=None, sa_steps=0,
                 stream=None, layout="gpu"):
    """Save U to ``path``.  HEADERONLY copies its header from ``template``; ILDG copies every other
    record of ``template`` and appends the SA step count to its xlf-info record."""
    real = _real_code(precision)
    file_real = real if reinterpret == STANDARD else _real_code("double" if reinterpret == DOUBLE else "float")
    _check_len(U, size)
    ptr, on_dev = _field(U, real, False)
    tmpl = None if template is None else str(template).encode()
    check(lib().gf_file_write(str(path).encode(), _format_code(ftype), file_real, size_arg(size), real,
                              _layout_code(layout), ctypes.c_void_p(ptr), on_dev, tmpl, int(sa_steps),
                              _stream_ptr(stream)), "gf_file_write")


class LinkFile:
    """``LinkFile<FileType, Standard, Gpu, Site>`` (lattice/LinkFile.hxx:57-67).

    ``load`` remembers the file's header (HEADERONLY) so that ``save`` writes it back, like the
    reference's FileType member object."""

    def __init__(self, ftype, reinterpret=STANDARD, precision="double", layout="gpu"):
        """layout: "gpu" (MemoryPattern = GpuPattern) or "timeslice" (GpuPatternTimeslice)."""
        self.ftype = _format_code(ftype)
        if self.ftype not in (PLAIN, HEADERONLY, VOGT):
            raise ValueError("LinkFile handles PLAIN, HEADERONLY and VOGT; use readILDG / readQCDSTAG")
        self.reinterpret = reinterpret
        self.precision = precision
        self.layout = _layout_code(layout)
        self._template = None

    def load(self, size, filename, U, stream=None) -> bool:
        read_config(filename, self.ftype, size, U, self.precision, self.reinterpret, stream, self.layout)
        self._template = filename
        return True

    def save(self, size, filename, U, stream=None) -> bool:
        write_config(filename, self.ftype, size, U, self.precision, self.reinterpret, self._template, 0, stream,
                     self.layout)
        return True


def readILDG(size, file_name, U, precision="double", stream=None):
    """apps/ildg.cpp:26-97."""
    read_config(file_name, ILDG, size, U, precision, DOUBLE, stream)


def writeILDG(size, file_name, output_name, U, steps, precision="double", stream=None):
    """apps/ildg.cpp:99-238: the records of ``file_name`` with U as the binary data."""
    write_config(output_name, ILDG, size, U, precision, DOUBLE, file_name, steps, stream)


def readQCDSTAG(size, file_name, U, precision="double", stream=None) -> bool:
    """apps/qcdstag.cpp:17-67."""
    read_config(file_name, QCDSTAG, size, U, precision, DOUBLE, stream)
    return True


def writeQCDSTAG(size, output_name, U, precision="double", stream=None) -> bool:
    """apps/qcdstag.cpp:69-121."""
    write_config(output_name, QCDSTAG, size, U, precision, DOUBLE, None, 0, stream)
    return True


def readILDG_timeslice(size, file_name, U, precision="double", stream=None):
    """apps/ildg.cpp:240-310 (GpuPatternTimeslice)."""
    read_config(file_name, ILDG, size, U, precision, DOUBLE, stream, "timeslice")


def writeILDG_timeslice(size, file_name, output_name, U, steps, precision="double", stream=None):
    """apps/ildg.cpp:312-451."""
    write_config(output_name, ILDG, size, U, precision, DOUBLE, file_name, steps, stream, "timeslice")


def readQCDSTAG_timeslice(size, file_name, U, precision="double", stream=None) -> bool:
    """apps/qcdstag.cpp:123-173."""
    read_config(file_name, QCDSTAG, size, U, precision, DOUBLE, stream, "timeslice")
    return True


def writeQCDSTAG_timeslice(size, output_name, U, precision="double", stream=None) -> bool:
    """apps/qcdstag.cpp:175-227."""
    write_config(output_name, QCDSTAG, size, U, precision, DOUBLE, None, 0, stream, "timeslice")
    return True
