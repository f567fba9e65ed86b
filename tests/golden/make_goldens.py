"""Generates tests/golden/reference_hashes.json from the reference's OWN code.

Run where the reference tree is present (``make -C oracle`` builds oracle/_ref/):

    python tests/golden/make_goldens.py

Every entry is the SHA-256 of what the reference code returns for a seeded input:
  * site updates, FP64, every gauge x algorithm, both parities
    (oracle/_ref/libref_pin_f64.so: GaugeFixingSubgroupStep.hxx + algorithms/*Update.hxx);
  * setHot, projectSU3 and the per-site gauge quality, FP64;
  * the bytes of the configuration files the reference's LinkFile / writeILDG / writeQCDSTAG
    write, and the array its readers load, with the GpuPattern memory pattern and with the
    Coulomb apps' GpuPatternTimeslice one (oracle/_ref/libref_io.so).
tests/test_golden.py recomputes the same with the oracle (no reference needed) and compares, so
the oracle stays pinned on machines without the reference tree.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "oracle"))

import _oracle as O  # noqa: E402
import gf_files as F  # noqa: E402

OUT = HERE / "reference_hashes.json"
SIZE4 = (4, 4, 4, 4)
SLICE = (1, 8, 8, 4)
FILE_SIZE = (4, 6, 4, 2)  # the extents libref_io.so is compiled for


def sha(a) -> str:
    if isinstance(a, np.ndarray):
        a = np.ascontiguousarray(a).tobytes()
    return hashlib.sha256(a).hexdigest()


def step_cases():
    """(name, gauge, algo, size, param) of the site-update cases."""
    out = []
    for gname, gauge in O.GAUGES.items():
        for aname, algo in O.ALGOS.items():
            size = SLICE if gauge == O.COULOMB else SIZE4
            param = 1.7 if algo == O.OR else (0.5 if algo == O.SR else 0.8)
            out.append((f"step/{gname}/{aname}", gauge, algo, size, param))
    return out


def run_steps(step_fn, gauge, algo, size, param):
    """Two parity passes from the seeded hot start; returns (U, Udw)."""
    U = O.set_hot(size, 3, 1, np.float64)
    Udw = O.set_hot(size, 4, 1, np.float64) if gauge == O.COULOMB else None
    for parity in (0, 1):
        step_fn(U, size, gauge, algo, parity, param, 11, 7 + parity, Udw=Udw)
    return U, Udw


def project_input():
    U = O.set_hot(SIZE4, 5, 2, np.float64)
    U += np.random.default_rng(0).standard_normal(U.shape) * 1e-3
    return U


FILE_TEXT = [("ildg-format", b"<?xml version=\"1.0\"?><ildgFormat>su3gauge 64 bit</ildgFormat>\0"),
             ("xlf-info", b"plaquette = 0.5876 beta = 6.0\0")]
HEADER = b"#header of a HEADERONLY configuration\n\x00\x01\x02\x03"


def file_inputs():
    """(U_in, U_out): the configuration put into the template file and the one written out."""
    return F.random_links(FILE_SIZE, 1), F.random_links(FILE_SIZE, 2)


def main():
    ref = O.ref_pin("f64")
    io_so = O.REF_DIR / "libref_io.so"
    if ref is None or not io_so.exists():
        sys.exit("oracle/_ref is not built: run `make -C oracle` where the reference tree is present")
    h = {}
    for name, gauge, algo, size, param in step_cases():
        U, Udw = run_steps(O.ref_step, gauge, algo, size, param)
        h[name] = sha(U) + ("" if Udw is None else "+" + sha(Udw))
    h["set_hot/f64"] = sha(O.ref_set_hot(SIZE4, 3, 1, np.float64))
    R = project_input()
    O.ref_project(R, SIZE4)
    h["project/f64"] = sha(R)
    for gname, gauge in O.GAUGES.items():
        size = SLICE if gauge == O.COULOMB else SIZE4
        g, a = O.ref_quality_sites(O.set_hot(size, 3, 1, np.float64), size, gauge)
        h[f"quality/{gname}"] = sha(g) + "+" + sha(a)

    io = ctypes.CDLL(str(io_so))
    dp = ctypes.POINTER(ctypes.c_double)
    Ua, Ub = file_inputs()
    V72 = Ua.size
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        cases = {  # name: (format code, reinterpret, template bytes)
            "plain_f64": (0, 1, F.payload_encode(Ua, FILE_SIZE, F.PLAIN)),
            "plain_f32": (0, 2, F.payload_encode(Ua, FILE_SIZE, F.PLAIN, np.float32)),
            "headeronly_f64": (1, 1, HEADER + F.payload_encode(Ua, FILE_SIZE, F.PLAIN)),
            "vogt_f64": (2, 1, F.vogt_header(FILE_SIZE, 8) + F.payload_encode(Ua, FILE_SIZE, F.PLAIN)),
        }
        for name, (fmt, reint, blob) in cases.items():
            (d / "in").write_bytes(blob)
            got = np.zeros(V72)
            rc = io.refio_linkfile(fmt, str(d / "in").encode(), str(d / "out").encode(), reint,
                                   got.ctypes.data_as(dp), Ub.ctypes.data_as(dp))
            assert rc == 0, (name, rc)
            h[f"file/{name}/read"] = sha(got)
            h[f"file/{name}/write"] = sha((d / "out").read_bytes())
        (d / "in").write_bytes(F.ildg_file(Ua, FILE_SIZE, FILE_TEXT))
        got = np.zeros(V72)
        io.refio_read_ildg(str(d / "in").encode(), got.ctypes.data_as(dp))
        h["file/ildg/read"] = sha(got)
        io.refio_write_ildg(str(d / "in").encode(), str(d / "out").encode(), Ub.ctypes.data_as(dp), 17)
        h["file/ildg/write"] = sha((d / "out").read_bytes())
        (d / "in").write_bytes(F.payload_encode(Ua, FILE_SIZE, F.QCDSTAG))
        got = np.zeros(V72)
        assert io.refio_read_qcdstag(str(d / "in").encode(), got.ctypes.data_as(dp)) == 0
        h["file/qcdstag/read"] = sha(got)
        io.refio_write_qcdstag(str(d / "out").encode(), Ub.ctypes.data_as(dp))
        h["file/qcdstag/write"] = sha((d / "out").read_bytes())
        # the Coulomb apps' memory pattern (GpuPatternTimeslice): reads and writes
        Tb = F.gpu_to_timeslice(Ub, FILE_SIZE)
        (d / "in").write_bytes(F.payload_encode(Ua, FILE_SIZE, F.PLAIN))
        got = np.zeros(V72)
        assert io.refio_linkfile_timeslice(0, str(d / "in").encode(), str(d / "out").encode(), 1,
                                           got.ctypes.data_as(dp), Tb.ctypes.data_as(dp)) == 0
        h["file/timeslice/plain/read"] = sha(got)
        h["file/timeslice/plain/write"] = sha((d / "out").read_bytes())
        (d / "in").write_bytes(F.ildg_file(Ua, FILE_SIZE, FILE_TEXT))
        got = np.zeros(V72)
        io.refio_read_ildg_timeslice(str(d / "in").encode(), got.ctypes.data_as(dp))
        h["file/timeslice/ildg/read"] = sha(got)
        io.refio_write_ildg_timeslice(str(d / "in").encode(), str(d / "out").encode(), Tb.ctypes.data_as(dp), 17)
        h["file/timeslice/ildg/write"] = sha((d / "out").read_bytes())
        (d / "in").write_bytes(F.payload_encode(Ua, FILE_SIZE, F.QCDSTAG))
        got = np.zeros(V72)
        assert io.refio_read_qcdstag_timeslice(str(d / "in").encode(), got.ctypes.data_as(dp)) == 0
        h["file/timeslice/qcdstag/read"] = sha(got)
        io.refio_write_qcdstag_timeslice(str(d / "out").encode(), Tb.ctypes.data_as(dp))
        h["file/timeslice/qcdstag/write"] = sha((d / "out").read_bytes())
    OUT.write_text(json.dumps(h, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(h)} hashes to {OUT}")


if __name__ == "__main__":
    main()
