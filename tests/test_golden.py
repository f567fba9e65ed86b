"""The oracle against the committed golden hashes of the reference's own outputs.

tests/golden/reference_hashes.json is made by tests/golden/make_goldens.py from the reference's
code (oracle/_ref); here the oracle recomputes every case without the reference and must hash
identically -- FP64 site updates, setHot, projectSU3, per-site quality, and the configuration
files written / read by the reference's LinkFile, writeILDG / readILDG and writeQCDSTAG /
readQCDSTAG.
"""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import _oracle as O

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
sys.path.insert(0, str(HERE.parent / "oracle"))

import gf_files as F  # noqa: E402
import make_goldens as G  # noqa: E402

GOLD = json.loads((HERE / "golden" / "reference_hashes.json").read_text())


def sha(a) -> str:
    if isinstance(a, np.ndarray):
        a = np.ascontiguousarray(a).tobytes()
    return hashlib.sha256(a).hexdigest()


@pytest.mark.parametrize("case", G.step_cases(), ids=[c[0] for c in G.step_cases()])
def test_oracle_step_hash(case):
    name, gauge, algo, size, param = case
    U, Udw = G.run_steps(O.step, gauge, algo, size, param)
    assert sha(U) + ("" if Udw is None else "+" + sha(Udw)) == GOLD[name]


def test_oracle_set_hot_project_quality_hashes():
    assert sha(O.set_hot(G.SIZE4, 3, 1, np.float64)) == GOLD["set_hot/f64"]
    U = G.project_input()
    O.project(U, G.SIZE4)
    assert sha(U) == GOLD["project/f64"]
    for gname, gauge in O.GAUGES.items():
        size = G.SLICE if gauge == O.COULOMB else G.SIZE4
        _, _, g, a = O.quality(O.set_hot(size, 3, 1, np.float64), size, gauge, per_site=True)
        assert sha(g) + "+" + sha(a) == GOLD[f"quality/{gname}"], gname


def test_file_formats_hash():
    Ua, Ub = G.file_inputs()
    S = G.FILE_SIZE
    f32 = Ua.astype(np.float32).astype(np.float64)
    assert sha(Ua) == GOLD["file/plain_f64/read"] == GOLD["file/headeronly_f64/read"] == GOLD["file/vogt_f64/read"]
    assert sha(Ua) == GOLD["file/ildg/read"] == GOLD["file/qcdstag/read"]
    assert sha(f32) == GOLD["file/plain_f32/read"]
    # the readers of the oracle recover the same arrays from the template files
    assert sha(F.payload_decode(F.payload_encode(Ua, S, F.PLAIN), S, F.PLAIN)) == GOLD["file/plain_f64/read"]
    assert sha(F.payload_decode(F.payload_encode(Ua, S, F.ILDG), S, F.ILDG)) == GOLD["file/ildg/read"]
    assert sha(F.payload_decode(F.payload_encode(Ua, S, F.QCDSTAG), S, F.QCDSTAG)) == GOLD["file/qcdstag/read"]
    # what the reference writes
    assert sha(F.payload_encode(Ub, S, F.PLAIN)) == GOLD["file/plain_f64/write"]
    assert sha(F.payload_encode(Ub, S, F.PLAIN, np.float32)) == GOLD["file/plain_f32/write"]
    assert sha(G.HEADER + F.payload_encode(Ub, S, F.PLAIN)) == GOLD["file/headeronly_f64/write"]
    assert sha(F.vogt_header(S, 8) + F.payload_encode(Ub, S, F.PLAIN)) == GOLD["file/vogt_f64/write"]
    tmpl = F.ildg_file(Ua, S, G.FILE_TEXT)
    assert sha(F.ildg_rewrite(tmpl, Ub, S, 17)) == GOLD["file/ildg/write"]
    assert sha(F.payload_encode(Ub, S, F.QCDSTAG)) == GOLD["file/qcdstag/write"]
    # GpuPatternTimeslice (Coulomb apps): same files, the arrays in timeslice order
    Ta = F.gpu_to_timeslice(Ua, S)
    for fmt in ("plain", "ildg", "qcdstag"):
        assert sha(Ta) == GOLD[f"file/timeslice/{fmt}/read"], fmt
    assert GOLD["file/timeslice/plain/write"] == GOLD["file/plain_f64/write"]
    assert GOLD["file/timeslice/ildg/write"] == GOLD["file/ildg/write"]
    assert GOLD["file/timeslice/qcdstag/write"] == GOLD["file/qcdstag/write"]
    assert np.array_equal(F.timeslice_to_gpu(Ta, S), Ua)
