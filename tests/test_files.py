"""Configuration files: gf_file_read / gf_file_write (GPU transcoder) against the oracle's
restatement of the formats (oracle/gf_files.py), which tests/test_golden.py pins to the
reference's own readers and writers.  Integer/byte work: everything is compared bit for bit.
"""
import numpy as np
import pytest

import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import gf_files as F  # noqa: E402

from su3_ma_gauge_gpu_b200 import GaugeFixError, files  # noqa: E402

SIZES = [(4, 6, 4, 2), (8, 6, 4, 10), (2, 2, 2, 2)]
FORMATS = {"plain": F.PLAIN, "headeronly": F.HEADERONLY, "vogt": F.VOGT, "ildg": F.ILDG, "qcdstag": F.QCDSTAG}
HEADER = b"opaque header\n\x00\xff"
TEXT = [("ildg-format", b"<ildgFormat>su3gauge</ildgFormat>\0"), ("xlf-info", b"beta = 6.0\0"),
        ("scidac-checksum", b"<checksum>0</checksum>\0")]


def _file_bytes(U, size, fmt, file_dtype=np.float64):
    if fmt == F.ILDG:
        return F.ildg_file(U, size, TEXT)
    body = F.payload_encode(U, size, fmt, file_dtype)
    if fmt == F.HEADERONLY:
        return HEADER + body
    if fmt == F.VOGT:
        return F.vogt_header(size, np.dtype(file_dtype).itemsize) + body
    return body


def test_timeslice_converter_matches_oracle():
    from su3_ma_gauge_gpu_b200 import synthetic as S

    for size in SIZES:
        U = F.random_links(size, 3)
        assert np.array_equal(S.gpupattern_to_timeslices(U, size), F.gpu_to_timeslice(U, size))


def test_python_api_argument_checks(tmp_path):
    with pytest.raises(ValueError):
        files.read_config(tmp_path / "x", "NOPE", (2, 2, 2, 2), np.zeros(72 * 16))
    with pytest.raises(ValueError):
        files.read_config(tmp_path / "x", "PLAIN", (2, 2, 2, 2), np.zeros(10))
    with pytest.raises(TypeError):
        files.read_config(tmp_path / "x", "PLAIN", (2, 2, 2, 2), np.zeros(72 * 16, np.float32))
    with pytest.raises(ValueError):
        files.LinkFile("ILDG")


@pytest.mark.gpu
@pytest.mark.parametrize("size", SIZES, ids=["x".join(map(str, s)) for s in SIZES])
@pytest.mark.parametrize("fname", list(FORMATS))
def test_read_matches_oracle(cuda, tmp_path, size, fname):
    torch = cuda
    fmt = FORMATS[fname]
    U = F.random_links(size, 11)
    path = tmp_path / "cfg"
    path.write_bytes(_file_bytes(U, size, fmt))
    dev = torch.empty(U.size, dtype=torch.float64, device="cuda")
    files.read_config(path, fmt, size, dev, "double", files.DOUBLE)
    assert np.array_equal(dev.cpu().numpy(), U)
    dev32 = torch.empty(U.size, dtype=torch.float32, device="cuda")
    files.read_config(path, fmt, size, dev32, "float", files.DOUBLE)
    assert np.array_equal(dev32.cpu().numpy(), U.astype(np.float32))
    host = np.zeros_like(U)
    files.read_config(path, fmt, size, host, "double", files.DOUBLE)  # host buffer
    assert np.array_equal(host, U)


@pytest.mark.gpu
@pytest.mark.parametrize("fname", ["plain", "headeronly", "vogt"])
def test_float_files(cuda, tmp_path, fname):
    torch = cuda
    fmt, size = FORMATS[fname], (4, 6, 4, 2)
    U = F.random_links(size, 12)
    path = tmp_path / "cfg"
    path.write_bytes(_file_bytes(U, size, fmt, np.float32))
    dev = torch.empty(U.size, dtype=torch.float64, device="cuda")
    files.read_config(path, fmt, size, dev, "double", files.FLOAT)
    assert np.array_equal(dev.cpu().numpy(), U.astype(np.float32).astype(np.float64))
    out = tmp_path / "out"
    files.write_config(out, fmt, size, dev, "double", files.FLOAT, template=path)
    assert out.read_bytes() == path.read_bytes()


@pytest.mark.gpu
@pytest.mark.parametrize("size", SIZES[:2], ids=["x".join(map(str, s)) for s in SIZES[:2]])
@pytest.mark.parametrize("fname", list(FORMATS))
def test_write_matches_oracle(cuda, tmp_path, size, fname):
    torch = cuda
    fmt = FORMATS[fname]
    Ua, Ub = F.random_links(size, 21), F.random_links(size, 22)
    tmpl = tmp_path / "template"
    tmpl.write_bytes(_file_bytes(Ua, size, fmt))
    out = tmp_path / "out"
    dev = torch.from_numpy(Ub).cuda()
    files.write_config(out, fmt, size, dev, "double", files.DOUBLE, template=tmpl, sa_steps=42)
    if fmt == F.ILDG:
        want = F.ildg_rewrite(tmpl.read_bytes(), Ub, size, 42)
    else:
        want = _file_bytes(Ub, size, fmt)
    assert out.read_bytes() == want
    # and back through the reader, from host memory this time
    back = np.zeros_like(Ub)
    files.read_config(out, fmt, size, back, "double", files.DOUBLE)
    assert np.array_equal(back, Ub)


@pytest.mark.gpu
@pytest.mark.parametrize("fname", ["plain", "headeronly", "ildg", "qcdstag"])
def test_timeslice_layout(cuda, tmp_path, fname):
    """GpuPatternTimeslice (the Coulomb apps' memory pattern): read, write back, and the array
    feeds a Coulomb context directly."""
    torch = cuda
    fmt, size = FORMATS[fname], (4, 6, 4, 2)
    U = F.random_links(size, 51)
    path = tmp_path / "cfg"
    path.write_bytes(_file_bytes(U, size, fmt))
    dev = torch.empty(U.size, dtype=torch.float64, device="cuda")
    files.read_config(path, fmt, size, dev, "double", files.DOUBLE, layout="timeslice")
    assert np.array_equal(dev.cpu().numpy(), F.gpu_to_timeslice(U, size))
    out = tmp_path / "out"
    files.write_config(out, fmt, size, dev, "double", files.DOUBLE, template=path, sa_steps=3, layout="timeslice")
    want = F.ildg_rewrite(path.read_bytes(), U, size, 3) if fmt == F.ILDG else path.read_bytes()
    assert out.read_bytes() == want


@pytest.mark.gpu
def test_coulomb_context_from_timeslice_file(cuda, tmp_path):
    """A configuration file read in the timeslice layout goes straight into a Coulomb context."""
    from su3_ma_gauge_gpu_b200 import synthetic as S
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    torch = cuda
    size = (4, 4, 4, 6)
    U, _ = S.smooth_config(size, 0.3, 7)
    path = tmp_path / "cfg.lime"
    path.write_bytes(F.ildg_file(U, size, TEXT))
    T = torch.empty(U.size, dtype=torch.float64, device="cuda")
    files.readILDG_timeslice(size, path, T)
    with GaugeFixer([size], gauge="coulomb", mixed=False) as gf:
        gf.load(0, T)
        g, a = gf.quality()
    import _oracle as O

    Ts = F.gpu_to_timeslice(U, size)
    Vs = int(np.prod(size[1:]))
    for t in range(size[0]):
        gq, aq = O.quality(Ts[t * 72 * Vs:(t + 1) * 72 * Vs].copy(), (1,) + size[1:], O.COULOMB)
        assert g[t] == pytest.approx(gq, rel=1e-12) and a[t] == pytest.approx(aq, rel=1e-10)


@pytest.mark.gpu
def test_linkfile_and_app_readers(cuda, tmp_path):
    """The reference-named entry points: LinkFile.load/save keeps the header; ILDG / QCDSTAG."""
    torch = cuda
    size = (4, 6, 4, 2)
    U = F.random_links(size, 31)
    src = tmp_path / "in.cfg"
    src.write_bytes(HEADER + F.payload_encode(U, size, F.PLAIN))
    lf = files.LinkFile("HEADERONLY", files.STANDARD)
    dev = torch.empty(U.size, dtype=torch.float64, device="cuda")
    assert lf.load(size, src, dev)
    assert lf.save(size, tmp_path / "out.cfg", dev)
    assert (tmp_path / "out.cfg").read_bytes() == src.read_bytes()
    (tmp_path / "in.lime").write_bytes(F.ildg_file(U, size, TEXT))
    files.readILDG(size, tmp_path / "in.lime", dev)
    files.writeILDG(size, tmp_path / "in.lime", tmp_path / "out.lime", dev, 5)
    assert (tmp_path / "out.lime").read_bytes() == F.ildg_rewrite(F.ildg_file(U, size, TEXT), U, size, 5)
    assert files.writeQCDSTAG(size, tmp_path / "q", dev)
    dev2 = torch.zeros_like(dev)
    assert files.readQCDSTAG(size, tmp_path / "q", dev2)
    assert torch.equal(dev, dev2)


@pytest.mark.gpu
def test_errors(cuda, tmp_path):
    torch = cuda
    size = (4, 6, 4, 2)
    U = F.random_links(size, 41)
    dev = torch.empty(U.size, dtype=torch.float64, device="cuda")
    with pytest.raises(GaugeFixError, match="cannot open"):
        files.read_config(tmp_path / "missing", "PLAIN", size, dev)
    (tmp_path / "short").write_bytes(F.payload_encode(U, size, F.PLAIN)[:-8])
    with pytest.raises(GaugeFixError, match="truncated"):
        files.read_config(tmp_path / "short", "PLAIN", size, dev)
    (tmp_path / "vogt").write_bytes(F.vogt_header((4, 6, 4, 4), 8) + F.payload_encode(U, size, F.PLAIN))
    with pytest.raises(GaugeFixError, match="VOGT extents"):
        files.read_config(tmp_path / "vogt", "VOGT", size, dev)
    (tmp_path / "vogt4").write_bytes(F.vogt_header(size, 4) + F.payload_encode(U, size, F.PLAIN))
    with pytest.raises(GaugeFixError, match="4-byte reals"):
        files.read_config(tmp_path / "vogt4", "VOGT", size, dev, reinterpret=files.DOUBLE)
    (tmp_path / "lime").write_bytes(F.ildg_file(F.random_links((4, 6, 4, 4), 1), (4, 6, 4, 4), TEXT))
    with pytest.raises(GaugeFixError, match="ildg-binary-data has"):
        files.read_config(tmp_path / "lime", "ILDG", size, dev)
    (tmp_path / "nolime").write_bytes(b"\0" * 200)
    with pytest.raises(GaugeFixError, match="magic"):
        files.read_config(tmp_path / "nolime", "ILDG", size, dev)
    (tmp_path / "nobin").write_bytes(b"".join(F.lime_record(t, d, i == 0, i == 1) for i, (t, d) in enumerate(TEXT[:2])))
    with pytest.raises(GaugeFixError, match="no ildg-binary-data"):
        files.read_config(tmp_path / "nobin", "ILDG", size, dev)
    with pytest.raises(GaugeFixError):
        files.read_config(tmp_path / "x", "PLAIN", (3, 6, 4, 2), torch.empty(72 * 144, dtype=torch.float64,
                                                                              device="cuda"))
