"""The batched driver (su3_ma_gauge_gpu_b200.apps): options, file names, copies, CSV, best copy."""
import sys
from pathlib import Path

import numpy as np
import pytest

import _oracle as O

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import gf_files as F  # noqa: E402

from su3_ma_gauge_gpu_b200 import apps  # noqa: E402


def test_options_and_file_names(tmp_path):
    cfg = tmp_path / "gf.cfg"
    cfg.write_text("# a driver config\nfbasename = conf_\nfending = .dat\nfnumberformat = 3\n"
                   "fstartnumber = 5\nfstepnumber = 2\nnconf = 3\ngaugecopies = 4\nrandomtrafo = false\n"
                   "precision = 1e-12\noutput_conf = out/\n")
    o = apps.ProgramOptions.from_config_file(cfg, seed=9)
    assert (o.gaugecopies, o.randomtrafo, o.seed, o.precision) == (4, False, 9, 1e-12)
    it = apps.FileIterator(o)
    assert it.ids() == [5, 7, 9]
    assert it.filename(7) == "conf_007.dat"
    assert it.output_filename(7) == "out/gaugefixed_007"
    assert it.output_functional(7) == "functional_007"
    bad = tmp_path / "bad.cfg"
    bad.write_text("nosuchoption = 1\n")
    with pytest.raises(ValueError):
        apps.ProgramOptions.from_config_file(bad)
    s = apps.schedule_for("mag", o)
    assert (s.sa_mode, s.sa_repeat, s.sr_max_iter) == (2, 5, 1000)
    assert s.precision == float(np.float32(1e-12))  # the reference keeps precision as a float


@pytest.mark.gpu
def test_landau_copies_best_copy_written(cuda, tmp_path, monkeypatch):
    from su3_ma_gauge_gpu_b200 import synthetic as S

    monkeypatch.chdir(tmp_path)
    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 21)
    Path("conf_0.bin").write_bytes(F.payload_encode(U, size, F.PLAIN))
    o = apps.ProgramOptions(ftype="PLAIN", fbasename="conf_", fending=".bin", gaugecopies=3, randomtrafo=True,
                            sasteps=0, ormaxiter=3000, precision=1e-12, checkprecision=20, microupdates=0)
    res = apps.run("landau", size, o)
    assert len(res) == 1
    r = res[0]
    csv = Path("functional_0").read_text().splitlines()
    assert csv[0] == "copy,functional" and len(csv) == 4
    Fs = [float(line.split(",")[1]) for line in csv[1:]]
    assert r.best_copy == int(np.argmax(Fs))
    assert max(r.thetas) < 1e-12
    out = np.frombuffer(Path("gaugefixed_0").read_bytes(), dtype=np.float64)
    back = F.payload_decode(out.tobytes(), size, F.PLAIN)
    g, a = O.quality(back, size, O.LANDAU)[:2]
    assert g == pytest.approx(Fs[r.best_copy], rel=1e-12)
    assert a < 1e-12
