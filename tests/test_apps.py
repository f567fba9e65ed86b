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


@pytest.mark.gpu
def test_reference_copy_sequence_matches_the_apps_loop(cuda, tmp_path, monkeypatch):
    """copies="reference" replays the Landau app's copy loop: each copy starts from the best copy so
    far and one Philox counter runs through the copies' random transformations and SA sweeps.  The
    oracle's restatement of the app's per-copy body (orc_fix_app), driven the same way, gives the
    same per-copy functionals (1e-10), the same best copy and the same written configuration."""
    from su3_ma_gauge_gpu_b200 import synthetic as S

    monkeypatch.chdir(tmp_path)
    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 23)
    Path("conf_0.bin").write_bytes(F.payload_encode(U, size, F.PLAIN))
    o = apps.ProgramOptions(ftype="PLAIN", fbasename="conf_", fending=".bin", gaugecopies=3, randomtrafo=True,
                            sasteps=4, samin=0.05, samax=0.5, microupdates=1, ormaxiter=3000, precision=1e-12,
                            checkprecision=20, seed=5)
    r = apps.run("landau", size, o, copies="reference")[0]
    prec = float(np.float32(1e-12))
    sch = O.app_schedule(random_trafo=1, sa_steps=4, sa_min=0.05, sa_max=0.5, micro_updates=1, or_max_iter=3000,
                         precision=prec, check_precision=20, reproject=100, seed=5)
    host, best_f, best, counter, fs = U.copy(), 0.0, 0, 0, []
    for c in range(3):
        X = host.copy()
        res, counter = O.fix_app(X, size, O.LANDAU, sch, counter=counter)
        fs.append(res.gff)
        if res.gff > best_f:
            best_f, best, host = res.gff, c, X
    assert r.functionals == pytest.approx(fs, rel=1e-10)
    assert r.best_copy == best
    out = F.payload_decode(Path("gaugefixed_0").read_bytes(), size, F.PLAIN)
    assert np.abs(out - host).max() < 1e-9


@pytest.mark.gpu
def test_coulomb_best_copy_per_timeslice(cuda, tmp_path, monkeypatch):
    """Coulomb with several gauge copies keeps, timeslice by timeslice, the copy with the largest
    functional (apps/CoulombGaugeFixingSU3_4D.cu:303-311).  The written configuration has, in every
    slice, that copy's spatial links and the best functional, and it is a gauge transform of the
    input: every plaquette is unchanged (its temporal links join W of different copies)."""
    from su3_ma_gauge_gpu_b200 import synthetic as S
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    monkeypatch.chdir(tmp_path)
    size = (4, 4, 4, 6)
    full, _ = S.smooth_config(size, 0.5, 27)
    Path("conf_0.bin").write_bytes(F.payload_encode(full, size, F.PLAIN))  # files hold the StandardPattern
    o = apps.ProgramOptions(ftype="PLAIN", fbasename="conf_", fending=".bin", gaugecopies=3, randomtrafo=True,
                            sasteps=0, ormaxiter=4000, precision=1e-12, checkprecision=20, microupdates=0)
    r = apps.run("coulomb", size, o)[0]
    lines = Path("functional_0").read_text().splitlines()[1:]
    g = np.zeros((3, size[0]))
    for line in lines:
        c, t, f = line.split(",")
        g[int(c), int(t)] = float(f)
    out_full = F.payload_decode(Path("gaugefixed_0").read_bytes(), size, F.PLAIN)
    out = S.gpupattern_to_timeslices(out_full, size)
    Vs = int(np.prod(size[1:]))
    for t in range(size[0]):
        gq, aq = O.quality(out[t * Vs * 72:(t + 1) * Vs * 72].copy(), (1,) + size[1:], O.COULOMB)
        assert gq == pytest.approx(g[:, t].max(), rel=1e-10)
        assert aq < 1e-11
    assert len(set(int(np.argmax(g[:, t])) for t in range(size[0]))) > 1  # slices come from several copies
    back = S.from_gpupattern(out_full, size)
    ref = S.from_gpupattern(full, size)
    assert np.abs(_plaquettes(back, size) - _plaquettes(ref, size)).max() < 1e-12
    assert r.output == "gaugefixed_0"


def _plaquettes(L, size):
    from su3_ma_gauge_gpu_b200 import synthetic as S

    vals = []
    for mu in range(4):
        for nu in range(mu + 1, 4):
            fm, fn = S.forward_neighbour_lex(size, mu), S.forward_neighbour_lex(size, nu)
            P = np.einsum("nij,njk,nlk,nml->nim", L[mu], L[nu][fm], L[mu][fn].conj(), L[nu].conj())
            vals.append(np.trace(P, axis1=1, axis2=2).real)
    return np.array(vals)
