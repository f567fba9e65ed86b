"""The C++ shim (include/gfix_culgt.hpp): a driver written like the reference's
Landau app compiles against it and links against libgfix.so (CPU test), and
its whole OR loop reproduces the oracle's driver (GPU test)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import _oracle as O
from su3_ma_gauge_gpu_b200 import synthetic as S

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "shim_driver.cpp"


def _build(tmp_path, X=4, T=8, double=True):
    exe = tmp_path / f"shim_driver_{X}_{T}_{int(double)}"
    cmd = ["g++", "-std=c++17", "-O2", f"-D_X_={X}", f"-D_T_={T}", "-I", str(ROOT / "include"),
           "-I", "/usr/local/cuda/include", str(SRC), "-o", str(exe),
           str(ROOT / "su3_ma_gauge_gpu_b200" / "libgfix.so"), f"-Wl,-rpath,{ROOT / 'su3_ma_gauge_gpu_b200'}",
           "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,/usr/local/cuda/lib64"]
    if double:
        cmd.insert(3, "-DDOUBLEPRECISION")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_shim_compiles_and_links(tmp_path):
    assert _build(tmp_path, double=True).exists()
    assert _build(tmp_path, double=False).exists()


@pytest.mark.gpu
def test_shim_driver_matches_oracle_driver(cuda, tmp_path):
    size = (8, 4, 4, 4)
    U, _ = S.smooth_config(size, 0.3, 77)
    exe = _build(tmp_path, X=4, T=8, double=True)
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    U.tofile(fin)
    r = subprocess.run([str(exe), str(fin), str(fout), "3000", "1e-11", "10", "50"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    sweeps, gff, theta = r.stdout.split()
    out = np.fromfile(fout, dtype=np.float64)
    ref = U.copy()
    sch = O.Schedule(0, 0, 0.01, 0.4, 0, 3000, 1.7, 1e-11, 10, 50, 1)
    res, _ = O.fix(ref, size, O.LANDAU, sch)
    assert int(sweeps) == res.or_iterations
    assert float(gff) == pytest.approx(res.gff, rel=1e-12)
    assert float(theta) < 1e-11
    assert np.abs(out - ref).max() < 1e-9
