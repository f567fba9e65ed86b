"""The C-ABI library loads and exports every entry point include/*.h declares;
argument validation works without touching the GPU (no compute calls here)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w \*]*?\b(gf\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = _declared_functions()
    for must in ("gf_or_step", "gf_sa_step", "gf_stats_generate", "gf_project_su3", "gf_last_error_string"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from su3_ma_gauge_gpu_b200 import _lib

    L = _lib.lib()
    missing = [n for n in _declared_functions() if not hasattr(L, n)]
    assert not missing, f"declared in include/ but not exported: {missing}"
    # the ctypes signature table covers the same set
    assert set(_lib.SIGNATURES) >= set(_declared_functions())


def test_library_is_built_for_sm100a():
    """The build passes exactly the sm_100a target to nvcc (the runtime answer is checked on the
    GPU by test_device_code_runs_as_sm100a)."""
    from su3_ma_gauge_gpu_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


@pytest.mark.gpu
def test_device_code_runs_as_sm100a(cuda):
    from su3_ma_gauge_gpu_b200 import _lib

    arch = ctypes.c_int()
    _lib.check(_lib.lib().gf_binary_arch(ctypes.byref(arch)), "gf_binary_arch")
    assert arch.value == 100


def test_validation_without_gpu():
    from su3_ma_gauge_gpu_b200 import _lib

    L = _lib.lib()
    assert L.gf_version().startswith(b"su3_ma_gauge_gpu_b200")
    bogus = ctypes.c_void_p(0x1000)  # never dereferenced: validation fails first
    s = _lib.size_arg((4, 4, 4, 3))
    assert L.gf_or_step(0, 1, bogus, None, s, 0, ctypes.c_float(1.7), None) == _lib.GF_ERR_INVALID
    assert b"even" in L.gf_last_error_string()
    s = _lib.size_arg((4, 4, 4, 4))
    assert L.gf_or_step(7, 1, bogus, None, s, 0, ctypes.c_float(1.7), None) == _lib.GF_ERR_INVALID
    assert L.gf_or_step(0, 5, bogus, None, s, 0, ctypes.c_float(1.7), None) == _lib.GF_ERR_INVALID
    assert L.gf_or_step(0, 1, None, None, s, 0, ctypes.c_float(1.7), None) == _lib.GF_ERR_INVALID
    assert L.gf_or_step(1, 1, bogus, bogus, s, 0, ctypes.c_float(1.7), None) == _lib.GF_ERR_INVALID  # slice
    assert L.gf_or_step(1, 1, bogus, None, _lib.size_arg((1, 4, 4, 4)), 0, ctypes.c_float(1.7), None) \
        == _lib.GF_ERR_INVALID  # Coulomb without UtDw
    assert L.gf_quality_prefactor_gff(0) == pytest.approx(1 / 12)
    assert L.gf_quality_prefactor_gff(1) == pytest.approx(1 / 9)
    assert L.gf_quality_prefactor_a(2) == pytest.approx(1 / 3)


def test_context_parameter_checks_without_gpu():
    """gf_create validates its parameters before touching the device."""
    from su3_ma_gauge_gpu_b200 import _lib

    L = _lib.lib()
    sizes = (ctypes.c_int32 * 4)(4, 4, 4, 4)
    h = ctypes.c_void_p()
    odd_t = (ctypes.c_int32 * 4)(3, 4, 4, 4)
    p = _lib.CtxParams(gauge=_lib.GF_COULOMB, ninstances=1, sizes=odd_t, mixed=2, stream=None)
    assert L.gf_create(ctypes.byref(p), ctypes.byref(h)) == _lib.GF_ERR_INVALID
    assert b"Nt = 3" in L.gf_last_error_string()
    p = _lib.CtxParams(gauge=_lib.GF_LANDAU, ninstances=1, sizes=sizes, mixed=3, stream=None)
    assert L.gf_create(ctypes.byref(p), ctypes.byref(h)) == _lib.GF_ERR_INVALID
    # a 6^3 timeslice has 108 sites per parity, not a whole number of 8-site tiles
    slice6 = (ctypes.c_int32 * 4)(2, 6, 6, 6)
    p = _lib.CtxParams(gauge=_lib.GF_COULOMB, ninstances=1, sizes=slice6, mixed=0, stream=None)
    assert L.gf_create(ctypes.byref(p), ctypes.byref(h)) == _lib.GF_ERR_INVALID
    assert b"multiple of 8 sites" in L.gf_last_error_string()
    p = _lib.CtxParams(gauge=_lib.GF_LANDAU, ninstances=0, sizes=sizes, mixed=0, stream=None)
    assert L.gf_create(ctypes.byref(p), ctypes.byref(h)) == _lib.GF_ERR_INVALID
