"""gf_quality_noalloc: the gauge quality without any allocation, checked
against gf_stats_generate through the C ABI.

Some callers cannot call cudaMalloc -- host frameworks that own all device
memory through their own pool, latency-critical loops where cudaMalloc's
device-wide synchronisation is not acceptable.  For them gf_quality_noalloc
keeps its reduction scratch in a fixed ~1 MiB device array (lattices up to
16,777,216 sites).  This file is collected last on purpose, and passes both on
its own in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

import _oracle as O
from su3_ma_gauge_gpu_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _stats(L, _lib, gauge, real, dU, size):
    h = ctypes.c_void_p()
    _lib.check(L.gf_stats_create(gauge, real, _lib.size_arg(size), _lib.GF_AVERAGE, ctypes.byref(h)), "create")
    g, a = ctypes.c_double(), ctypes.c_double()
    _lib.check(L.gf_stats_generate(h, dU.data_ptr(), None, ctypes.byref(g), ctypes.byref(a)), "generate")
    L.gf_stats_destroy(h)
    return g.value, a.value


def _noalloc(L, _lib, gauge, real, dU, size):
    g, a = ctypes.c_double(), ctypes.c_double()
    _lib.check(L.gf_quality_noalloc(gauge, real, dU.data_ptr(), _lib.size_arg(size), _lib.GF_AVERAGE, None,
                                    ctypes.byref(g), ctypes.byref(a)), "gf_quality_noalloc")
    return g.value, a.value


@pytest.mark.parametrize("gauge,real", [(O.LANDAU, 1), (O.LANDAU, 0), (O.MAG, 1), (O.COULOMB, 1)])
def test_noalloc_matches_allocating_entry_point_twice(cuda, gauge, real):
    from su3_ma_gauge_gpu_b200 import _lib

    torch = cuda
    L = _lib.lib()
    size = (1, 8, 8, 4) if gauge == O.COULOMB else (8, 8, 8, 16)  # 16 blocks of partial sums
    dtype = np.float64 if real == 1 else np.float32
    fields = [S.smooth_config(size, 0.3, seed, dtype=dtype)[0] for seed in (41, 42)]
    # two calls in a row (on different fields): the shared scratch keeps the last call's
    # contents, and the second answer must not depend on them
    for U in fields:
        dU = torch.from_numpy(U).cuda()
        want = _stats(L, _lib, gauge, real, dU, size)
        got = _noalloc(L, _lib, gauge, real, dU, size)
        assert got[0] == pytest.approx(want[0], rel=1e-12, abs=1e-14)
        assert got[1] == pytest.approx(want[1], rel=1e-12)


def test_noalloc_rejects_lattices_beyond_the_fixed_scratch(cuda):
    from su3_ma_gauge_gpu_b200 import _lib

    L = _lib.lib()
    g, a = ctypes.c_double(), ctypes.c_double()
    big = _lib.size_arg((66, 64, 64, 64))  # 17.3M sites > 16,777,216: rejected before any launch
    st = L.gf_quality_noalloc(0, 1, ctypes.c_void_p(0x1000), big, _lib.GF_AVERAGE, None, ctypes.byref(g),
                              ctypes.byref(a))
    assert st == _lib.GF_ERR_INVALID
    assert b"exceeds the fixed scratch limit" in L.gf_last_error_string()
