"""Pins the CPU oracle to the reference before anything is compared against it.

The reference has no tests or golden vectors of its own, so the pin is the
reference's own code: oracle/Makefile compiles its site-update code
(GaugeFixingSubgroupStep.hxx, algorithms/*Update.hxx, SU3/Quaternion/Matrix/
Complex/Link/SiteIndex/SiteCoord, PhiloxWrapper + Random123) for the host into
oracle/_ref/.  In FP64 (the reference's serialised accumulation order) the C
oracle must agree with it BIT FOR BIT; in FP32 the reference sums with
shared-memory atomics in a nondeterministic order, so agreement is to float
rounding.  The committed golden hashes (tests/golden/) pin the oracle where the
reference tree is absent.
"""
import ctypes

import numpy as np
import pytest

import _oracle as O

HAVE_REF = O.ref_pin("f64") is not None and O.ref_pin("f32") is not None
needs_ref = pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (reference tree absent)")

SIZE4 = (4, 4, 4, 4)
SLICE = (1, 8, 8, 4)


@needs_ref
def test_philox_known_answers_vs_random123():
    orc, ref = O.oracle(), O.ref_pin("f64")
    rng = np.random.default_rng(12345)
    # edge inputs (all zeros, all ones, pi digits) plus random ones
    cases = [([0, 0, 0, 0], [0, 0]), ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2),
             ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0])]
    cases += [(list(rng.integers(0, 2**32, 4)), list(rng.integers(0, 2**32, 2))) for _ in range(500)]
    for c, k in cases:
        c = np.array(c, dtype=np.uint32)
        k = np.array(k, dtype=np.uint32)
        a = np.zeros(4, np.uint32)
        b = np.zeros(4, np.uint32)
        orc.orc_philox4x32_10(c.ctypes.data_as(ctypes.c_void_p), k.ctypes.data_as(ctypes.c_void_p),
                              a.ctypes.data_as(ctypes.c_void_p))
        ref.ref_philox4x32_10_f64(c.ctypes.data_as(ctypes.c_void_p), k.ctypes.data_as(ctypes.c_void_p),
                                  b.ctypes.data_as(ctypes.c_void_p))
        assert np.array_equal(a, b), (c, k, a, b)


@needs_ref
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_rand_sequence_matches_philox_wrapper(prec):
    orc, ref = O.oracle(), O.ref_pin(prec)
    for tid, seed, ctr in [(0, 0, 0), (77, 5, 9), (2**31 - 1, 1234, 2**32 - 1)]:
        a = np.zeros(64)
        b = np.zeros(64)
        getattr(orc, "orc_rand_sequence_" + prec)(ctypes.c_uint32(tid), ctypes.c_uint32(seed), ctypes.c_uint32(ctr),
                                                  64, a.ctypes.data_as(ctypes.c_void_p))
        getattr(ref, "ref_rand_sequence_" + prec)(ctypes.c_uint32(tid), ctypes.c_uint32(seed), ctypes.c_uint32(ctr),
                                                  64, b.ctypes.data_as(ctypes.c_void_p))
        assert np.array_equal(a, b)
        assert (a > 0).all() and (a < 1).all()


@needs_ref
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_set_hot_matches_reference(dtype):
    a = O.ref_set_hot(SIZE4, 3, 1, dtype)
    b = O.set_hot(SIZE4, 3, 1, dtype)
    assert np.array_equal(a, b)


def _fields(gauge, dtype):
    size = SLICE if gauge == O.COULOMB else SIZE4
    U = O.set_hot(size, 3, 1, dtype)
    Udw = O.set_hot(size, 4, 1, dtype) if gauge == O.COULOMB else None
    return size, U, Udw


@needs_ref
@pytest.mark.parametrize("gauge", list(O.GAUGES.values()), ids=list(O.GAUGES))
@pytest.mark.parametrize("algo", list(O.ALGOS.values()), ids=list(O.ALGOS))
def test_step_fp64_bit_exact_vs_reference_code(gauge, algo):
    size, U, Udw = _fields(gauge, np.float64)
    R, Rdw = U.copy(), None if Udw is None else Udw.copy()
    param = 1.7 if algo == O.OR else (0.5 if algo == O.SR else 0.8)
    for parity in (0, 1):
        O.ref_step(R, size, gauge, algo, parity, param, 11, 7 + parity, Udw=Rdw)
        O.step(U, size, gauge, algo, parity, param, 11, 7 + parity, Udw=Udw)
    assert np.abs(R - O.set_hot(size, 3, 1)).max() > 1e-3  # the step did something
    assert np.array_equal(U, R)
    if Udw is not None:
        assert np.array_equal(Udw, Rdw)


@needs_ref
@pytest.mark.parametrize("gauge", list(O.GAUGES.values()), ids=list(O.GAUGES))
@pytest.mark.parametrize("algo", [O.OR, O.MICRO, O.SR, O.RANDOM], ids=["or", "micro", "sr", "random"])
def test_step_fp32_vs_reference_code(gauge, algo):
    """FP32: the reference accumulates with atomics in arbitrary order -> rounding-level agreement."""
    size, U, Udw = _fields(gauge, np.float32)
    R, Rdw = U.copy(), None if Udw is None else Udw.copy()
    param = 1.7 if algo == O.OR else 0.5
    for parity in (0, 1):
        O.ref_step(R, size, gauge, algo, parity, param, 11, 7 + parity, Udw=Rdw)
        O.step(U, size, gauge, algo, parity, param, 11, 7 + parity, Udw=Udw)
    tol = 1e-4 if gauge == O.MAG else 1e-5
    assert O.rows01_maxdiff(U, R, size) < tol


@needs_ref
@pytest.mark.parametrize("gauge", list(O.GAUGES.values()), ids=list(O.GAUGES))
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_quality_bit_exact_vs_reference_code(gauge, dtype):
    size, U, _ = _fields(gauge, dtype)
    g_ref, a_ref = O.ref_quality_sites(U, size, gauge)
    _, _, g, a = O.quality(U, size, gauge, per_site=True)
    assert np.array_equal(g, g_ref)
    assert np.array_equal(a, a_ref)


@needs_ref
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_project_bit_exact_vs_reference_code(dtype):
    U = O.set_hot(SIZE4, 5, 2, dtype)
    U += (np.random.default_rng(0).standard_normal(U.shape) * 1e-3).astype(dtype)  # off the group
    R = U.copy()
    O.ref_project(R, SIZE4)
    O.project(U, SIZE4)
    assert np.array_equal(U, R)


def test_layout_helpers():
    orc = O.oracle()
    size = np.array([4, 6, 2, 8], np.int32)
    V = int(np.prod(size))
    seen = set()
    for t in range(size[0]):
        for x in range(size[1]):
            for y in range(size[2]):
                for z in range(size[3]):
                    c = np.array([t, x, y, z], np.int32)
                    s = orc.orc_site_index(size.ctypes.data_as(ctypes.c_void_p), c.ctypes.data_as(ctypes.c_void_p))
                    assert (s >= V // 2) == bool((t + x + y + z) & 1)
                    back = np.zeros(4, np.int32)
                    orc.orc_site_coords(size.ctypes.data_as(ctypes.c_void_p), ctypes.c_int64(s),
                                        back.ctypes.data_as(ctypes.c_void_p))
                    assert list(back) == [t, x, y, z]
                    seen.add(s)
    assert seen == set(range(V))
