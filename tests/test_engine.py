"""GPU tests of the context-level engine (packed layout, batching, mixed
precision, device-side convergence) against the plugin-level path and the CPU
oracle's whole-run driver."""
import numpy as np
import pytest

import _oracle as O
from su3_ma_gauge_gpu_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _plugin_sweeps(torch, U, size, algo, n, param=0.0, seed=0, counter=0, gauge=O.LANDAU):
    """n sweeps through the plugin ABI on a reference-layout copy of U."""
    import ctypes

    from su3_ma_gauge_gpu_b200 import _lib

    L = _lib.lib()
    real = 1 if U.dtype == np.float64 else 0
    dU = torch.from_numpy(U.copy()).cuda()
    s = _lib.size_arg(size)
    for k in range(n):
        for parity in (0, 1):
            c = counter + 2 * k + parity
            if algo == "or":
                st = L.gf_or_step(gauge, real, dU.data_ptr(), None, s, parity, ctypes.c_float(param), None)
            elif algo == "micro":
                st = L.gf_micro_step(gauge, real, dU.data_ptr(), None, s, parity, None)
            elif algo == "sa":
                st = L.gf_sa_step(gauge, real, dU.data_ptr(), None, s, parity, ctypes.c_float(param), seed, c, None)
            else:
                st = L.gf_random_trafo(gauge, real, dU.data_ptr(), None, s, parity, seed, c, None)
            _lib.check(st, algo)
    return dU


def test_import_export_roundtrip(cuda):
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    torch = cuda
    size = (4, 4, 6, 8)
    U, _ = S.smooth_config(size, 0.3, 5)
    want = U.copy()
    O.project(want, size)
    for mixed in (False, True):
        with GaugeFixer([size], mixed=mixed) as gf:
            gf.load(0, U)  # host numpy path
            out = np.zeros_like(U)
            gf.store(0, out)
            tol = 1e-14 if not mixed else 2e-7
            assert np.abs(out - want).max() < tol
            dU = torch.from_numpy(U).cuda()
            gf.load(0, dU)  # device path
            dout = torch.zeros_like(dU)
            gf.store(0, dout)
            assert np.abs(dout.cpu().numpy() - want).max() < tol


@pytest.mark.parametrize("algo", ["or", "micro", "sa", "random"])
def test_packed_sweeps_bit_identical_to_plugin_path(cuda, algo):
    """Same kernel body, different HBM layout: FP64 results must agree bit for bit."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    torch = cuda
    size = (4, 6, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 8)
    param = {"or": 1.7, "sa": 0.5}.get(algo, 0.0)
    ref = _plugin_sweeps(torch, U, size, algo, 3, param, seed=3, counter=10).cpu().numpy()
    with GaugeFixer([size], mixed=False) as gf:
        gf.load(0, U)
        gf.sweeps(algo, 3, param, seed=3, rng_counter=10)
        g, a = gf.quality()
        out = np.zeros_like(U)
        gf.store(0, out)
    want = ref.copy()
    O.project(want, size)  # store() reunitarises like the reference's closing projectSU3
    assert np.abs(out - want).max() < 1e-14
    g_ref, a_ref = O.quality(ref, size, O.LANDAU)
    assert g[0] == pytest.approx(g_ref, rel=1e-13)
    assert a[0] == pytest.approx(a_ref, rel=1e-10)


def test_batched_uneven_instances(cuda):
    """Three lattices of different extents in one launch == each one on its own."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    torch = cuda
    sizes = [(4, 4, 4, 4), (2, 6, 4, 8), (6, 4, 2, 4)]
    fields = [S.smooth_config(s, 0.3, 20 + i)[0] for i, s in enumerate(sizes)]
    with GaugeFixer(sizes, mixed=False) as gf:
        for i, U in enumerate(fields):
            gf.load(i, U)
        gf.sweeps("sa", 2, 0.7, seed=9, rng_counter=4)
        gf.sweeps("or", 5, 1.7)
        outs = []
        for i, U in enumerate(fields):
            o = np.zeros_like(U)
            gf.store(i, o)
            outs.append(o)
    for i, (U, s) in enumerate(zip(fields, sizes)):
        # instance i draws with seed + i
        d = _plugin_sweeps(torch, U, s, "sa", 2, 0.7, seed=9 + i, counter=4)
        ref = _plugin_sweeps(torch, d.cpu().numpy(), s, "or", 5, 1.7).cpu().numpy()
        O.project(ref, s)
        assert np.abs(outs[i] - ref).max() < 1e-13, i


def _sched(**kw):
    from su3_ma_gauge_gpu_b200.engine import Schedule

    base = dict(or_max_iter=3000, precision=1e-11, check_precision=20, reproject=100, micro_updates=0)
    base.update(kw)
    return Schedule(**base)


def test_fix_fp64_matches_oracle_driver(cuda):
    """gf_fix (plain FP64) against the oracle's restatement of the Landau driver loop."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 31)
    sch = _sched(precision=1e-11, check_precision=10, reproject=50)
    with GaugeFixer([size], mixed=False) as gf:
        gf.load(0, U)
        rep = gf.fix(sch)[0]
        out = np.zeros_like(U)
        gf.store(0, out)
    ref = U.copy()
    osch = O.Schedule(0, 0, 0.01, 0.4, 0, sch.or_max_iter, 1.7, sch.precision, sch.check_precision, sch.reproject, 1)
    r, _ = O.fix(ref, size, O.LANDAU, osch)
    assert rep.converged and rep.theta < 1e-11
    assert rep.or_sweeps == r.or_iterations
    assert rep.gff == pytest.approx(r.gff, rel=1e-12)
    assert np.abs(out - ref).max() < 1e-9


@pytest.mark.parametrize("reproject,check", [(7, 10), (3, 10), (30, 20)])
def test_fix_reprojection_cadence_matches_oracle_driver(cuda, reproject, check):
    """The drivers reproject right after sweep i whenever i % reproject == 0
    (apps/LandauGaugeFixingSU3_4D.cu:249-252), also when reproject is smaller than, or not a multiple
    of, checkprecision: gf_fix (plain FP64) reproduces the oracle driver's field to 1e-12 per
    link after a fixed number of sweeps, and its sweep count and functional at convergence."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 33)
    for max_iter, prec in ((47, 1e-30), (3000, 1e-11)):
        sch = _sched(precision=prec, check_precision=check, reproject=reproject, or_max_iter=max_iter)
        with GaugeFixer([size], mixed=False) as gf:
            gf.load(0, U)
            rep = gf.fix(sch)[0]
            out = np.zeros_like(U)
            gf.store(0, out)
        ref = U.copy()
        osch = O.Schedule(0, 0, 0.01, 0.4, 0, sch.or_max_iter, 1.7, sch.precision, sch.check_precision,
                          sch.reproject, 1)
        r, _ = O.fix(ref, size, O.LANDAU, osch)
        assert rep.or_sweeps == r.or_iterations
        if max_iter < 100:  # budget spent: this run also checks after its last, partial chunk
            assert np.abs(out - ref).max() < 1e-12
        else:
            assert rep.converged
            assert rep.gff == pytest.approx(r.gff, rel=1e-12)
            assert np.abs(out - ref).max() < 1e-9


def test_landau_app_fix_with_sa_matches_oracle_driver(cuda):
    """The Landau app's whole loop in FP64 -- random gauge transformation, SA with linearly falling
    temperature and microcanonical steps after every SA sweep, OR to theta < 1e-12, reprojections --
    through gf_fix and through the oracle's restatement (apps/LandauGaugeFixingSU3_4D.cu:185-271) on
    the same input and Philox key/counters: the same sweep counts, functional and field."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 93)
    prec = float(np.float32(1e-12))
    kw = dict(random_trafo=1, sa_steps=12, sa_min=0.01, sa_max=0.8, micro_updates=2, or_max_iter=4000,
              precision=prec, check_precision=10, reproject=7, seed=21)
    with GaugeFixer([size], mixed=False) as gf:
        gf.load(0, U)
        rep = gf.fix(Schedule(rng_counter=6, **kw))[0]
        out = np.zeros_like(U)
        gf.store(0, out)
    ref = U.copy()
    r, ctr = O.fix_app(ref, size, O.LANDAU, O.app_schedule(**kw), counter=6)
    assert ctr == 6 + 2 + 2 * 12
    assert (rep.sa_sweeps, rep.or_sweeps) == (r.sa_sweeps, r.or_iterations)
    assert rep.converged and r.theta < 1e-12
    assert rep.gff == pytest.approx(r.gff, rel=1e-10)
    assert np.abs(out - ref).max() < 1e-9


def test_mag_app_fix_matches_oracle_driver(cuda):
    """The MAG app's whole schedule in FP64 -- random trafo, the SA do-while (5 heat-bath sweeps, each
    with a microcanonical sweep, per temperature, the step slowed 15x in its window), SR until
    theta < 1e-6, OR to theta < 1e-12, reprojections -- through gf_fix and through the oracle's
    restatement of apps/MAGaugeFixingSU3_4D.cu:222-333 on the same input and Philox key/counters:
    the same sweep count in every phase, the same functional, and the same field up to the
    diagonal U(1) x U(1) transformations that leave the MAG functional unchanged (compared through
    |U_ij|).  The anneal is short and cold: a hot heat bath amplifies the rounding differences of
    the two summation orders until the runs end at different maxima of equal functional."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 91)
    prec = float(np.float32(1e-12))
    sch = Schedule.mag_app(random_trafo=1, sa_steps=3, sa_min=0.1, sa_max=0.5, sa_slow_lo=0.2, sa_slow_hi=0.3,
                           micro_updates=1, or_max_iter=4000, precision=prec, check_precision=10, reproject=20,
                           seed=3, rng_counter=5)
    with GaugeFixer([size], gauge="mag", mixed=False) as gf:
        gf.load(0, U)
        rep = gf.fix(sch)[0]
        out = np.zeros_like(U)
        gf.store(0, out)
    ref = U.copy()
    osch = O.app_schedule(random_trafo=1, sa_steps=3, sa_min=0.1, sa_max=0.5, micro_updates=1, sa_mode=2,
                          sa_repeat=5, sa_slow_lo=0.2, sa_slow_hi=0.3, sa_slow_factor=15.0, sr_max_iter=1000,
                          sr_parameter=1.7, sr_stop_theta=1e-6, or_max_iter=4000, precision=prec, check_precision=10,
                          reproject=20, seed=3)
    r, _ = O.fix_app(ref, size, O.MAG, osch, counter=5)
    assert (rep.sa_sweeps, rep.sr_sweeps, rep.or_sweeps) == (r.sa_sweeps, r.sr_iterations, r.or_iterations)
    assert rep.converged and r.theta < 1e-12
    assert rep.gff == pytest.approx(r.gff, rel=1e-10)
    assert np.abs(np.abs(O.links(out, size)) - np.abs(O.links(ref, size))).max() < 1e-8


def test_coulomb_app_fix_matches_oracle_slice_loop(cuda):
    """The Coulomb app's loop (apps/CoulombGaugeFixingSU3_4D.cu:199-311): timeslices one after the
    other, each with random trafo, SA + a microcanonical sweep after every SA sweep, OR to
    theta < 1e-12, the Philox counter running on from slice to slice.  gf_fix batches all slices and,
    with rng_streams = 1, gives each slice the key word and counters the app's loop gives it: per
    slice the same sweep counts and functional, and the same exported field -- temporal links
    included, which the app multiplies from both sides one slice at a time."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    size = (4, 4, 6, 4)
    U = np.concatenate([S.smooth_config((1,) + size[1:], 0.3, 140 + t)[0] for t in range(size[0])])
    prec = float(np.float32(1e-12))
    kw = dict(random_trafo=1, sa_steps=5, sa_min=0.01, sa_max=1.0, micro_updates=1, or_max_iter=4000, precision=prec,
              check_precision=10, reproject=20, seed=11)
    with GaugeFixer([size], gauge="coulomb", mixed=False) as gf:
        gf.load(0, U)
        reps = gf.fix(Schedule(rng_counter=4, rng_streams=1, **kw))
        out = np.zeros_like(U)
        gf.store(0, out)
    ref = U.copy()
    res, ctr = O.fix_coulomb(ref, size, O.app_schedule(**kw), counter=4)
    assert ctr == 4 + size[0] * 12
    for t in range(size[0]):
        assert (reps[t].sa_sweeps, reps[t].or_sweeps) == (res[t].sa_sweeps, res[t].or_iterations), t
        assert reps[t].converged and res[t].theta < 1e-12
        assert reps[t].gff == pytest.approx(res[t].gff, rel=1e-10), t
    assert np.abs(out - ref).max() < 1e-9


@pytest.mark.parametrize("gauge,mixed", [("landau", False), ("landau", True), ("mag", False), ("coulomb", False)],
                         ids=["landau-fp64", "landau-mixed", "mag-fp64", "coulomb-fp64"])
def test_persistent_chunks_bit_identical_to_per_pass_launches(cuda, gauge, mixed):
    """schedule.persistent = 1 runs each check chunk's sweeps and reprojections as one cooperative
    launch with grid barriers; the fix is bit for bit the one the per-pass launches give (same
    site update, same order), on a batch of uneven lattices, with reprojections inside chunks."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    if gauge == "coulomb":
        sizes = [(4, 4, 6, 4), (2, 8, 4, 4)]
        fields = [np.concatenate([S.smooth_config((1,) + s[1:], 0.3, 150 + 10 * i + t)[0] for t in range(s[0])])
                  for i, s in enumerate(sizes)]
    else:
        sizes = [(2, 2, 2, 6), (4, 4, 4, 4), (8, 8, 8, 8)]
        fields = [S.smooth_config(s, 0.3, 160 + i)[0] for i, s in enumerate(sizes)]
    outs, reps = {}, {}
    for persistent in (0, 1):
        with GaugeFixer(sizes, gauge=gauge, mixed=mixed) as gf:
            gf.set_pass_shape("fp64", 0, 4)
            if mixed:
                gf.set_pass_shape("fp32", 0, 4)
            for i, U in enumerate(fields):
                gf.load(i, U)
            reps[persistent] = gf.fix(_sched(precision=1e-12, switch_theta=1e-9, check_precision=10, reproject=7,
                                             or_max_iter=3000, autotune=0, persistent=persistent))
            outs[persistent] = []
            for i, U in enumerate(fields):
                o = np.zeros_like(U)
                gf.store(i, o)
                outs[persistent].append(o)
    for a, b in zip(reps[0], reps[1]):
        assert (a.gff, a.theta, a.or_sweeps, a.or_sweeps_fp64) == (b.gff, b.theta, b.or_sweeps, b.or_sweeps_fp64)
        assert b.converged
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)


def test_persistent_chunk_wait_runs_out_and_reports_timeout(cuda):
    """Every grid-barrier wait of the persistent chunk kernel is bounded.  With a barrier that waits
    for one arrival that never comes, every block gives up after the budget (2 ms), the kernel
    returns, and gf_fix reports GF_ERR_TIMEOUT; the context stays usable and the next fix on a
    reloaded field converges to the per-pass result."""
    from su3_ma_gauge_gpu_b200 import _lib
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    size = (8, 8, 8, 8)
    U, _ = S.smooth_config(size, 0.3, 170)
    with GaugeFixer([size], mixed=False) as gf:
        gf.load(0, U)
        with pytest.raises(_lib.GaugeFixError) as err:
            gf.fix(_sched(precision=1e-12, check_precision=10, persistent=1, wait_budget_us=2000, wait_test_missing=1))
        assert err.value.status == _lib.GF_ERR_TIMEOUT
        assert "ran out" in str(err.value)
        gf.load(0, U)
        rep = gf.fix(_sched(precision=1e-12, check_precision=10, persistent=1))[0]
    with GaugeFixer([size], mixed=False) as gf:
        gf.load(0, U)
        ref = gf.fix(_sched(precision=1e-12, check_precision=10))[0]
    assert rep.converged and rep.gff == pytest.approx(ref.gff, rel=1e-13) and rep.or_sweeps == ref.or_sweeps


def test_check_chunk_graphs_are_kept_across_fixes(cuda):
    """The captured check-chunk graphs belong to the context: a second gf_fix with the same schedule
    replays them (same launches counted, same result), and changing the launch shape drops them."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 171)
    with GaugeFixer([size], mixed=False) as gf:
        gf.set_pass_shape("fp64", 0, 4)
        res = []
        for _ in range(2):
            gf.load(0, U)
            l0 = gf.kernel_launches()
            res.append((gf.fix(_sched(precision=1e-12, check_precision=10, autotune=0))[0], gf.kernel_launches() - l0))
        gf.set_pass_shape("fp64", 1, 4)
        gf.load(0, U)
        third = gf.fix(_sched(precision=1e-12, check_precision=10, autotune=0))[0]
    (a, na), (b, nb) = res
    assert (a.gff, a.or_sweeps) == (b.gff, b.or_sweeps) and na == nb
    assert third.gff == a.gff and third.or_sweeps == a.or_sweeps


def _mixed_vs_fp64(size, eps, seed):
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    U, f0 = S.smooth_config(size, eps, seed)
    res = {}
    for mixed in (False, True):
        with GaugeFixer([size], mixed=mixed) as gf:
            gf.load(0, U)
            res[mixed] = gf.fix(_sched(precision=1e-12, switch_theta=1e-9, check_precision=10))[0]
    return res, f0


def test_fix_mixed_reaches_fp64_fixed_point(cuda):
    """Mixed precision: FP32 bulk to 1e-9, FP64 polish to 1e-12.  Rounding the links to FP32 is not
    a gauge transformation, so the FP32 phase moves the field slightly off its gauge orbit: F
    agrees with plain FP64 to the FP32 drift (1e-6 relative), not to 1e-10."""
    res, f0 = _mixed_vs_fp64((8, 8, 8, 8), 0.1, 2)
    assert res[False].converged and res[True].converged
    assert res[True].theta < 1e-12
    assert 0 < res[True].or_sweeps_fp64 < res[True].or_sweeps
    assert res[True].gff == pytest.approx(res[False].gff, rel=1e-6)
    assert res[True].gff >= f0 - 1e-12  # fixing the transformed field recovers at least F(untransformed)


def test_fix_mixed_rough_field_reports_copy(cuda):
    """eps = 0.3 fields have many nearby maxima (Gribov copies): FP32 rounding early in the run
    may select another one.  Both runs converge; F agrees to the copy spread (<1e-5 relative)."""
    res, _ = _mixed_vs_fp64((8, 8, 8, 8), 0.3, 2)
    assert res[False].converged and res[True].converged
    assert res[True].gff == pytest.approx(res[False].gff, rel=1e-5)


@pytest.mark.parametrize("prec", ["fp32", "fp64", "refine"])
def test_pipelined_pass_bit_identical_to_direct(cuda, prec):
    """Every launch shape of the OR pass -- cp.async-pipelined (2, 4, 8 warps per block), register
    prefetch (persistent), 64-register FP32, thread per site, two lanes per site (direct and
    persistent) -- computes exactly what the direct pass computes, on a batch of uneven lattices
    (the first has 3 eight-site tiles, so two-lane warps straddle instances); in refine mode
    including the accumulated W (the export applies it)."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    sizes = [(2, 2, 2, 6), (4, 4, 4, 4), (2, 6, 4, 8), (8, 8, 8, 8)]
    fields = [S.smooth_config(s, 0.3, 50 + i)[0] for i, s in enumerate(sizes)]
    mixed = {"fp32": True, "fp64": False, "refine": "refine"}[prec]
    outs = {}
    if prec == "refine":
        shapes = [(0, 4), (2, 4), (3, 4), (4, 4), (5, 4), (6, 4), (7, 4), (7, 4, 1), (3, 4, 1), (7, 4, 1, 1)]
    else:
        shapes = [(0, 4), (1, 2), (1, 4), (1, 8), (3, 4), (6, 4), (1, 4, 1), (1, 8, 1), (3, 4, 1), (1, 4, 1, 1),
                  (1, 4, 1, 0, 3), (1, 4, 0, 0, 3)] + (
            [(2, 4), (4, 4), (5, 4), (7, 4), (7, 4, 1), (7, 4, 1, 1)] if prec == "fp32" else [])
    for shape in shapes:
        variant, warps = shape[:2]
        with GaugeFixer(sizes, mixed=mixed) as gf:
            real = "fp64" if prec == "fp64" else "fp32"
            gf.set_pass_shape(real, variant, warps)
            if len(shape) > 2:
                gf.set_pass_order(real, bool(shape[2]), len(shape) > 3 and bool(shape[3]))
            if len(shape) > 4:
                gf.set_pass_stages(real, shape[4])
            for i, U in enumerate(fields):
                gf.load(i, U)
            gf.sweeps("or", 4, 1.7)
            res = []
            for i, U in enumerate(fields):
                o = np.zeros_like(U)
                gf.store(i, o)
                res.append(o)
            outs[shape] = res
    base = outs[(0, 4)]
    for key, res in outs.items():
        for i in range(len(sizes)):
            assert np.array_equal(res[i], base[i]), (key, i)


@pytest.mark.parametrize("mixed", [False, True, "refine"], ids=["fp64", "fp32", "refine"])
def test_coulomb_register_prefetch_pass_bit_identical_to_direct(cuda, mixed):
    """Coulomb slices on the persistent register-prefetch pass (variant 3, with and without the
    alternating walk) and on the two-lane passes (6; 7 with the walk, register-capped): the
    temporal direction carries the slice's W as its up link and has no down link, as in the direct
    pass, and the two-lane sum (0 + v1) + (v2 + v3) is the 4-lane butterfly's, so OR sweeps are bit
    for bit the direct pass's; the export applies W to the temporal links, so W is compared too."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    sizes = [(4, 4, 6, 4), (2, 8, 4, 4)]
    fields = [np.concatenate([S.smooth_config((1,) + s[1:], 0.3, 190 + 10 * i + t)[0] for t in range(s[0])])
              for i, s in enumerate(sizes)]
    real = "fp64" if mixed is False else "fp32"
    outs = {}
    for variant, alternate, capped in ((0, False, False), (3, False, False), (3, True, False), (6, False, False),
                                       (7, False, False), (7, True, False), (7, True, True)):
        with GaugeFixer(sizes, gauge="coulomb", mixed=mixed) as gf:
            gf.set_pass_shape(real, variant, 4)
            gf.set_pass_order(real, alternate, capped)
            for i, U in enumerate(fields):
                gf.load(i, U)
            gf.sweeps("or", 4, 1.7)
            res = []
            for i, U in enumerate(fields):
                o = np.zeros_like(U)
                gf.store(i, o)
                res.append(o)
            outs[(variant, alternate, capped)] = res
    base = outs[(0, False, False)]
    for key, res in outs.items():
        for i in range(len(sizes)):
            assert np.array_equal(res[i], base[i]), (key, i)


def test_pass_stages_need_the_four_warp_pipelined_pass(cuda):
    """Three cp.async stages exist for the pipelined pass with 4 warps per block only; any other
    shape, or a stage count other than 2 or 3, is refused."""
    from su3_ma_gauge_gpu_b200 import _lib
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    with GaugeFixer([(4, 4, 4, 4)], mixed=False) as gf:
        gf.set_pass_shape("fp64", 0, 4)
        with pytest.raises(_lib.GaugeFixError):
            gf.set_pass_stages("fp64", 3)
        gf.set_pass_shape("fp64", 1, 8)
        with pytest.raises(_lib.GaugeFixError):
            gf.set_pass_stages("fp64", 3)
        gf.set_pass_shape("fp64", 1, 4)
        gf.set_pass_stages("fp64", 3)
        gf.set_pass_stages("fp64", 2)
        with pytest.raises(_lib.GaugeFixError):
            gf.set_pass_stages("fp64", 4)


@pytest.mark.parametrize("gauge", ["landau", "mag", "u1xu1"])
@pytest.mark.parametrize("algo", ["sa", "micro", "sr"])
def test_thread_per_site_pass_matches_direct(cuda, gauge, algo):
    """The FP32 thread-per-site pass sums the four directions in the 4-lane butterfly's order and
    draws the same Philox numbers as the direct pass; for OR the two are bit-identical
    (test_pipelined_pass_bit_identical_to_direct).  For the other rules the compiler may contract
    a product differently in the two kernels, so one sweep agrees to FP32 rounding."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    sizes = [(4, 4, 4, 4), (2, 6, 4, 8)]
    fields = [S.smooth_config(s, 0.3, 70 + i)[0] for i, s in enumerate(sizes)]
    outs = []
    for variant in (0, 4):
        with GaugeFixer(sizes, gauge=gauge, mixed=True) as gf:
            gf.set_pass_shape("fp32", variant, 4)
            for i, U in enumerate(fields):
                gf.load(i, U)
            gf.sweeps(algo, 1, 0.7, 5, 11)
            res = []
            for i, U in enumerate(fields):
                o = np.zeros_like(U)
                gf.store(i, o)
                res.append(o)
            outs.append(res)
    # U1xU1 microcanonical steps divide by the norm of a two-component quaternion, which is small
    # at some sites of a Haar-transformed field: there one rounding difference grows to ~2e-5
    tol = 1e-4 if (gauge, algo) == ("u1xu1", "micro") else 1e-5
    for a, b in zip(*outs):
        assert np.abs(a - b).max() < tol


@pytest.mark.parametrize("prec", ["fp32", "fp64", "refine"])
@pytest.mark.parametrize("gauge", ["landau", "mag", "u1xu1"])
@pytest.mark.parametrize("algo", ["sa", "micro", "sr", "random"])
def test_two_lane_pass_matches_direct(cuda, gauge, algo, prec):
    """The two-lanes-per-site pass sums the four directions in the 4-lane butterfly's order and both
    lanes of a site draw the Philox numbers the direct pass draws, for every update rule: one sweep
    agrees with the direct pass to FP32 rounding (FP64: 1e-13)."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    sizes = [(2, 2, 2, 6), (4, 4, 4, 4), (2, 6, 4, 8)]
    fields = [S.smooth_config(s, 0.3, 75 + i)[0] for i, s in enumerate(sizes)]
    mixed = {"fp32": True, "fp64": False, "refine": "refine"}[prec]
    real = "fp64" if prec == "fp64" else "fp32"
    outs = []
    for variant in (0, 6):
        with GaugeFixer(sizes, gauge=gauge, mixed=mixed) as gf:
            gf.set_pass_shape(real, variant, 4)
            for i, U in enumerate(fields):
                gf.load(i, U)
            gf.sweeps(algo, 1, 0.7, 5, 11)
            res = []
            for i, U in enumerate(fields):
                o = np.zeros_like(U)
                gf.store(i, o)
                res.append(o)
            outs.append(res)
    # U1xU1 micro and SR steps normalise a two-component quaternion that is small at some sites of a
    # Haar-transformed field: there one FP32 rounding difference grows to a few 1e-5
    tol = 1e-13 if prec == "fp64" else (1e-4 if (gauge, algo) in (("u1xu1", "micro"), ("u1xu1", "sr")) else 1e-5)
    for a, b in zip(*outs):
        assert np.abs(a - b).max() < tol


def test_autotune_picks_a_shape(cuda):
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    size = (8, 8, 8, 16)
    U, _ = S.smooth_config(size, 0.3, 3)
    with GaugeFixer([size], mixed=True) as gf:
        gf.load(0, U)
        before = np.zeros_like(U)
        gf.store(0, before)
        c32, c64 = gf.autotune()
        # codes + 1000: the same shape with the alternating walk (gf_set_pass_order)
        assert c32 % 1000 in (0, 64, 100, 32, 33, 16, 116, 2, 4, 8) and c64 % 1000 in (0, 100, 16, 2, 4, 8)
        assert c32 < 200000 and c64 < 200000
        after = np.zeros_like(U)
        gf.store(0, after)
        assert np.array_equal(before, after)  # tuning ran on a scratch copy


def _coulomb_reference_flow(torch, U, size, nsweeps, algo="or", param=1.7, seed=0, counter=0):
    """The reference's Coulomb app flow through the plugin ABI: timeslices one after the other,
    each with UtUp = slice t and UtDw = slice t-1 (apps/CoulombGaugeFixingSU3_4D.cu:199-311)."""
    import ctypes

    from su3_ma_gauge_gpu_b200 import _lib

    L = _lib.lib()
    Nt = size[0]
    Vs = int(np.prod(size[1:]))
    slices = [torch.from_numpy(U[t * Vs * 72:(t + 1) * Vs * 72].copy()).cuda() for t in range(Nt)]
    ss = _lib.size_arg((1,) + tuple(size[1:]))
    for t in range(Nt):
        up, dw = slices[t], slices[(t - 1) % Nt]
        for k in range(nsweeps):
            for parity in (0, 1):
                if algo == "or":
                    st = L.gf_or_step(1, 1, up.data_ptr(), dw.data_ptr(), ss, parity, ctypes.c_float(param), None)
                else:
                    st = L.gf_sa_step(1, 1, up.data_ptr(), dw.data_ptr(), ss, parity, ctypes.c_float(param),
                                      seed + t, counter + 2 * k + parity, None)
                _lib.check(st, "coulomb step")
    for t in range(Nt):
        _lib.check(L.gf_project_su3(1, slices[t].data_ptr(), ss, None), "project")
    return np.concatenate([s.cpu().numpy() for s in slices])


@pytest.mark.parametrize("algo", ["or", "sa"])
def test_coulomb_batched_matches_sequential_timeslices(cuda, algo):
    """All timeslices in one launch (W tracking) == the reference's slice-by-slice loop."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    torch = cuda
    size = (4, 4, 6, 4)
    Vs = int(np.prod(size[1:]))
    # the reference's timeslice layout: Nt consecutive GpuPattern arrays of {1, Nx, Ny, Nz}
    U = np.concatenate([S.smooth_config((1,) + size[1:], 0.3, 60 + t)[0] for t in range(size[0])])
    n = 3
    param = 1.7 if algo == "or" else 0.6
    ref = _coulomb_reference_flow(torch, U, size, n, algo, param, seed=7, counter=5)
    with GaugeFixer([size], gauge="coulomb", mixed=False) as gf:
        assert gf.ninstances == size[0]
        gf.load(0, U)
        gf.sweeps(algo, n, param, seed=7, rng_counter=5)
        out = np.zeros_like(U)
        gf.store(0, out)
    a = out.reshape(size[0], 4, 3, 3, 2, Vs)
    b = ref.reshape(size[0], 4, 3, 3, 2, Vs)
    assert np.abs(a[:, 1:] - b[:, 1:]).max() < 1e-13          # spatial links
    assert np.abs(a[:, 0] - b[:, 0]).max() < 1e-12            # temporal links via W
    assert np.abs(a[:, 0] - U.reshape(size[0], 4, 3, 3, 2, Vs)[:, 0]).max() > 1e-3


def test_coulomb_fix_every_slice(cuda):
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    size = (4, 8, 8, 8)
    U = np.concatenate([S.smooth_config((1,) + size[1:], 0.3, 80 + t)[0] for t in range(size[0])])
    with GaugeFixer([size], gauge="coulomb", mixed=True) as gf:
        gf.load(0, U)
        reps = gf.fix(_sched(precision=1e-12, switch_theta=1e-9, check_precision=10, or_max_iter=5000))
        g, a = gf.quality()
    assert len(reps) == size[0]
    assert all(r.converged and r.theta < 1e-12 for r in reps)
    assert np.all(a < 1e-12)
    # each slice against the oracle's Coulomb quality of the exported field
    out = np.zeros_like(U)
    with GaugeFixer([size], gauge="coulomb", mixed=True) as gf:
        gf.load(0, U)
        gf.fix(_sched(precision=1e-12, switch_theta=1e-9, check_precision=10, or_max_iter=5000))
        gf.store(0, out)
    Vs = int(np.prod(size[1:]))
    for t in range(size[0]):
        gq, aq = O.quality(out[t * Vs * 72:(t + 1) * Vs * 72].copy(), (1,) + size[1:], O.COULOMB)
        assert aq < 1e-11
        assert gq == pytest.approx(reps[t].gff, rel=1e-9)


@pytest.mark.parametrize("fold", [0, 1], ids=["fp64-polish", "iterative-refinement"])
def test_coulomb_refine_lands_on_the_fp64_maximum(cuda, fold):
    """Refine mode for Coulomb timeslices: each slice's FP32 working copy tracks its gauge
    transformation in its temporal planes, and the folds / the switch apply it exactly to the FP64
    master.  Every slice reaches theta < 1e-12 with a functional equal to the plain-FP64 batched fix
    (which test_coulomb_batched_matches_sequential_timeslices pins to the reference's slice-by-slice
    flow) to 1e-10 relative, and the exported field (temporal links W(t) U_0 W(t+1)^dagger) has the
    oracle's Coulomb quality of that functional."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    size = (4, 8, 8, 8)
    Vs = int(np.prod(size[1:]))
    U = np.concatenate([S.smooth_config((1,) + size[1:], 0.3, 180 + t)[0] for t in range(size[0])])
    sch = _sched(precision=1e-12, switch_theta=1e-9, check_precision=10, or_max_iter=6000, fold=fold)
    reps, outs = {}, {}
    for mode in (False, "refine"):
        with GaugeFixer([size], gauge="coulomb", mixed=mode) as gf:
            gf.load(0, U)
            reps[mode] = gf.fix(sch)
            outs[mode] = np.zeros_like(U)
            gf.store(0, outs[mode])
    for t in range(size[0]):
        r, f = reps["refine"][t], reps[False][t]
        assert r.converged and r.theta < 1e-12
        assert r.or_sweeps_fp64 < r.or_sweeps
        assert r.gff == pytest.approx(f.gff, rel=1e-10), t
        gq, aq = O.quality(outs["refine"][t * Vs * 72:(t + 1) * Vs * 72].copy(), (1,) + size[1:], O.COULOMB)
        assert gq == pytest.approx(f.gff, rel=1e-10)
        assert aq < 1e-11
    # the temporal links of both exports agree: the same per-slice transformations were applied
    a = outs["refine"].reshape(size[0], 4, 3, 3, 2, Vs)[:, 0]
    b = outs[False].reshape(size[0], 4, 3, 3, 2, Vs)[:, 0]
    assert np.abs(a - b).max() < 1e-5


def test_coulomb_refine_export_is_gauge_equivalent(cuda):
    """A refine Coulomb context exported mid-run (working copy current, W32 not yet folded) is a gauge
    transform of its input: every plaquette, spatial and temporal, is unchanged to FP64 rounding."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    size = (4, 4, 6, 4)
    Vs = int(np.prod(size[1:]))
    U = np.concatenate([S.smooth_config((1,) + size[1:], 0.3, 190 + t)[0] for t in range(size[0])])
    with GaugeFixer([size], gauge="coulomb", mixed="refine") as gf:
        gf.load(0, U)
        gf.sweeps("or", 25, 1.7)
        out = np.zeros_like(U)
        gf.store(0, out)
    full_in = S.from_gpupattern(_timeslices_to_gpupattern(U, size), size)
    full_out = S.from_gpupattern(_timeslices_to_gpupattern(out, size), size)
    assert np.abs(_plaquettes(full_out, size) - _plaquettes(full_in, size)).max() < 1e-12
    assert np.abs(out - U).max() > 1e-3


def _timeslices_to_gpupattern(T, size):
    """Inverse of synthetic.gpupattern_to_timeslices (for the plaquette check)."""
    nt, nx, ny, nz = size
    vs, v = nx * ny * nz, nt * nx * ny * nz
    t, x, y, z = (a.reshape(-1) for a in np.meshgrid(np.arange(nt), np.arange(nx), np.arange(ny), np.arange(nz),
                                                     indexing="ij"))
    l = ((t * nx + x) * ny + y) * nz + z
    s_full = l // 2 + ((t + x + y + z) % 2) * (v // 2)
    s_slice = ((x * ny + y) * nz + z) // 2 + ((x + y + z) % 2) * (vs // 2)
    src = np.asarray(T).reshape(nt, 72, vs)
    out = np.empty((72, v), dtype=src.dtype)
    out[:, s_full] = src[t, :, s_slice].T
    return out.reshape(-1)


def _plaquettes(L, size):
    vals = []
    for mu in range(4):
        for nu in range(mu + 1, 4):
            fm, fn = S.forward_neighbour_lex(size, mu), S.forward_neighbour_lex(size, nu)
            P = np.einsum("nij,njk,nlk,nml->nim", L[mu], L[nu][fm], L[mu][fn].conj(), L[nu].conj())
            vals.append(np.trace(P, axis1=1, axis2=2).real)
    return np.array(vals)


def _mag_app_temperatures(sa_steps, sa_min, sa_max, lo, hi, factor):
    """Temperatures of the MAG app's do-while (apps/MAGaugeFixingSU3_4D.cu:233-266), in float32."""
    f = np.float32
    T, base = f(sa_max), f((f(sa_max) - f(sa_min)) / f(sa_steps))
    out = []
    while True:
        step = base / f(factor) if (float(T) <= hi and float(T) >= lo) else base
        out.append(float(T))
        T = f(T - step)
        if not T >= f(sa_min):
            return out


def test_mag_app_schedule(cuda):
    """SA do-while with 5 sweeps per temperature and the slowed window, SR, then OR in mixed
    precision, for MAG.  MAG's theta stalls near 2e-7 in FP32 (the oracle shows the same floor),
    far above switch_theta: the stall rule moves the instance to the FP64 polish."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 90)
    sch = Schedule.mag_app(sa_steps=20, sa_min=0.01, sa_max=1.4, micro_updates=1, or_max_iter=4000,
                           precision=1e-12, switch_theta=1e-9, check_precision=10, reproject=20, seed=3)
    temps = _mag_app_temperatures(20, 0.01, 1.4, 0.7, 0.88, 15.0)
    with GaugeFixer([size], gauge="mag", mixed=True) as gf:
        gf.load(0, U)
        g0, _ = gf.quality()
        rep = gf.fix(sch)[0]
    assert rep.sa_sweeps == 5 * len(temps)
    assert rep.sr_sweeps >= 1
    assert rep.converged and rep.theta < 1e-12
    assert 0 < rep.or_sweeps_fp64 < rep.or_sweeps
    assert rep.gff > g0[0]  # the MAG functional increased


def test_u1xu1_fix_after_mag_keeps_the_mag_functional(cuda):
    """The residual U(1)xU(1) gauge fixing after MAG applies only diagonal transformations, which
    leave the MAG functional sum |U_jj|^2 unchanged while they raise the U1xU1 functional: fix MAG,
    then 200 U1xU1 OR sweeps, and compare.  (The U1xU1 theta is the full-matrix Landau measure,
    U1xU1KernelsSU3.hxx:114-191, which diagonal transformations cannot drive to zero.)"""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 91)
    sch = Schedule(or_max_iter=3000, precision=1e-12, switch_theta=1e-9, check_precision=20, reproject=20,
                   micro_updates=0)
    out = np.zeros_like(U)
    with GaugeFixer([size], gauge="mag", mixed=False) as gf:
        gf.load(0, U)
        rep = gf.fix(sch)[0]
        gf.store(0, out)
    assert rep.converged
    with GaugeFixer([size], gauge="u1xu1", mixed=False) as gu:
        gu.load(0, out)
        f0, _ = gu.quality()
        ru = gu.fix(Schedule(or_max_iter=200, precision=1e-12, check_precision=20, reproject=20, micro_updates=0))[0]
        gu.store(0, out)
    assert ru.or_sweeps == 200 and ru.gff > f0[0]
    with GaugeFixer([size], gauge="mag", mixed=False) as gq:
        gq.load(0, out)
        g, _ = gq.quality()
    assert g[0] == pytest.approx(rep.gff, rel=1e-12)


def test_stall_rule_off_keeps_mag_in_fp32(cuda):
    """With stall_checks = 0 the switch waits for theta < switch_theta, which FP32 MAG never
    reaches: the run stays in FP32 and ends at the sweep cap (the old behaviour)."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 90)
    sch = Schedule(or_max_iter=600, precision=1e-12, switch_theta=1e-9, check_precision=20, reproject=20,
                   micro_updates=0, stall_checks=0)
    with GaugeFixer([size], gauge="mag", mixed=True) as gf:
        gf.load(0, U)
        rep = gf.fix(sch)[0]
    assert rep.or_sweeps_fp64 == 0 and not rep.converged
    assert 1e-8 < rep.theta < 1e-5


@pytest.mark.parametrize("fold", [0, 1], ids=["fp64-polish", "iterative-refinement"])
def test_refine_mode_lands_on_the_fp64_maximum(cuda, fold):
    """Refine mode (FP64 master + FP32 working copy + accumulated W): the FP32 sweeps only
    choose a gauge transformation, applied exactly to the FP64 master, so the mixed run reaches
    the plain-FP64 maximum to 1e-10 relative in F -- with FP64 polish sweeps (fold = 0) and with
    iterative refinement (fold = 1: FP32 sweeps folded into the master after every check, theta
    measured on the master)."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    size = (8, 8, 8, 8)
    res = {}
    for eps in (0.1, 0.3):
        U, _ = S.smooth_config(size, eps, 2)
        for mode in (False, "refine"):
            with GaugeFixer([size], mixed=mode) as gf:
                gf.load(0, U)
                res[(eps, mode)] = gf.fix(_sched(precision=1e-12, switch_theta=1e-9, check_precision=10,
                                                 fold=fold))[0]
        r, f = res[(eps, "refine")], res[(eps, False)]
        assert r.converged and r.theta < 1e-12
        if fold:
            assert r.or_sweeps_fp64 < r.or_sweeps // 2  # most sweeps in FP32
        else:
            assert 0 < r.or_sweeps_fp64 < r.or_sweeps
        assert r.gff == pytest.approx(f.gff, rel=1e-10), eps


def test_refine_export_is_gauge_equivalent(cuda):
    """Gauge-invariant check of the refine switch: the plaquette field of the exported
    configuration equals the input's (the FP64 master only ever receives W U W^dagger)."""
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    size = (4, 4, 6, 4)
    U, _ = S.smooth_config(size, 0.3, 12)
    with GaugeFixer([size], mixed="refine") as gf:
        gf.load(0, U)
        gf.sweeps("or", 30, 1.7)
        gf.to_fp64()
        out = np.zeros_like(U)
        gf.store(0, out)

    def plaquettes(F):
        L = S.from_gpupattern(F, size)
        vals = []
        for mu in range(4):
            for nu in range(mu + 1, 4):
                fm, fn = S.forward_neighbour_lex(size, mu), S.forward_neighbour_lex(size, nu)
                P = np.einsum("nij,njk,nlk,nml->nim", L[mu], L[nu][fm], L[mu][fn].conj(), L[nu].conj())
                vals.append(np.trace(P, axis1=1, axis2=2).real)
        return np.array(vals)

    assert np.abs(plaquettes(out) - plaquettes(U)).max() < 1e-12
