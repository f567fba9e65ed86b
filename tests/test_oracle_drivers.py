"""The oracle's whole-run drivers (oracle/gf_oracle_impl.h orc_fix_app, orc_fix_coulomb): the apps'
per-copy loops for every gauge and the Coulomb app's slice loop, checked on the host against the
oracle's Landau driver and against the apps' temperature and counter bookkeeping."""
import numpy as np

import _oracle as O
from su3_ma_gauge_gpu_b200 import synthetic as S


def mag_app_temperatures(sa_steps, sa_min, sa_max, lo, hi, factor):
    """Temperatures of the MAG app's SA do-while (apps/MAGaugeFixingSU3_4D.cu:233-266), in float32."""
    f = np.float32
    T, base = f(sa_max), f((f(sa_max) - f(sa_min)) / f(sa_steps))
    out = []
    while True:
        step = f(base / f(factor)) if (float(T) <= hi and float(T) >= lo) else base
        out.append(float(T))
        T = f(T - step)
        if not T >= f(sa_min):
            return out


def test_app_driver_reproduces_the_landau_driver():
    """sa_mode 0 without SR is the Landau app's loop: orc_fix_app and orc_fix give the same bits."""
    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 7)
    kw = dict(random_trafo=1, sa_steps=6, sa_min=0.05, sa_max=0.6, micro_updates=2, or_max_iter=400,
              or_parameter=1.7, precision=1e-10, check_precision=10, reproject=7, seed=5)
    A, B = U.copy(), U.copy()
    ra, ca = O.fix_app(A, size, O.LANDAU, O.app_schedule(**kw), counter=3)
    rb, cb = O.fix(B, size, O.LANDAU, O.Schedule(kw["random_trafo"], kw["sa_steps"], kw["sa_min"], kw["sa_max"],
                                                kw["micro_updates"], kw["or_max_iter"], kw["or_parameter"],
                                                kw["precision"], kw["check_precision"], kw["reproject"],
                                                kw["seed"]), counter=3)
    assert np.array_equal(A, B)
    assert (ra.gff, ra.theta, ra.or_iterations) == (rb.gff, rb.theta, rb.or_iterations)
    assert ca == cb == 3 + 2 + 2 * 6
    assert ra.sa_sweeps == 6 and ra.sr_iterations == 0


def test_mag_app_driver_bookkeeping():
    """The MAG app's loop: 5 SA sweeps per do-while temperature, two Philox counters per SA and SR
    sweep, SR stops at theta < 1e-6, and the MAG functional rises."""
    size = (4, 4, 4, 8)
    U, _ = S.smooth_config(size, 0.3, 9)
    g0, _ = O.quality(U, size, O.MAG)
    sch = O.app_schedule(random_trafo=1, sa_steps=8, sa_min=0.01, sa_max=1.4, micro_updates=1, sa_mode=2,
                         sa_repeat=5, sa_slow_lo=0.7, sa_slow_hi=0.88, sa_slow_factor=15.0, sr_max_iter=1000,
                         sr_parameter=1.7, sr_stop_theta=1e-6, or_max_iter=3000, precision=1e-12, check_precision=10,
                         reproject=20, seed=3)
    r, c = O.fix_app(U, size, O.MAG, sch, counter=0)
    temps = mag_app_temperatures(8, 0.01, 1.4, 0.7, 0.88, 15.0)
    assert r.sa_sweeps == 5 * len(temps)
    assert c == 2 + 2 * r.sa_sweeps + 2 * r.sr_iterations
    assert 1 <= r.sr_iterations <= 1000
    assert r.theta < 1e-12 and r.gff > g0


def test_coulomb_slice_loop_runs_the_counter_on():
    """The Coulomb app fixes timeslice t with UtDw = slice t-1 and one process-wide Philox counter:
    slice t draws its random trafo and SA sweeps from the counters slice t-1 left off at, so fixing
    slice 0 alone with the same start counter gives slice 0's result bit for bit, and every slice
    ends below the target precision.  (Slice 0's temporal links are changed again by slice 1's fix,
    which right-multiplies them as its UtDw, and slice 1's reprojections of its UtDw touch slice 0's
    spatial links at rounding level.)"""
    size = (4, 4, 6, 4)
    Vs = int(np.prod(size[1:]))
    U = np.concatenate([S.smooth_config((1,) + size[1:], 0.3, 40 + t)[0] for t in range(size[0])])
    sch = O.app_schedule(random_trafo=1, sa_steps=5, sa_min=0.01, sa_max=1.0, micro_updates=1, or_max_iter=3000,
                         precision=1e-12, check_precision=10, reproject=20, seed=11)
    A = U.copy()
    res, c = O.fix_coulomb(A, size, sch, counter=4)
    assert c == 4 + size[0] * (2 + 2 * 5)
    assert all(r.theta < 1e-12 and r.sa_sweeps == 5 for r in res)
    up = U[:Vs * 72].copy()
    dw = U[(size[0] - 1) * Vs * 72:].copy()
    r0, c0 = O.fix_app(up, (1,) + size[1:], O.COULOMB, sch, counter=4, Udw=dw)
    assert c0 == 4 + 12 and r0.gff == res[0].gff
    assert np.abs(up[18 * Vs:] - A[18 * Vs:Vs * 72]).max() < 1e-14
