"""One lattice split into t-slabs (su3_ma_gauge_gpu_b200.tslab): the halo exchange around every
parity pass reproduces the single-lattice sweep bit for bit (overrelaxation is deterministic and
each site update reads only its 8 links).  CPU: the oracle plays the pass, ranks emulated in one
process and as world-size-2 gloo process groups; GPU: the library's plugin pass, ranks emulated
one after the other on one device."""
import os
import socket

import numpy as np
import pytest

import _oracle as O
from su3_ma_gauge_gpu_b200 import synthetic as S
from su3_ma_gauge_gpu_b200.tslab import (SlabExchange, TSlab, emulate_finish, emulate_overlapped_pass,
                                        emulate_parity_pass, emulate_refresh_halo, gpu_or_pass, gpu_or_slices,
                                        gpu_step_slices, parity_pass, quality)

SIZE = (8, 4, 6, 4)


def _oracle_pass(U, size, parity):
    O.step(U, size, O.LANDAU, O.OR, parity, 1.7, nthreads=2)


def _oracle_slices(U, size, parity, t_begin, t_end):
    O.step_slices(U, size, O.LANDAU, O.OR, parity, t_begin, t_end, 1.7, nthreads=2)


def _reference(U, nsweeps):
    R = U.copy()
    for _ in range(nsweeps):
        for p in (0, 1):
            _oracle_pass(R, SIZE, p)
    return R


@pytest.mark.parametrize("gauge,algo", [(O.MAG, O.OR), (O.U1XU1, O.OR), (O.LANDAU, O.MICRO), (O.MAG, O.MICRO)])
def test_emulated_slabs_other_gauges_and_updates(gauge, algo):
    """Every deterministic update of the 4D gauges reads only a site's 8 links: the slabs give
    the single-lattice result bit for bit for MAG and U1xU1, OR and microcanonical."""
    U, _ = S.smooth_config(SIZE, 0.3, 35)

    def run(A, size, parity):
        O.step(A, size, gauge, algo, parity, 1.7, nthreads=2)

    slabs = [TSlab(SIZE, r, 2) for r in range(2)]
    Us = [s.scatter(U) for s in slabs]
    R = U.copy()
    for _ in range(2):
        for p in (0, 1):
            emulate_parity_pass(slabs, Us, p, run)
            run(R, SIZE, p)
    out = np.zeros_like(U)
    for s, L in zip(slabs, Us):
        s.gather_into(L, out)
    assert np.array_equal(out, R)


def test_slab_geometry_checks():
    with pytest.raises(ValueError):
        TSlab((8, 4, 4, 4), 0, 3)  # 8 does not split in 3
    with pytest.raises(ValueError):
        TSlab((6, 4, 4, 4), 0, 2)  # slabs of 3 timeslices: odd
    s = TSlab(SIZE, 1, 2)
    assert s.local_size == (6, 4, 6, 4) and s.t0 == 4
    assert s.boundary_out(np.arange(72 * s.V, dtype=float), 0).size == s.Vs // 2 * 12


@pytest.mark.parametrize("world", [1, 2, 4])
def test_emulated_slabs_match_single_lattice(world):
    U, _ = S.smooth_config(SIZE, 0.3, 31)
    slabs = [TSlab(SIZE, r, world) for r in range(world)]
    Us = [s.scatter(U) for s in slabs]
    for _ in range(3):
        for p in (0, 1):
            emulate_parity_pass(slabs, Us, p, _oracle_pass)
    out = np.zeros_like(U)
    for s, L in zip(slabs, Us):
        s.gather_into(L, out)
    R = _reference(U, 3)
    assert np.array_equal(out, R)
    # the functional and theta summed over the owned sites of the slabs, halos refreshed first
    emulate_refresh_halo(slabs, Us)
    _, _, g, a = O.quality(R, SIZE, O.LANDAU, per_site=True)
    gs = sum(s.owned_sum(O.quality(L, s.local_size, O.LANDAU, per_site=True)[2]) for s, L in zip(slabs, Us))
    ts = sum(s.owned_sum(O.quality(L, s.local_size, O.LANDAU, per_site=True)[3]) for s, L in zip(slabs, Us))
    assert gs == pytest.approx(float(g.sum()), rel=1e-13)
    assert ts == pytest.approx(float(a.sum()), rel=1e-11)


@pytest.mark.parametrize("world", [1, 2, 4])
def test_emulated_overlapped_slabs_match_single_lattice(world):
    """The overlapped pass -- interior slices while the forward message travels, then the last
    owned slice, then the first from the halo, the return message waited for only by the next
    pass -- gives the single-lattice sweep bit for bit, without ever updating the halo sites."""
    U, _ = S.smooth_config(SIZE, 0.3, 36)
    slabs = [TSlab(SIZE, r, world) for r in range(world)]
    Us = [s.scatter(U) for s in slabs]
    halos = [L.reshape(72, -1)[:, :2 * s.Vs // 2].copy() for s, L in zip(slabs, Us)]  # parity-0 halo sites
    pending = {}
    for _ in range(3):
        for p in (0, 1):
            emulate_overlapped_pass(slabs, Us, p, _oracle_slices, pending)
    emulate_finish(slabs, Us, pending)
    out = np.zeros_like(U)
    for s, L in zip(slabs, Us):
        s.gather_into(L, out)
    assert np.array_equal(out, _reference(U, 3))
    for s, L, h0 in zip(slabs, Us, halos):  # halo slice 0's parity-0 sites: never updated
        assert np.array_equal(L.reshape(72, -1)[12:, :s.Vs // 2], h0[12:, :s.Vs // 2])


@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("gauge,algo,param", [(O.LANDAU, O.SA, 0.8), (O.MAG, O.SA, 0.8), (O.MAG, O.SR, 0.5),
                                              (O.LANDAU, O.RANDOM, 0.0)])
def test_emulated_slabs_random_updates_match_single_lattice(world, gauge, algo, param):
    """Each slab site draws its Philox numbers as its site of the whole lattice
    (TSlab.rng_site_offset), so the heat bath, stochastic relaxation and random transformations
    over slabs -- overlapped pass, interior first -- give the single-lattice sweep bit for bit."""
    U, _ = S.smooth_config(SIZE, 0.3, 37)
    slabs = [TSlab(SIZE, r, world) for r in range(world)]
    Us = [s.scatter(U) for s in slabs]
    R = U.copy()
    pending = {}
    for sweep in range(2):
        for p in (0, 1):
            ctr = 10 * sweep + p
            runs = [lambda A, size, parity, t0, t1, s=s, ctr=ctr:
                    O.step_slices(A, size, gauge, algo, parity, t0, t1, param, 7, ctr, nthreads=2,
                                  rng_site_offset=s.rng_site_offset) for s in slabs]
            emulate_overlapped_pass(slabs, Us, p, runs, pending)
            O.step(R, SIZE, gauge, algo, p, param, 7, ctr, nthreads=2)
    emulate_finish(slabs, Us, pending)
    out = np.zeros_like(U)
    for s, L in zip(slabs, Us):
        s.gather_into(L, out)
    assert np.array_equal(out, R)


def test_slab_rng_site_offset_maps_local_to_global_sites():
    """rng_site_offset is the shift between a slab's local and global parity-split indices."""
    for world in (1, 2, 4):
        for r in range(world):
            s = TSlab(SIZE, r, world)
            assert np.array_equal(s._owned_local % (s.V // 2) + s.rng_site_offset,
                                  s._owned_global % (int(np.prod(SIZE)) // 2))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, U, q, overlapped=False, heat_bath=False):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        slab = TSlab(SIZE, rank, world)
        L = slab.scatter(U)
        ex = SlabExchange(slab, L) if overlapped else None
        for sweep in range(2):
            for p in (0, 1):
                if heat_bath:  # SA at T = 0.8 with the whole lattice's Philox stream, counter 10 sweep + p
                    ex.parity_pass(L, p, lambda A, size, parity, t0, t1, c=10 * sweep + p: O.step_slices(
                        A, size, O.LANDAU, O.SA, parity, t0, t1, 0.8, 7, c, nthreads=2,
                        rng_site_offset=slab.rng_site_offset))
                elif overlapped:
                    ex.parity_pass(L, p, _oracle_slices)
                else:
                    parity_pass(slab, L, p, _oracle_pass)
        if overlapped:
            ex.finish(L)
        sums = quality(slab, L, lambda A, size: O.quality(A, size, O.LANDAU, per_site=True)[2:])
        out = np.zeros_like(U)
        slab.gather_into(L, out)
        q.put((rank, out, sums))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("overlapped", [False, True], ids=["whole-pass", "overlapped"])
def test_gloo_two_ranks_match_single_lattice(overlapped):
    import torch.multiprocessing as mp

    U, _ = S.smooth_config(SIZE, 0.3, 32)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, U, q, overlapped)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res = {r: (o, s) for r, o, s in got}
    out = np.zeros_like(U)
    for r in range(2):
        sl = TSlab(SIZE, r, 2)
        out.reshape(72, -1)[:, sl._owned_global] = res[r][0].reshape(72, -1)[:, sl._owned_global]
    R = _reference(U, 2)
    assert np.array_equal(out, R)
    _, _, g, a = O.quality(R, SIZE, O.LANDAU, per_site=True)
    for r in range(2):  # every rank holds the all-reduced sums
        assert res[r][1][0] == pytest.approx(float(g.sum()), rel=1e-13)
        assert res[r][1][1] == pytest.approx(float(a.sum()), rel=1e-11)


def test_gloo_two_ranks_heat_bath_matches_single_lattice():
    """Two gloo ranks with the overlapped exchange run the heat bath, each slab drawing the whole
    lattice's Philox stream (TSlab.rng_site_offset): the single lattice's SA sweeps bit for bit."""
    import torch.multiprocessing as mp

    U, _ = S.smooth_config(SIZE, 0.3, 33)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, U, q, True, True)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res = {r: o for r, o, _ in got}
    out = np.zeros_like(U)
    for r in range(2):
        sl = TSlab(SIZE, r, 2)
        out.reshape(72, -1)[:, sl._owned_global] = res[r].reshape(72, -1)[:, sl._owned_global]
    R = U.copy()
    for sweep in range(2):
        for p in (0, 1):
            O.step(R, SIZE, O.LANDAU, O.SA, p, 0.8, 7, 10 * sweep + p, nthreads=2)
    assert np.array_equal(out, R)


@pytest.mark.gpu
@pytest.mark.parametrize("world", [1, 2])
def test_gpu_slabs_match_plugin_pass(cuda, world):
    """The library's own pass on every slab, ranks one after the other on one GPU, against the
    same pass on the whole lattice."""
    torch = cuda
    from su3_ma_gauge_gpu_b200 import LandauKernelsSU3

    U, _ = S.smooth_config(SIZE, 0.3, 33)
    dU = torch.from_numpy(U).cuda()
    k = LandauKernelsSU3(SIZE, "double")
    for _ in range(3):
        for p in (0, 1):
            k.orStep(0, 0, dU, None, p, 1.7)
    slabs = [TSlab(SIZE, r, world) for r in range(world)]
    Us = [s.scatter(torch.from_numpy(U).cuda(), xp=torch) for s in slabs]
    run = gpu_or_pass(1.7)
    for _ in range(3):
        for p in (0, 1):
            emulate_parity_pass(slabs, Us, p, run)
    out = torch.zeros_like(dU)
    for s, L in zip(slabs, Us):
        s.gather_into(L, out)
    assert torch.equal(out, dU)


@pytest.mark.gpu
@pytest.mark.parametrize("world", [1, 2, 4])
def test_gpu_overlapped_slabs_match_plugin_pass(cuda, world):
    """The overlapped slab pass with the library's timeslice-range pass (gf_step_slices), ranks
    emulated on one GPU in the order the messages allow, against the whole-lattice plugin pass;
    and the range pass over slices [0, a) + [a, Nt) equals the whole pass."""
    torch = cuda
    from su3_ma_gauge_gpu_b200 import LandauKernelsSU3

    U, _ = S.smooth_config(SIZE, 0.3, 37)
    dU = torch.from_numpy(U).cuda()
    k = LandauKernelsSU3(SIZE, "double")
    for _ in range(3):
        for p in (0, 1):
            k.orStep(0, 0, dU, None, p, 1.7)
    run = gpu_or_slices(1.7)
    slabs = [TSlab(SIZE, r, world) for r in range(world)]
    Us = [s.scatter(torch.from_numpy(U).cuda(), xp=torch) for s in slabs]
    pending = {}
    for _ in range(3):
        for p in (0, 1):
            emulate_overlapped_pass(slabs, Us, p, run, pending)
    emulate_finish(slabs, Us, pending)
    out = torch.zeros_like(dU)
    for s, L in zip(slabs, Us):
        s.gather_into(L, out)
    assert torch.equal(out, dU)
    A = torch.from_numpy(U).cuda()
    B = torch.from_numpy(U).cuda()
    k.orStep(0, 0, A, None, 1, 1.7)
    run(B, SIZE, 1, 0, 3)
    run(B, SIZE, 1, 3, SIZE[0])
    assert torch.equal(A, B)


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("precision", ["double", "float"])
def test_gpu_slabs_heat_bath_matches_plugin_pass(cuda, world, precision):
    """The heat bath over slabs with the library's range pass (gf_step_slices_at with each slab's
    rng_site_offset), ranks emulated on one GPU, against the whole-lattice plugin saStep with the
    same seed and counters: bit for bit, in FP64 and FP32."""
    torch = cuda
    from su3_ma_gauge_gpu_b200 import LandauKernelsSU3

    dt = np.float64 if precision == "double" else np.float32
    U = S.smooth_config(SIZE, 0.3, 38)[0].astype(dt)
    dU = torch.from_numpy(U.copy()).cuda()
    k = LandauKernelsSU3(SIZE, precision)
    slabs = [TSlab(SIZE, r, world) for r in range(world)]
    Us = [s.scatter(torch.from_numpy(U.copy()).cuda(), xp=torch) for s in slabs]
    pending = {}
    for sweep in range(2):
        runs = [gpu_step_slices(s, "sa", 0.8, precision=precision, seed=5, counter=10 * sweep) for s in slabs]
        for p in (0, 1):
            k.saStep(0, 0, dU, None, p, 0.8, 5, 10 * sweep + p)
            emulate_overlapped_pass(slabs, Us, p, runs, pending)
    emulate_finish(slabs, Us, pending)
    out = torch.zeros_like(dU)
    for s, L in zip(slabs, Us):
        s.gather_into(L, out)
    assert torch.equal(out, dU)
