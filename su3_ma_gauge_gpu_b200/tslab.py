"""One lattice over several GPUs: t-slabs with a halo exchange per parity pass.

The reference's multi-GPU driver splits ONE lattice into slabs of timeslices, one per MPI rank,
and around every parity pass of the boundary sites sends the temporal links of the boundary
slice forward and returns them updated (apps/MultiGPU_MPI/MultiGPU_MPI_Communicator.hxx:351-430).
This module does the same with torch.distributed point-to-point messages (NCCL over NVLink on
GPUs, gloo on CPU) around the library's own parity pass, unchanged:

* rank r owns the timeslices [r*T, (r+1)*T) (T = Nt / world, even) and keeps them as slices
  2 .. T+1 of a local lattice of extent T + 2, whose slices 0 and 1 are a halo.  Site parity is
  the same locally and globally because every slab starts at an even t.
* A site of the first owned slice reads its down temporal link U_t(x - t) from halo slice 1; no
  other owned site reads the halo.  In the pass of parity p those links belong to the
  parity-(1-p) sites of slice 1 -- the last owned slice of rank r-1, where the pass of parity p
  does not touch them.  So before the pass rank r-1 sends them (rows 0 and 1: Vs/2 x 12 reals,
  the reference's message) and after it rank r returns them, updated, into rank r-1's last slice.
* The pass also updates the halo sites of parity p; they read wrapped or stale neighbours and
  write only halo links and the wrapped parity-(1-p) temporal links of the last owned slice --
  exactly the links the returned message overwrites.  Nothing owned is left corrupted.

In the GpuPattern layout the message is a plain block of the field: the temporal links of slice t
and parity q are the contiguous run h in [t Vs/2, (t+1) Vs/2) of the parity-q half of each of the
12 planes of rows 0 and 1 -- a (12, Vs/2) slice with row stride V.  So messages are packed and
unpacked by one strided copy each, never by index lists.

SlabExchange runs a pass with the exchange overlapped, as the reference splits its pass
(MultiGPU_MPI_Communicator.hxx:351-430): the forward message is posted first, the interior slices
(which read no halo) are updated while it travels, then the last owned slice (once the previous
pass's returned links are in), then the first owned slice from the halo, and the return message
is posted without waiting -- the next pass waits for it only before it updates the last slice.
The halo sites themselves are never updated.  With NCCL the waits are stream dependencies, so the
host never blocks inside a sweep.

The functional and theta are summed with all_reduce.  Every update rule gives the single-lattice
result bit for bit: overrelaxation and microcanonical steps are deterministic, and the random ones
(heat bath, stochastic relaxation, random transformations) draw each site's Philox numbers by its
index in the whole lattice -- in the parity-split order a slab's sites are the global ones shifted
by one constant, `TSlab.rng_site_offset`, which gf_step_slices_at takes.
"""
from __future__ import annotations

import numpy as np


def _site_index(size, t, x, y, z):
    """Parity-split index of sites (arrays of coordinates) in a lattice of extents `size`."""
    nt, nx, ny, nz = size
    v = nt * nx * ny * nz
    l = ((t * nx + x) * ny + y) * nz + z
    return l // 2 + ((t + x + y + z) % 2) * (v // 2)


class TSlab:
    """The slab of rank `rank` out of `world` for a lattice of extents `size` = (Nt, Nx, Ny, Nz).

    Arrays are GpuPattern arrays (18 reals per link) of the local lattice `self.local_size`:
    CUDA tensors with the library's plugin pass, or any array type the injected pass accepts."""

    def __init__(self, size, rank: int, world: int):
        nt, nx, ny, nz = (int(v) for v in size)
        if world < 1 or not 0 <= rank < world or nt % world or (nt // world) % 2:
            raise ValueError("Nt must split into `world` slabs of an even number of timeslices")
        self.size = (nt, nx, ny, nz)
        self.rank, self.world = rank, world
        self.T = nt // world
        self.t0 = rank * self.T
        self.local_size = (self.T + 2, nx, ny, nz)
        self.V = (self.T + 2) * nx * ny * nz
        self.Vs = nx * ny * nz
        x, y, z = (a.reshape(-1) for a in np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"))
        self._xyz = (x, y, z)
        V = self.V
        ls = self.local_size
        # owned sites (slices 2 .. T+1) in local parity-split order, and their global indices
        tl = np.repeat(np.arange(2, self.T + 2), self.Vs)
        xx, yy, zz = (np.tile(a, self.T) for a in (x, y, z))
        self._owned_local = _site_index(ls, tl, xx, yy, zz)
        self._owned_global = _site_index(self.size, tl - 2 + self.t0, xx, yy, zz)
        self._owned_mask = np.zeros(V, dtype=bool)
        self._owned_mask[self._owned_local] = True
        # local site h (either parity) is global site h + rng_site_offset: local slice t is global
        # slice t0 - 2 + t, and in the parity-split order a slice holds Vs / 2 sites of each parity
        self.rng_site_offset = (self.t0 - 2) * self.Vs // 2

    # ---- moving whole fields between the global array and the slabs (set-up, checks) ----------
    def scatter(self, Uglob, xp=np):
        """Local array of this rank from the global GpuPattern array: owned slices, halo slices
        filled from the two slices before t0 (so the halo holds unitary links)."""
        nt = self.size[0]
        Vg = int(np.prod(self.size))
        x, y, z = self._xyz
        Ug = Uglob.reshape(72, Vg)
        out = xp.zeros((72, self.V), dtype=Uglob.dtype) if xp is np else None
        loc_list, glob_list = [], []
        for tl in range(self.T + 2):
            tg = (self.t0 + tl - 2) % nt
            loc_list.append(_site_index(self.local_size, np.full(self.Vs, tl), x, y, z))
            glob_list.append(_site_index(self.size, np.full(self.Vs, tg), x, y, z))
        loc = np.concatenate(loc_list)
        glob = np.concatenate(glob_list)
        if xp is np:
            out[:, loc] = Ug[:, glob]
            return out.reshape(-1)
        import torch

        out = torch.zeros((72, self.V), dtype=Uglob.dtype, device=Uglob.device)
        out[:, torch.as_tensor(loc, device=Uglob.device)] = Ug[:, torch.as_tensor(glob, device=Uglob.device)]
        return out.reshape(-1)

    def gather_into(self, Ulocal, Uglob):
        """Write this rank's owned slices into the global GpuPattern array (in place)."""
        Vg = int(np.prod(self.size))
        Ug = Uglob.reshape(72, Vg)
        Ul = Ulocal.reshape(72, self.V)
        if isinstance(Uglob, np.ndarray):
            Ug[:, self._owned_global] = Ul[:, self._owned_local]
        else:
            import torch

            dev = Uglob.device
            Ug[:, torch.as_tensor(self._owned_global, device=dev)] = Ul[:, torch.as_tensor(self._owned_local,
                                                                                         device=dev)]

    # ---- the exchange ---------------------------------------------------------------------------
    def rows_view(self, U, t, q):
        """Rows 0, 1 (the 12 stored reals) of the temporal links of local slice t, sites of parity q:
        a (12, Vs/2) view of the GpuPattern array U (numpy array or tensor; no copy)."""
        half = self.Vs // 2
        s0 = t * half + q * (self.V // 2)
        return U.reshape(72, self.V)[:12, s0:s0 + half]

    def boundary_out(self, U, p):
        """Before the pass of parity p: what goes to rank r+1 (its halo), a contiguous copy."""
        v = self.rows_view(U, self.T + 1, 1 - p)
        return v.copy() if isinstance(v, np.ndarray) else v.clone()

    def halo_in(self, U, p, msg):
        self.rows_view(U, 1, 1 - p)[...] = msg

    def halo_out(self, U, p):
        """After the pass of parity p: the updated halo links that go back to rank r-1."""
        v = self.rows_view(U, 1, 1 - p)
        return v.copy() if isinstance(v, np.ndarray) else v.clone()

    def boundary_in(self, U, p, msg):
        self.rows_view(U, self.T + 1, 1 - p)[...] = msg

    def owned_sum(self, per_site):
        """Sum of a per-site array (local parity-split order) over the owned sites."""
        if isinstance(per_site, np.ndarray):
            return float(per_site[self._owned_mask].sum())
        import torch

        mask = self.__dict__.get("_tmask")
        if mask is None or mask.device != per_site.device:
            mask = torch.as_tensor(self._owned_mask, device=per_site.device)
            self._tmask = mask
        return float(per_site[mask].sum().item())


def parity_pass(slab: TSlab, U, parity: int, run_pass, group=None):
    """One parity pass of the whole lattice, this rank's share: halo in, run_pass(U, local_size,
    parity) on the local lattice, updated halo back.  Ring point-to-point messages through
    torch.distributed; with one rank the ring is a local copy."""
    p = parity
    if slab.world == 1:
        slab.halo_in(U, p, slab.boundary_out(U, p))
        run_pass(U, slab.local_size, p)
        slab.boundary_in(U, p, slab.halo_out(U, p))
        return
    import torch
    import torch.distributed as dist

    nxt, prv = (slab.rank + 1) % slab.world, (slab.rank - 1) % slab.world
    host = isinstance(U, np.ndarray)  # host arrays (CPU runs): messages travel as CPU tensors

    def ring(msg, to, frm):
        send = torch.from_numpy(np.ascontiguousarray(msg)) if host else msg.contiguous()
        recv = torch.empty_like(send)
        reqs = dist.batch_isend_irecv([dist.P2POp(dist.isend, send, to, group),
                                       dist.P2POp(dist.irecv, recv, frm, group)])
        for r in reqs:
            r.wait()
        return recv.numpy() if host else recv

    slab.halo_in(U, p, ring(slab.boundary_out(U, p), nxt, prv))
    run_pass(U, slab.local_size, p)
    slab.boundary_in(U, p, ring(slab.halo_out(U, p), prv, nxt))


def refresh_halo(slab: TSlab, U, group=None):
    """Bring the halo's temporal links of BOTH parities up to date (the sweep keeps only those the
    next pass reads current) -- needed before the functional and theta, whose first owned slice
    reads every down temporal link."""
    if slab.world == 1:
        for p in (0, 1):
            slab.halo_in(U, p, slab.boundary_out(U, p))
        return
    import torch
    import torch.distributed as dist

    host = isinstance(U, np.ndarray)
    nxt, prv = (slab.rank + 1) % slab.world, (slab.rank - 1) % slab.world
    for p in (0, 1):
        msg = slab.boundary_out(U, p)
        send = torch.from_numpy(np.ascontiguousarray(msg)) if host else msg.contiguous()
        recv = torch.empty_like(send)
        reqs = dist.batch_isend_irecv([dist.P2POp(dist.isend, send, nxt, group),
                                       dist.P2POp(dist.irecv, recv, prv, group)])
        for r in reqs:
            r.wait()
        slab.halo_in(U, p, recv.numpy() if host else recv)


def quality(slab: TSlab, U, per_site, group=None):
    """(sum of the functional terms, sum of the theta terms) over the whole lattice: per_site(U,
    local_size) returns the per-site arrays of the local lattice; owned sites are summed and the
    sums all-reduced.  Normalise like the single-lattice quality."""
    refresh_halo(slab, U, group)
    g, a = per_site(U, slab.local_size)
    sums = [slab.owned_sum(g), slab.owned_sum(a)]
    if slab.world > 1:
        import torch
        import torch.distributed as dist

        t = torch.tensor(sums, dtype=torch.float64)
        if not isinstance(U, np.ndarray):
            t = t.to(U.device)
        dist.all_reduce(t, group=group)
        sums = [float(v) for v in t.cpu()]
    return sums[0], sums[1]


def emulate_refresh_halo(slabs, Us):
    world = len(slabs)
    for p in (0, 1):
        outs = [slabs[r].boundary_out(Us[r], p) for r in range(world)]
        for r in range(world):
            slabs[r].halo_in(Us[r], p, outs[(r - 1) % world])


def emulate_parity_pass(slabs, Us, parity: int, run_pass):
    """The same pass for all ranks of one process (one GPU, or CPU), ranks one after the other:
    every message is a copy.  No rank waits on another inside a kernel."""
    world = len(slabs)
    outs = [slabs[r].boundary_out(Us[r], parity) for r in range(world)]  # fancy indexing copies
    for r in range(world):
        slabs[r].halo_in(Us[r], parity, outs[(r - 1) % world])
    for r in range(world):
        run_pass(Us[r], slabs[r].local_size, parity)
    backs = [slabs[r].halo_out(Us[r], parity) for r in range(world)]
    for r in range(world):
        slabs[r].boundary_in(Us[r], parity, backs[(r + 1) % world])


class SlabExchange:
    """Parity passes of one slab with the boundary exchange overlapped (see the module docstring).

    run_slices(U, local_size, parity, t_begin, t_end) updates the sites of local slices
    [t_begin, t_end) (gpu_or_slices for the library's pass).  Buffers are allocated once; call
    finish() after the last pass (before reading the last owned slice or the functional)."""

    def __init__(self, slab: TSlab, U, group=None):
        self.slab, self.group = slab, group
        self.host = isinstance(U, np.ndarray)
        shape = (12, slab.Vs // 2)
        if self.host:
            self.buf = {k: np.empty(shape, dtype=U.dtype) for k in ("fs", "fr", "bs", "br")}
        else:
            import torch

            self.buf = {k: torch.empty(shape, dtype=U.dtype, device=U.device) for k in ("fs", "fr", "bs", "br")}
        self.pending = None  # (works of the return exchange, parity of its links)

    def _post(self, send, to, recv, frm):
        """send -> rank `to`, recv <- rank `frm`; returns the works (a local copy for one rank)."""
        if self.slab.world == 1:
            recv[...] = send
            return []
        import torch
        import torch.distributed as dist

        s = torch.from_numpy(send) if self.host else send
        r = torch.from_numpy(recv) if self.host else recv
        return dist.batch_isend_irecv([dist.P2POp(dist.isend, s, to, self.group),
                                       dist.P2POp(dist.irecv, r, frm, self.group)])

    @staticmethod
    def _wait(works):
        for w in works:
            w.wait()  # NCCL: the current stream waits; gloo: the host waits

    def _finish_return(self, U):
        if self.pending is not None:
            works, q = self.pending
            self._wait(works)
            self.slab.rows_view(U, self.slab.T + 1, q)[...] = self.buf["br"]
            self.pending = None

    def parity_pass(self, U, p, run_slices):
        sl = self.slab
        T, ls = sl.T, sl.local_size
        nxt, prv = (sl.rank + 1) % sl.world, (sl.rank - 1) % sl.world
        b = self.buf
        b["fs"][...] = sl.rows_view(U, T + 1, 1 - p)
        fwd = self._post(b["fs"], nxt, b["fr"], prv)
        run_slices(U, ls, p, 3, T + 1)        # interior: reads no halo and no returned link
        self._finish_return(U)                # the previous pass's links, updated by rank r+1
        run_slices(U, ls, p, T + 1, T + 2)    # last owned slice
        self._wait(fwd)
        sl.rows_view(U, 1, 1 - p)[...] = b["fr"]
        run_slices(U, ls, p, 2, 3)            # first owned slice, from the halo
        b["bs"][...] = sl.rows_view(U, 1, 1 - p)
        self.pending = (self._post(b["bs"], prv, b["br"], nxt), 1 - p)

    def finish(self, U):
        self._finish_return(U)


def emulate_overlapped_pass(slabs, Us, parity: int, run_slices, pending):
    """SlabExchange.parity_pass for all ranks of one process (one GPU or CPU), the ranks' steps
    interleaved in the order the messages allow: every message is a copy and no rank waits on
    another inside a kernel.  `run_slices` is one callable for every rank or a list with one per
    rank (e.g. gpu_step_slices of each slab).  `pending` carries the return messages between
    passes (start with {}; call emulate_finish at the end)."""
    world = len(slabs)
    p = parity
    run = run_slices if isinstance(run_slices, (list, tuple)) else [run_slices] * world
    outs = [slabs[r].boundary_out(Us[r], p) for r in range(world)]
    for r in range(world):
        run[r](Us[r], slabs[r].local_size, p, 3, slabs[r].T + 1)
    emulate_finish(slabs, Us, pending)
    for r in range(world):
        run[r](Us[r], slabs[r].local_size, p, slabs[r].T + 1, slabs[r].T + 2)
    for r in range(world):
        slabs[r].halo_in(Us[r], p, outs[(r - 1) % world])
        run[r](Us[r], slabs[r].local_size, p, 2, 3)
    backs = [slabs[r].halo_out(Us[r], p) for r in range(world)]
    pending.update({r: (backs[(r + 1) % world], p) for r in range(world)})


def emulate_finish(slabs, Us, pending):
    for r, (msg, p) in list(pending.items()):
        slabs[r].boundary_in(Us[r], p, msg)
    pending.clear()


def gpu_or_slices(omega: float = 1.7, gauge: str = "landau", precision: str = "double"):
    """run_slices for SlabExchange: the library's OR pass over a range of timeslices
    (gf_step_slices) on the local lattice, CUDA tensors."""
    import ctypes

    from . import _lib

    g = {"landau": _lib.GF_LANDAU, "mag": _lib.GF_MAG, "u1xu1": _lib.GF_U1XU1}.get(gauge)
    if g is None:
        raise ValueError("t-slabs are for the 4D gauges (landau, mag, u1xu1)")
    real = _lib.GF_FP64 if precision in ("double", "fp64") else _lib.GF_FP32
    sizes = {}

    def run(U, local_size, parity, t_begin, t_end):
        if t_end <= t_begin:
            return
        s = sizes.get(local_size)
        if s is None:
            s = sizes[local_size] = _lib.size_arg(local_size)
        import torch

        stream = torch.cuda.current_stream().cuda_stream
        _lib.check(_lib.lib().gf_step_slices(g, real, 0, ctypes.c_void_p(U.data_ptr()), s, parity, ctypes.c_float(omega),
                                             0, 0, t_begin, t_end, ctypes.c_void_p(stream)), "gf_step_slices")

    return run


def gpu_step_slices(slab: TSlab, algo: str = "or", param: float = 1.7, gauge: str = "landau",
                    precision: str = "double", seed: int = 0, counter: int = 0):
    """run_slices for SlabExchange with any update rule: the library's pass over a range of the
    slab's timeslices (gf_step_slices_at) whose random draws are the whole lattice's
    (`slab.rng_site_offset`); the pass of parity p draws with counter + p, as the reference's
    drivers advance the counter per pass."""
    import ctypes

    from . import _lib

    g = {"landau": _lib.GF_LANDAU, "mag": _lib.GF_MAG, "u1xu1": _lib.GF_U1XU1}.get(gauge)
    if g is None:
        raise ValueError("t-slabs are for the 4D gauges (landau, mag, u1xu1)")
    a = {"or": 0, "micro": 1, "sa": 2, "sr": 3, "random": 4}[algo]
    real = _lib.GF_FP64 if precision in ("double", "fp64") else _lib.GF_FP32
    sizes = {}

    def run(U, local_size, parity, t_begin, t_end):
        if t_end <= t_begin:
            return
        s = sizes.get(local_size)
        if s is None:
            s = sizes[local_size] = _lib.size_arg(local_size)
        import torch

        stream = torch.cuda.current_stream().cuda_stream
        _lib.check(_lib.lib().gf_step_slices_at(g, real, a, ctypes.c_void_p(U.data_ptr()), s, parity,
                                                ctypes.c_float(param), seed, counter + parity, t_begin, t_end,
                                                ctypes.c_longlong(slab.rng_site_offset), ctypes.c_void_p(stream)),
                   "gf_step_slices_at")

    return run


def gpu_or_pass(omega: float = 1.7, gauge: str = "landau", precision: str = "double"):
    """run_pass for parity_pass: the library's in-place plugin pass (gf_or_step) on the local
    lattice, CUDA tensors.  Coulomb's per-timeslice pass is not a slab pass and is refused."""
    from . import plugins

    cls = {"landau": plugins.LandauKernelsSU3, "mag": plugins.MAGKernelsSU3,
           "u1xu1": plugins.U1xU1KernelsSU3}.get(gauge)
    if cls is None:
        raise ValueError("t-slabs are for the 4D gauges (landau, mag, u1xu1)")
    kernels = {}

    def run(U, local_size, parity):
        k = kernels.get(local_size)
        if k is None:
            k = kernels[local_size] = cls(local_size, precision)
        k.orStep(0, 0, U, None, parity, omega)

    return run
