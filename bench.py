#!/usr/bin/env python
"""Benchmark: time to gauge-fix a 32^4 Landau configuration to theta < 1e-12.

Workload (one "step"): the 32^4 lattice built from U = exp(i*0.3*H) (H traceless
Hermitian, N(0,1) entries) under a seeded Haar gauge transformation, gauge-fixed
with overrelaxation (omega = 1.7) in mixed precision -- FP32 12-real storage until
theta < 1e-9, then FP64 polish sweeps to theta < 1e-12 -- through the library's
context API: import of the reference-layout (GpuPattern, FP64) field, gf_fix,
export of the reunitarised field.  The same input is also fixed in plain FP64 to
report the mixed/FP64 time-to-theta ratio and the functional error.

Metric: site updates per second over the whole job (sum over ranks of
V x OR sweeps done / max-over-ranks time).  ``value`` has the input resident in
HBM; ``e2e`` runs the same call with pinned host buffers (H2D of rows 0,1 of the
input and D2H of the full output inside the timed region).

Multi-GPU: one process per GPU, each fixing its own configuration (seed + rank);
gauge copies are independent, so there is no data-path collective ("weak").

``--impl reference`` times the reference's path on the host cores instead: the
reference has no CPU implementation, so this is the C restatement of its device
code (oracle/, built with OpenMP over the sites of one parity), each step one FP64
OR sweep of the same 32^4 field.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Gsite-updates/s & HBM GB/s; time-to-theta<1e-12 mixed/batched vs plain FP64"
UNIT = "Gsite-updates/s"
SIZE = (32, 32, 32, 32)
EPS = 0.3
# 8 links x 12 reals x (read + write); the refine-mode FP32 pass also reads and writes the two
# tracked columns of the site's W - 1 (6 complex floats = 48 B each way)
BYTES_PER_SITE_UPDATE = {"fp32": 768, "fp64": 1536, "fp32_refine": 768 + 96}


def pass_kernel_name(code: int, real: str, refine: bool) -> str:
    """The OR-pass kernel an autotuner choice stands for (gf_autotune's output codes)."""
    if code >= 100000:
        return pass_kernel_name(code - 100000, real, refine) + ", three cp.async stages"
    if code >= 10000:
        return pass_kernel_name(code - 10000, real, refine) + ", registers capped"
    if code >= 1000:
        return pass_kernel_name(code - 1000, real, refine) + ", odd-parity passes walked backwards"
    r = "float" if real == "fp32" else "double"
    w = ", W" if refine and real == "fp32" else ""
    if code == 100:
        return f"k_batched_pass_rp<{r}, LANDAU, OR{w}> (register prefetch, persistent)"
    if code == 32:
        return f"k_batched_pass_site<{r}, LANDAU, OR{w}> (one thread per site)"
    if code == 33:
        return f"k_batched_pass_site_staged<LANDAU, OR{w}> (one thread per site, cp.async pipelined)"
    if code == 16:
        return f"k_batched_pass_pair<{r}, LANDAU, OR{w}> (two lanes per site)"
    if code == 116:
        return f"k_batched_pass_pair_rp<{r}, LANDAU, OR{w}> (two lanes per site, register prefetch, persistent)"
    if code == 64:
        return f"k_batched_pass<{r}, LANDAU, OR{w}> (64 registers)"
    if code in (2, 4, 8):
        return f"k_batched_pass_staged<{r}, LANDAU, OR, {code} warps>"
    return f"k_batched_pass<{r}, LANDAU, OR{w}>"


def apply_pass_code(gf, real: str, code: int) -> None:
    """Set the OR-pass launch shape an autotuner code stands for (gf_autotune's output codes)."""
    stages3, code = code >= 100000, code % 100000
    capped, code = code >= 10000, code % 10000
    alternate, code = code >= 1000, code % 1000
    variant, warps = {0: (0, 4), 64: (2, 4), 100: (3, 4), 32: (4, 4), 33: (5, 4), 16: (6, 4), 116: (7, 4),
                      2: (1, 2), 4: (1, 4), 8: (1, 8)}[code]
    gf.set_pass_shape(real, variant, warps)
    gf.set_pass_order(real, alternate, capped)
    if stages3:
        gf.set_pass_stages(real, 3)


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if gpu_id:
            cmd += ["-i", gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.file.flush()
        rows = [r.split(", ") for r in Path(self.file.name).read_text().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.file.name)
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                power.append(float(r[3]))
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        pmax = max(power)
        loaded = [s for s, p in zip(sm, power) if p >= 0.5 * pmax] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": pmax}


def cpu_oracle():
    sys.path.insert(0, str(ROOT / "tests"))
    import _oracle  # the oracle is loaded only for the baseline leg and the reference arm

    return _oracle


def host_cpu_info() -> dict:
    """The host threads this process may use, the CPU model and the load average around a CPU timing
    (the host cores of a GPU box are shared with other users' jobs)."""
    try:
        threads = len(os.sched_getaffinity(0))
    except Exception:
        threads = os.cpu_count() or 1
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return {"threads": threads, "nproc": os.cpu_count(), "model": model, "loadavg_1m": os.getloadavg()[0]}


CPU_SWEEPS = 20
CPU_WARMUP = 3


def cpu_or_sweeps(U, size, sweeps: int = CPU_SWEEPS, warmup: int = CPU_WARMUP) -> dict:
    """FP64 OR sweeps (omega = 1.7, both parities) of the C restatement of the reference's device code
    on every host thread this process may use: `warmup` untimed sweeps, then `sweeps` sweeps timed one
    by one.  The bench's cpu_baseline and the reference arm both time through this function."""
    O = cpu_oracle()
    info = host_cpu_info()
    n_thr = info["threads"]
    W = U.copy()

    def sweep():
        for parity in (0, 1):
            O.step(W, size, O.LANDAU, O.OR, parity, 1.7, nthreads=n_thr)

    for _ in range(warmup):
        sweep()
    times = []
    for _ in range(sweeps):
        t0 = time.perf_counter()
        sweep()
        times.append(time.perf_counter() - t0)
    info["loadavg_1m_after"] = os.getloadavg()[0]
    V = O.volume(size)
    mean = sum(times) / len(times)
    return {"value": V / mean / 1e9, "unit": UNIT, "cores": n_thr, "kind": "port",
            "sweeps": len(times), "warmup": warmup, "s_per_sweep": {"mean": mean, "median": statistics.median(times),
                                                                   "min": min(times), "max": max(times)},
            "host": info,
            "sample": f"{len(times)} FP64 OR sweeps (omega=1.7, after {warmup} untimed) of the 32^4 input, C restatement "
                      f"of the reference's device code (the reference has no CPU path), OpenMP over the sites of a "
                      f"parity on {n_thr} host threads ({info['model']})"}


def run_reference(args):
    rank, _, world = env_rank()
    if rank != 0:
        return
    from su3_ma_gauge_gpu_b200 import synthetic as S

    dev = None
    try:
        import torch

        dev = "cuda" if torch.cuda.is_available() else None
    except Exception:
        pass
    U, _ = S.smooth_config(SIZE, EPS, 1234, device=dev)
    r = cpu_or_sweeps(U, SIZE, sweeps=args.steps, warmup=args.warmup)
    val = r["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["s_per_sweep"]["mean"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "Landau OR sweep of a 32^4 SU(3) lattice (eps=0.3 smooth field under a Haar "
                               "gauge transform), FP64; one step = one sweep (both parities)",
                   "lattice": list(SIZE)},
        "cpu_baseline": r,
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reference_gpu_leg(dU_in, gpu_id, fixes) -> dict | None:
    """The reference's own CUDA kernels on the same GPU (oracle/_ref, built from the reference tree for
    the 32^4 extent with its Makefile's flags), as the checker of the headline: the Landau app's
    overrelaxation loop (apps/LandauGaugeFixingSU3_4D.cu:244-271) in FP64 on the same input to
    theta < 1e-12, and the per-sweep time of its FP32 and FP64 OR kernels under a clock record.
    `fixes` maps a name to this library's gf_report of the same input; their functional errors
    against the reference path are returned.  None when the reference kernels were not built."""
    import numpy as np
    import torch

    O = cpu_oracle()
    lib64 = O.refgpu("libref_gpu_X32T32_f64.so")
    lib32 = O.refgpu("libref_gpu_X32T32_f32.so")
    if lib64 is None or lib32 is None:
        return None
    V = O.volume(SIZE)
    nn = torch.from_numpy(O.refgpu_neighbours(lib64, SIZE)).cuda()
    out = {}
    clocks = ClockSampler(gpu_id)
    dU = dU_in.clone()
    F, th, n, ms = O.refgpu_or_loop(lib64, 0, dU.data_ptr(), nn.data_ptr(), 1.7, float(np.float32(1e-12)), 20, 100)
    out["fix_fp64"] = {"F": F, "theta": th, "or_sweeps": n, "ms": ms,
                       "note": "reference kernels driven by the Landau app's OR loop; its quality check is the "
                               "reference's single-thread reduction, inside the time"}
    for prec, lib, dt in (("fp32", lib32, torch.float32), ("fp64", lib64, torch.float64)):
        x = dU_in.to(dt)
        for _ in range(3):
            for p in (0, 1):
                lib.refgpu_step(0, 0, x.data_ptr(), None, nn.data_ptr(), p, 1.7, 0, 0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(20):
            for p in (0, 1):
                lib.refgpu_step(0, 0, x.data_ptr(), None, nn.data_ptr(), p, 1.7, 0, 0)
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 20
        nb = 4 if prec == "fp32" else 8
        out[f"or_sweep_{prec}"] = {"ms_per_sweep": t, "gsite_updates_per_s": V / (t * 1e-3) / 1e9,
                                   "GBs_192B_per_site": 192 * nb * V / (t * 1e-3) / 1e9}
        del x
    out["clocks"] = clocks.stop()
    out["F_rel_err_vs_reference"] = {k: abs(r.gff - F) / abs(F) for k, r in fixes.items()}
    del dU, nn
    torch.cuda.empty_cache()
    return out


def run_profile_target_sa(nsweeps: int):
    """A short launch sequence of the MAG heat-bath pass for ncu: the MAG 48^4 workload's field
    construction at 32^4 (U = exp(i*0.5*H) under a Haar gauge transform) in a refine context,
    `nsweeps` SA sweeps at T = 0.7 with the two-lane direct pass (the shape SA runs with when the
    OR pass is the two-lane register-prefetch one), then with one thread per site."""
    import torch

    from su3_ma_gauge_gpu_b200 import synthetic as S
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    dU, _ = S.smooth_config(SIZE, 0.5, 4849, device="cuda", as_tensor=True)
    torch.cuda.empty_cache()
    with GaugeFixer([SIZE], gauge="mag", mixed="refine") as gf:
        gf.load(0, dU)
        for variant in (6, 4):
            gf.set_pass_shape("fp32", variant, 4)
            gf.sweeps("sa", nsweeps, 0.7, 9, 1)
        g, a = gf.quality()
    torch.cuda.synchronize()
    print(json.dumps({"profile_target": "ok", "mode": "mag-sa", "sweeps_per_shape": nsweeps, "F": float(g[0]),
                      "theta": float(a[0])}))


def run_profile_target(nsweeps: int, mode: str = "fast"):
    """A short, fixed launch sequence of the hot kernels for ncu (see profiles/): the 32^4 input,
    `nsweeps` OR sweeps per launch shape in FP32, then the same in FP64 (shape = (variant, order):
    gf_set_pass_shape, and gf_set_pass_order with alternate = order & 1, capped = order >> 1).
    mode "fast": FP32 storage; FP32 shapes direct, pipelined, two lanes per site (direct, register
    prefetch, register prefetch with alternating walk, the same register-capped); FP64 direct,
    pipelined (alternating walk).
    mode "refine": FP64 master + FP32 working copy with W; FP32 shapes direct, 64-register, register
    prefetch, thread per site (plain, pipelined), two lanes per site (direct, register prefetch, with
    alternating walk, the same register-capped); then FP64 direct, pipelined (4 warps; with
    alternating walk; the same with three cp.async stages), register prefetch.  A third entry in a
    shape is the stage count (gf_set_pass_stages)."""
    import torch

    from su3_ma_gauge_gpu_b200 import synthetic as S
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer

    dU, _ = S.smooth_config(SIZE, EPS, 1234, device="cuda", as_tensor=True)
    torch.cuda.empty_cache()  # keep the device footprint of the profiled launches small
    if mode == "fast":
        shapes = {"fp32": [(0, 0), (1, 0), (6, 0), (7, 0), (7, 1), (7, 3)], "fp64": [(0, 0), (1, 0), (1, 1)]}
    else:
        shapes = {"fp32": [(0, 0), (2, 0), (3, 0), (4, 0), (5, 0), (6, 0), (7, 0), (7, 1), (7, 3)],
                  "fp64": [(0, 0), (1, 0), (1, 1), (1, 1, 3), (3, 0)]}
    with GaugeFixer([SIZE], mixed=True if mode == "fast" else "refine") as gf:
        gf.load(0, dU)
        for real in ("fp32", "fp64"):
            if real == "fp64":
                gf.to_fp64()
            for variant, order, *stages in shapes[real]:
                gf.set_pass_shape(real, variant, 4)
                gf.set_pass_order(real, bool(order & 1), bool(order >> 1))
                if stages:
                    gf.set_pass_stages(real, stages[0])
                gf.sweeps("or", nsweeps, 1.7)
        g, a = gf.quality()
        gf.store(0, dU)
    torch.cuda.synchronize()
    print(json.dumps({"profile_target": "ok", "sweeps_per_shape": nsweeps, "F": float(g[0]), "theta": float(a[0])}))


def run_launch_list(args):
    """One step of the headline workload (import + gf_fix + export of the 32^4 field, the bench's
    mixed mode and schedule) for a profiler's launch list: no warm-up, no clock sampling, the check
    chunks launched directly instead of replayed from CUDA graphs (the same kernels in the same
    order), the step inside the NVTX range "headline_step" (ncu --nvtx --nvtx-include
    "headline_step/").  --pass-fp32 / --pass-fp64 fix the launch shapes by autotuner code (a
    profiler distorts the autotuner's timings); without them the autotuner picks."""
    import torch

    from su3_ma_gauge_gpu_b200 import synthetic as S
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    dU, _ = S.smooth_config(SIZE, EPS, 1234, device="cuda", as_tensor=True)
    torch.cuda.empty_cache()
    out = torch.empty_like(dU)
    sched = Schedule(or_max_iter=20000, precision=1e-12, switch_theta=args.switch_theta, check_precision=args.check,
                     fold=args.fold, reproject=100, micro_updates=0, use_graphs=0, autotune=0)
    with GaugeFixer([SIZE], mixed="refine" if args.mixed == "refine" else True) as gf:
        gf.load(0, dU)
        if args.pass_fp32 is not None and args.pass_fp64 is not None:
            apply_pass_code(gf, "fp32", args.pass_fp32)
            apply_pass_code(gf, "fp64", args.pass_fp64)
            tuned = (args.pass_fp32, args.pass_fp64)
        else:
            tuned = gf.autotune()
        before = gf.kernel_launches()
        gf.load(0, dU)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("headline_step")
        rep = gf.fix(sched)[0]
        gf.store(0, out)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        step = gf.kernel_launches() - before
    print(json.dumps({"launch_list": "ok", "launches_before_step": before, "launches_in_step": step,
                      "launch_shape": tuned, "or_sweeps": rep.or_sweeps, "fp64_sweeps": rep.or_sweeps_fp64,
                      "theta": rep.theta}))


GRIBOV_LATTICES = [((12, 12, 12, 12), 24), ((16, 16, 16, 16), 24), ((40, 20, 20, 20), 16)]


def _clocked(fn, gpu_id=None):
    """Run fn() -> dict under an nvidia-smi clock record; the record goes into the dict."""
    clocks = ClockSampler(gpu_id)
    try:
        r = fn()
    finally:
        clk = clocks.stop()
    r["clocks"] = clk
    return r


def _timed_fix(gf, loads, sched, steps, warmup, stream):
    """warmup + steps full fixes (import, gf_fix) timed with CUDA events; returns (ms, reports)."""
    import torch

    reps = None
    for _ in range(warmup):
        for i, U in enumerate(loads):
            gf.load(i, U)
        reps = gf.fix(sched)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(max(1, steps)):
        for i, U in enumerate(loads):
            gf.load(i, U)
        reps = gf.fix(sched)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / max(1, steps), reps


def run_gribov(args, steps=None, warmup=None, shard=None):
    """64 random-gauge-start Gribov copies of three uneven lattices (24 x 12^4, 24 x 16^4,
    16 x 20^3x40, eps = 0.3 smooth fields), all fixed in ONE batch: every parity pass is one
    launch over all copies, per-copy convergence decided on the device, check chunks replayed
    from CUDA graphs, autotuned pass shape, refine mixed precision (FP32 working copies on an
    FP64 master).  Reports copies/s and the best functional per lattice.  shard = (rank, world):
    this rank fixes its share of the copies, balanced by volume (distributed.shard_weighted)."""
    import numpy as np
    import torch

    from su3_ma_gauge_gpu_b200 import synthetic as S
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    dbases = [S.smooth_config(size, EPS, 500 + k, device="cuda", as_tensor=True)[0]
              for k, (size, _) in enumerate(GRIBOV_LATTICES)]
    sizes, owner = [], []
    for k, (size, n) in enumerate(GRIBOV_LATTICES):
        sizes += [size] * n
        owner += [k] * n
    if shard is not None:
        from su3_ma_gauge_gpu_b200.distributed import shard_weighted

        mine = shard_weighted([float(np.prod(sz)) for sz in sizes], shard[0], shard[1])
        sizes = [sizes[i] for i in mine]
        owner = [owner[i] for i in mine]
    stream = torch.cuda.Stream()
    sched = Schedule(random_trafo=1, seed=77, or_max_iter=20000, precision=1e-12, switch_theta=1e-9,
                     check_precision=args.check, reproject=100, micro_updates=0)
    with GaugeFixer(sizes, mixed="refine", stream=stream) as gf:
        gf.load(0, dbases[0])
        gf.autotune()
        ms, reps = _timed_fix(gf, [dbases[k] for k in owner], sched, steps, warmup, stream)
    vols = [int(np.prod(s)) for s in sizes]
    updates = sum(v * r.or_sweeps for v, r in zip(vols, reps))
    best = {}
    for k, (size, _) in enumerate(GRIBOV_LATTICES):
        fs = sorted((r.gff for r, o in zip(reps, owner) if o == k), reverse=True)
        if len(fs) >= 2:
            best["x".join(map(str, size))] = {"best_F": fs[0], "second_F": fs[1], "min_F": fs[-1], "copies": len(fs),
                                              "best_minus_second_rel": (fs[0] - fs[1]) / fs[0]}
    return {"workload": "gribov", "mixed": "refine", "copies": len(sizes), "total_sites": sum(vols),
            "steps": steps, "warmup": warmup, "ms_per_batch": ms, "copies_per_s": len(sizes) / (ms * 1e-3),
            "gsite_updates_per_s": updates / (ms * 1e-3) / 1e9, "all_converged": all(r.converged for r in reps),
            "max_theta": max(r.theta for r in reps),
            "or_sweeps": {"min": min(r.or_sweeps for r in reps), "max": max(r.or_sweeps for r in reps)},
            "best_per_lattice": best}


def run_plain8(args, steps=None, warmup=None):
    """The 8^4 plain-method configuration: Haar-random links, FP64 (the reference's full 18-real
    array in, out), OR omega = 1.7 to theta < 1e-12, at most 20000 sweeps; timed per fix, once with
    one launch per parity pass (check chunks replayed from CUDA graphs) and once with one persistent
    cooperative launch per check chunk."""
    import numpy as np
    import torch

    from su3_ma_gauge_gpu_b200 import synthetic as S
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    size = (8, 8, 8, 8)
    V = int(np.prod(size))
    U = torch.from_numpy(S.hot_config(size, 4242)).cuda()
    out = torch.empty_like(U)
    stream = torch.cuda.Stream()
    res = {"workload": "plain8", "steps": steps, "warmup": warmup}
    for name, persistent in (("per_pass_launches", 0), ("persistent_chunks", 1)):
        sched = Schedule(or_max_iter=20000, precision=1e-12, check_precision=args.check, reproject=100,
                         micro_updates=0, persistent=persistent)
        with GaugeFixer([size], mixed=False, stream=stream) as gf:
            gf.load(0, U)
            gf.autotune()
            rep = None
            for _ in range(warmup):
                gf.load(0, U)
                rep = gf.fix(sched)[0]
            torch.cuda.synchronize()
            l0 = gf.kernel_launches()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(max(1, steps)):
                gf.load(0, U)
                rep = gf.fix(sched)[0]
                gf.store(0, out)
            e1.record(stream)
            torch.cuda.synchronize()
            launches = (gf.kernel_launches() - l0) / max(1, steps)
        ms = e0.elapsed_time(e1) / max(1, steps)
        res[name] = {"ms_per_fix": ms, "or_sweeps": rep.or_sweeps, "theta": rep.theta, "F": rep.gff,
                     "converged": rep.converged, "us_per_sweep": ms * 1e3 / max(1, rep.or_sweeps),
                     "gsite_updates_per_s": V * rep.or_sweeps / (ms * 1e-3) / 1e9, "kernel_launches": launches}
    return res


def run_coulomb48(args, steps=None, warmup=None):
    """Coulomb gauge on a 48^3 x 16 lattice (eps = 0.3 smooth field under a Haar gauge transform):
    all 16 timeslices fixed as independent instances in the same launches; per slice 500 SA
    sweeps, T 1.0 -> 0.01, a microcanonical sweep after every 3rd SA sweep, then OR omega = 1.7
    to theta < 1e-12; refine mixed precision (FP32 working copy, FP64 master), FP64 reductions."""
    import numpy as np
    import torch

    from su3_ma_gauge_gpu_b200 import synthetic as S
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    size = (16, 48, 48, 48)
    U, _ = S.smooth_config(size, EPS, 4848, device="cuda")
    T = torch.from_numpy(S.gpupattern_to_timeslices(U, size)).cuda()
    del U
    stream = torch.cuda.Stream()
    sched = Schedule(sa_steps=500, sa_min=0.01, sa_max=1.0, micro_updates=1, micro_every=3, or_max_iter=20000,
                     precision=1e-12, switch_theta=1e-9, check_precision=args.check, reproject=100, seed=7)
    with GaugeFixer([size], gauge="coulomb", mixed="refine", stream=stream) as gf:
        gf.load(0, T)
        gf.autotune()
        ms, reps = _timed_fix(gf, [T], sched, steps, warmup, stream)
    V = int(np.prod(size))
    sweeps = sum(r.or_sweeps + r.sa_sweeps for r in reps) / len(reps)
    return {"workload": "coulomb48x16", "mixed": "refine", "steps": steps, "warmup": warmup, "ms_per_fix": ms,
            "timeslices": len(reps), "all_converged": all(r.converged for r in reps),
            "max_theta": max(r.theta for r in reps),
            "or_sweeps": {"min": min(r.or_sweeps for r in reps), "max": max(r.or_sweeps for r in reps)},
            "sa_sweeps": reps[0].sa_sweeps, "mean_F": float(np.mean([r.gff for r in reps])),
            "gsite_updates_per_s": V * sweeps / (ms * 1e-3) / 1e9}


def run_mag48(args, steps=None, warmup=None):
    """Maximal Abelian gauge on a 48^4 lattice, U = exp(i*0.5*H) under a Haar gauge transform: 3000
    SA sweeps (Philox heat-bath, geometric T 1.4 -> 0.01), then OR omega = 1.7, FP32 working copy
    with the gauge transformation tracked (refine mode), FP64 polish to theta < 1e-12.  Then the
    U(1)xU(1) check: 500 OR sweeps of the U1xU1 app's residual diagonal gauge fixing on the
    MAG-fixed field, whose MAG functional sum |U_jj|^2 such diagonal transformations must leave
    unchanged while the U1xU1 functional rises (the U1xU1 theta is the full-matrix Landau measure,
    which diagonal transformations cannot drive to zero).  The input is generated on the GPU and
    stays there."""
    import numpy as np
    import torch

    from su3_ma_gauge_gpu_b200 import synthetic as S
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    stages = {}
    t0 = time.perf_counter()
    size = (48, 48, 48, 48)
    dU, _ = S.smooth_config(size, 0.5, 4849, device="cuda", as_tensor=True)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    stages["input_s"] = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    sched = Schedule(sa_steps=3000, sa_min=0.01, sa_max=1.4, sa_geometric=1, micro_updates=0, or_max_iter=20000,
                     precision=1e-12, switch_theta=1e-9, check_precision=args.check, reproject=100, seed=9)
    t0 = time.perf_counter()
    with GaugeFixer([size], gauge="mag", mixed="refine", stream=stream) as gf:
        gf.load(0, dU)
        gf.autotune()
        ms, reps = _timed_fix(gf, [dU], sched, steps, warmup, stream)
        gf.store(0, dU)  # the MAG-fixed field, reunitarised, in place of the input
    stages["mag_fix_s"] = time.perf_counter() - t0
    r = reps[0]
    V = int(np.prod(size))
    u1 = Schedule(or_max_iter=500, precision=1e-12, switch_theta=1e-9, check_precision=args.check, reproject=100,
                  micro_updates=0)
    t0 = time.perf_counter()
    with GaugeFixer([size], gauge="u1xu1", mixed="refine", stream=stream) as gu:
        gu.load(0, dU)
        f_u1_before = float(gu.quality()[0][0])
        gu.autotune()
        ms_u1, reps_u1 = _timed_fix(gu, [dU], u1, 1, 0, stream)
        gu.store(0, dU)
    stages["u1xu1_s"] = time.perf_counter() - t0
    with GaugeFixer([size], gauge="mag", mixed=False, stream=stream) as gq:
        gq.load(0, dU)
        f_after = float(gq.quality()[0][0])
    ru = reps_u1[0]
    return {"workload": "mag48", "mixed": "refine", "steps": steps, "warmup": warmup, "ms_per_fix": ms,
            "sa_sweeps": r.sa_sweeps, "or_sweeps": r.or_sweeps, "or_sweeps_fp64": r.or_sweeps_fp64, "theta": r.theta,
            "F": r.gff, "converged": r.converged, "footprint_fp32_12_gb": V * 4 * 48 / 1e9,
            "gsite_updates_per_s": V * (r.or_sweeps + r.sa_sweeps) / (ms * 1e-3) / 1e9,
            "u1xu1_check": {"ms": ms_u1, "or_sweeps": ru.or_sweeps, "F_u1_before": f_u1_before,
                            "F_u1_after": ru.gff, "F_mag_after": f_after,
                            "F_mag_rel_change": abs(f_after - r.gff) / abs(r.gff)},
            "wall_s": stages}


EXTRA_CONFIGS = {
    # name: (runner, timed steps, warm-up fixes) for the default run's per-configuration keys
    "plain8": (run_plain8, 3, 1),
    "coulomb48x16": (run_coulomb48, 1, 1),
    "gribov64": (run_gribov, 1, 1),
    "mag48": (run_mag48, 1, 0),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--check", type=int, default=20, help="sweeps between quality checks")
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--switch-theta", type=float, default=1e-9,
                    help="theta at which the mixed run moves from FP32 sweeps to the FP64 polish")
    ap.add_argument("--fold", type=int, default=1, choices=[0, 1],
                    help="refine mode: 1 = iterative refinement below switch-theta (FP32 sweeps folded into "
                         "the FP64 master after every check), 0 = FP64 polish sweeps")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--mixed", default="refine", choices=["fast", "refine"],
                    help="mixed-precision mode of the headline run: fast = FP32 storage converted to FP64 at "
                         "the switch; refine = FP64 master + FP32 working copy + accumulated gauge transform")
    ap.add_argument("--workload", default="landau32", choices=["landau32", "gribov", "plain8", "coulomb48", "mag48"],
                    help="landau32: the headline 32^4 mixed-precision fix; gribov: 64 random-gauge copies of "
                         "uneven lattices in one batch; plain8: the 8^4 Haar-random FP64 plain fix; coulomb48: "
                         "48^3x16 Coulomb, 16 timeslices batched, 500 SA + OR; mag48: 48^4 MAG, 3000 SA + OR")
    ap.add_argument("--extras", default="all",
                    help="comma-separated configurations to run after the headline on a single GPU and report as "
                         "extra keys (plain8, coulomb48x16, gribov64, mag48), 'all' or 'none'")
    ap.add_argument("--profile-mode", default="fast", choices=["fast", "refine", "mag-sa"])
    ap.add_argument("--pass-fp32", type=int, default=None, help="launch-list mode: FP32 pass shape (autotuner code)")
    ap.add_argument("--pass-fp64", type=int, default=None, help="launch-list mode: FP64 pass shape (autotuner code)")
    ap.add_argument("--launch-list", action="store_true",
                    help="one headline step without graphs, warm-up or clock sampling, for ncu's launch list")
    ap.add_argument("--profile", type=int, default=0, metavar="N",
                    help="profiling target: import the 32^4 input, N FP32 OR sweeps, switch to FP64, N FP64 "
                         "sweeps, one quality check; no timing output")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.profile:
        if args.profile_mode == "mag-sa":
            run_profile_target_sa(args.profile)
        else:
            run_profile_target(args.profile, args.profile_mode)
        return
    if args.launch_list:
        run_launch_list(args)
        return
    runners = {"gribov": run_gribov, "plain8": run_plain8, "coulomb48": run_coulomb48, "mag48": run_mag48}
    if args.workload in runners:
        print(json.dumps(_clocked(lambda: runners[args.workload](args))), flush=True)
        return

    import numpy as np
    import torch

    rank, local_rank, world = env_rank()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from su3_ma_gauge_gpu_b200 import synthetic as S
    from su3_ma_gauge_gpu_b200.engine import GaugeFixer, Schedule

    V = int(np.prod(SIZE))
    U_host, f0 = S.smooth_config(SIZE, EPS, 1234 + rank, device="cuda")
    U_pin = torch.from_numpy(U_host).pin_memory()
    U_pin_np = U_pin.numpy()
    out_pin = torch.empty_like(U_pin).pin_memory()
    out_pin_np = out_pin.numpy()
    dU_in = U_pin.cuda()
    dU_out = torch.empty_like(dU_in)
    stream = torch.cuda.Stream()
    sched = Schedule(or_max_iter=20000, precision=1e-12, switch_theta=args.switch_theta, check_precision=args.check,
                     fold=args.fold,
                     reproject=100, micro_updates=0)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def timed(gf, step_fn, steps, warmup, nvtx_name=None):
        reps = None
        for _ in range(warmup):
            reps = step_fn(gf)
        barrier()
        torch.cuda.synchronize()
        l0 = gf.kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if nvtx_name:  # lets a profiler's launch list select exactly the timed steps
            torch.cuda.nvtx.range_push(nvtx_name)
        for _ in range(steps):
            reps = step_fn(gf)
        if nvtx_name:
            torch.cuda.nvtx.range_pop()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1) / steps
        return ms, reps, (gf.kernel_launches() - l0) / steps

    def step_resident(gf):
        gf.load(0, dU_in)
        r = gf.fix(sched)[0]
        gf.store(0, dU_out)
        return r

    def step_host(gf):
        gf.load(0, U_pin_np)
        r = gf.fix(sched)[0]
        gf.store(0, out_pin_np)
        return r

    gpu_id = None
    try:
        gpu_id = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        pass

    mixed_mode = "refine" if args.mixed == "refine" else True
    other_mode = True if args.mixed == "refine" else "refine"
    gf = GaugeFixer([SIZE], mixed=mixed_mode, stream=stream)
    gf.load(0, dU_in)
    tuned = gf.autotune()  # launch shape of the OR pass per precision (0 = direct, else warps/block)
    clocks = ClockSampler(gpu_id)
    ms, rep, launches = timed(gf, step_resident, args.steps, args.warmup, nvtx_name="timed_steps")
    clk = clocks.stop()
    ms_e2e, rep_e2e, _ = timed(gf, step_host, max(1, args.steps - 1), 1)

    # dominant kernels: OR parity passes timed alone on the same stream (CUDA events), per launch
    def pass_ms(nsweeps=20):
        gf.load(0, dU_in)
        gf.sweeps("or", 2, 1.7)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        gf.sweeps("or", nsweeps, 1.7)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / (2 * nsweeps)

    t32 = pass_ms()
    gf.close()

    # the other mixed-precision mode, for the record
    gfo = GaugeFixer([SIZE], mixed=other_mode, stream=stream)
    ms_other, rep_other, _ = timed(gfo, step_resident, 1, 1)
    gfo.close()

    res64 = None
    ms64 = None
    if not args.no_fp64:
        gf64 = GaugeFixer([SIZE], mixed=False, stream=stream)
        ms64, res64, _ = timed(gf64, step_resident, 1, 1)
        gf64.load(0, dU_in)
        gf64.sweeps("or", 2, 1.7)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        gf64.sweeps("or", 10, 1.7)
        e1.record(stream)
        torch.cuda.synchronize()
        t64 = e0.elapsed_time(e1) / 20
        gf64.close()
    else:
        t64 = None

    sweeps = rep.or_sweeps
    site_updates = V * sweeps
    ms_max = max_over_ranks(ms)
    ms_e2e_max = max_over_ranks(ms_e2e)
    total_updates = sum_over_ranks(float(site_updates))
    value = total_updates / (ms_max * 1e-3) / 1e9
    e2e = sum_over_ranks(float(V * rep_e2e.or_sweeps)) / (ms_e2e_max * 1e-3) / 1e9

    peak, peak_kind = measured_peak_hbm()
    Vh = V // 2
    n64 = rep.or_sweeps_fp64
    n32 = sweeps - n64
    # algorithmic bytes (8 links x 12 reals, read and written) -- the roofline's numerator; refine mode's
    # FP32 pass also moves the two tracked columns of W - 1 (reported as gbs_moved)
    b32 = BYTES_PER_SITE_UPDATE["fp32"]
    m32 = BYTES_PER_SITE_UPDATE["fp32_refine" if args.mixed == "refine" else "fp32"]
    kern = {"fp32": {"ms_per_launch": t32, "gbs": Vh * b32 / (t32 * 1e-3) / 1e9, "launches_per_step": 2 * n32,
                     "bytes_per_site_update": b32, "bytes_moved_per_site_update": m32,
                     "gbs_moved": Vh * m32 / (t32 * 1e-3) / 1e9}}
    if t64 is not None:
        kern["fp64"] = {"ms_per_launch": t64, "gbs": Vh * BYTES_PER_SITE_UPDATE["fp64"] / (t64 * 1e-3) / 1e9,
                        "launches_per_step": 2 * n64, "bytes_per_site_update": BYTES_PER_SITE_UPDATE["fp64"]}
    dom = max(kern, key=lambda k: kern[k]["ms_per_launch"] * kern[k]["launches_per_step"])
    # dram bytes of one launch of the chosen kernel, from the ncu summaries (profiles/), keyed by mode and
    # autotuner code; null when that kernel has not been captured
    traffic = None
    tfile = ROOT / "profiles" / "or_pass_traffic.json"
    if tfile.exists():
        try:
            tkey = "fp32_refine" if dom == "fp32" and args.mixed == "refine" else dom
            code = str(tuned[0 if dom == "fp32" else 1])
            traffic = json.loads(tfile.read_text()).get(tkey, {}).get(code)
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": kern[dom]["gbs"], "peak": peak, "unit": "GB/s",
                "frac": kern[dom]["gbs"] / peak, "traffic": traffic,
                "kernel": pass_kernel_name(tuned[0 if dom == "fp32" else 1], dom, args.mixed == "refine")
                + " (one parity pass)",
                "launch_shape": {"fp32": tuned[0], "fp64": tuned[1]},
                "algorithmic_bytes_per_launch": Vh * kern[dom]["bytes_per_site_update"], "peak_kind": peak_kind,
                "per_precision": kern}

    # several GPUs: the Gribov batch sharded over the ranks by volume, no data-path collective
    gribov_sharded = None
    if world > 1:
        g = run_gribov(args, steps=1, warmup=1, shard=(rank, world))
        ms_g = max_over_ranks(g["ms_per_batch"])
        copies = sum_over_ranks(float(g["copies"]))
        updates = sum_over_ranks(g["gsite_updates_per_s"] * g["ms_per_batch"] * 1e-3 * 1e9)
        gribov_sharded = {"ranks": world, "copies": int(copies), "ms_max_over_ranks": ms_g,
                          "copies_per_s": copies / (ms_g * 1e-3), "gsite_updates_per_s": updates / (ms_g * 1e-3) / 1e9,
                          "sharding": "copies by volume (distributed.shard_weighted)"}

    # the checker and the baselines, on rank 0 of a single-GPU run only: the reference's own kernels on
    # this GPU, and the C restatement of its device code on the host cores
    ref_gpu = None
    cpu = None
    extras = {}
    if rank == 0 and world == 1:
        fixes = {"mixed": rep}
        if res64 is not None:
            fixes["fp64"] = res64
        ref_gpu = reference_gpu_leg(dU_in, gpu_id, fixes)
        cpu = cpu_or_sweeps(U_host, SIZE)
        names = list(EXTRA_CONFIGS) if args.extras == "all" else \
            [n for n in args.extras.split(",") if n in EXTRA_CONFIGS]
        del dU_in, dU_out
        torch.cuda.empty_cache()
        for name in names:
            fn, st, wu = EXTRA_CONFIGS[name]
            try:
                extras[name] = _clocked(lambda: fn(args, steps=st, warmup=wu), gpu_id)
            except Exception as e:  # a failing extra configuration is reported, not fatal for the headline
                extras[name] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.empty_cache()

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": "Landau gauge fix of a 32^4 SU(3) lattice to theta<1e-12: U=exp(i*0.3*H) under a "
                               "seeded Haar gauge transform, OR omega=1.7, FP32 12-real sweeps to "
                               f"theta<{args.switch_theta:g}, then "
                               + ("iterative refinement to theta<1e-12 (FP32 sweeps folded into an FP64 master "
                                  "after every check, theta measured on the master in FP64)"
                                  if args.mixed == "refine" and args.fold else "FP64 polish sweeps to theta<1e-12")
                               + f" ({args.mixed} mixed precision); one step = import + gf_fix + export",
                   "lattice": list(SIZE), "instances_per_gpu": 1, "check_every": args.check,
                   "l2": "inputs larger than L2 (FP32 field 201 MB, FP64 403 MB > 126 MB)"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": V * 4 * 12 * 8, "d2h_bytes_per_step": V * 72 * 8,
                "ms_per_step": ms_e2e_max},
        "gpu_launches": int(round(launches)),
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clk,
        "time_to_theta": {
            "mixed_mode": args.mixed, "fold": args.fold, "switch_theta": args.switch_theta,
            "mixed_ms": ms_max, "fp64_ms": ms64,
            "fp64_over_mixed": (ms64 / ms_max) if ms64 else None,
            "mixed": {"or_sweeps": sweeps, "fp64_sweeps": n64, "theta": rep.theta, "F": rep.gff},
            "other_mixed_mode": {"mode": "fast" if args.mixed == "refine" else "refine", "ms": ms_other,
                                 "or_sweeps": rep_other.or_sweeps, "fp64_sweeps": rep_other.or_sweeps_fp64,
                                 "theta": rep_other.theta, "F": rep_other.gff,
                                 "F_rel_err_vs_fp64": (abs(rep_other.gff - res64.gff) / abs(res64.gff))
                                 if res64 else None},
            "fp64": ({"or_sweeps": res64.or_sweeps, "theta": res64.theta, "F": res64.gff} if res64 else None),
            "F_rel_err_vs_fp64": (abs(rep.gff - res64.gff) / abs(res64.gff)) if res64 else None,
            "F_pre_transform": f0,
            "F_rel_vs_pre_transform": (rep.gff - f0) / f0,
            "reference_kernels": ref_gpu,
            "F_rel_err_vs_reference": (ref_gpu or {}).get("F_rel_err_vs_reference"),
            "fp64_gsite_updates_per_s": (V * res64.or_sweeps / (ms64 * 1e-3) / 1e9) if res64 else None,
        },
        "configs": extras,
        "gribov64_sharded": gribov_sharded,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
