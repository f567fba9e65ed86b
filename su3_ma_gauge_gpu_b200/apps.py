"""The reference's gauge-fixing drivers, batched: configurations from files, gauge copies, the
per-copy functional CSV and the best copy written back.

The reference drivers (apps/LandauGaugeFixingSU3_4D.cu, apps/MAGaugeFixingSU3_4D.cu,
apps/U1xU1GaugeFixingSU3_4D.cu, apps/CoulombGaugeFixingSU3_4D.cu) loop over the files of a
``FileIterator`` (apps/program_options/FileIterator.hxx), and for every file over its gauge
copies one after the other: reload, random gauge transformation, SA (+ micro), SR (MAG), OR,
reprojection, functional, keep the best copy, write it (apps/MAGaugeFixingSU3_4D.cu:151-154,
197-373).  Here all copies of a configuration are instances of ONE context and are fixed
together (every parity pass is one launch over all copies, convergence per copy on the device),
and the file I/O is the GPU transcoder.  Options keep the reference's names and defaults
(apps/program_options/ProgramOptions.hxx:223-266).

Gauge copies run in one of two ways (``copies=``):

* ``"batched"`` (default): all copies of a configuration are instances of ONE context, fixed
  together from the same input; copy c draws its random gauge transformation and heat-bath numbers
  from Philox key word seed + c.  For GF_COULOMB every copy is a lattice of Nt timeslices, and the
  written configuration takes, timeslice by timeslice, the copy with the largest functional of that
  slice (gf_export_slices) -- the rule of apps/CoulombGaugeFixingSU3_4D.cu:303-311.
* ``"reference"``: the apps' own sequence (apps/LandauGaugeFixingSU3_4D.cu:184-283,
  apps/MAGaugeFixingSU3_4D.cu:197-373): copies one after the other, each starting from the best
  copy found so far (the apps reload their host array, which holds it), one Philox counter running
  on through the random transformations, SA and SR sweeps of all copies (PhiloxWrapper's
  process-wide counter, lattice/rng/PhiloxWrapper.hxx:90,142-145), a hot start drawing counter 0.
  For GF_COULOMB with one copy this is the batched fix with ``rng_streams = 1``, which gives every
  timeslice the key word and counters of the app's slice loop; several Coulomb copies run batched.

The precision is compared as a float, like the reference's ``float precision``.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import files
from .engine import GaugeFixer, Schedule


@dataclass
class ProgramOptions:
    """apps/program_options/ProgramOptions.hxx:223-266 (option names and defaults)."""

    output_SA_functional: str = "functional"
    output_conf: str = ""
    output_ending: str = ""
    save_each: bool = False
    doSA: bool = True
    ftype: str = "PLAIN"
    fbasename: str = ""
    fending: str = ".vogt"
    fnumberformat: int = 1
    fstartnumber: int = 0
    fstepnumber: int = 1
    nconf: int = 1
    fappendix: str = "gaugefixed_"
    reinterpret: str = "STANDARD"
    hotgaugefield: bool = False
    seed: int = 1
    gaugecopies: int = 1
    randomtrafo: bool = True
    reproject: int = 100
    sasteps: int = 1000
    samin: float = 0.01
    samax: float = 0.4
    microupdates: int = 3
    ormaxiter: int = 1000
    orparameter: float = 1.7
    srmaxiter: int = 1000
    srparameter: float = 1.7
    precision: float = 1e-7
    checkprecision: int = 100

    @classmethod
    def from_config_file(cls, path, **overrides) -> "ProgramOptions":
        """A boost::program_options config file (``key = value`` lines, ``#`` comments);
        keyword arguments override it, like the reference's command line."""
        fields = {f.name: f for f in dataclasses.fields(cls)}
        vals = {}
        for line in Path(path).read_text().splitlines():
            line = line.split("#", 1)[0].strip()
            if not line or "=" not in line:
                continue
            k, v = (x.strip() for x in line.split("=", 1))
            if k not in fields:
                raise ValueError(f"unknown option {k!r} in {path}")
            t = fields[k].type
            if t in ("bool", bool):
                vals[k] = v.lower() in ("1", "true", "yes", "on")
            elif t in ("int", int):
                vals[k] = int(v)
            elif t in ("float", float):
                vals[k] = float(v)
            else:
                vals[k] = v
        vals.update(overrides)
        return cls(**vals)


class FileIterator:
    """apps/program_options/FileIterator.hxx: the input, output and functional file names."""

    def __init__(self, options: ProgramOptions):
        self.o = options

    def ids(self):
        o = self.o
        return [o.fstartnumber + k * o.fstepnumber for k in range(o.nconf)]

    def _num(self, i: int) -> str:
        return str(i).rjust(self.o.fnumberformat, "0")

    def filename(self, i: int) -> str:
        return f"{self.o.fbasename}{self._num(i)}{self.o.fending}"

    def output_filename(self, i: int) -> str:
        return f"{self.o.output_conf}{self.o.fappendix}{self._num(i)}{self.o.output_ending}"

    def output_functional(self, i: int) -> str:
        return f"{self.o.output_SA_functional}_{self._num(i)}"


def schedule_for(gauge: str, o: ProgramOptions, **extra) -> Schedule:
    """The driver loop of each app as a gf_fix schedule."""
    base = dict(random_trafo=int(o.randomtrafo), seed=int(o.seed), sa_steps=o.sasteps if o.doSA else 0,
                sa_min=o.samin, sa_max=o.samax, micro_updates=o.microupdates, or_max_iter=o.ormaxiter,
                or_parameter=o.orparameter, precision=float(np.float32(o.precision)),
                check_precision=o.checkprecision, reproject=o.reproject)
    if gauge == "mag":
        base.update(sa_mode=2, sa_repeat=5, sa_slow_lo=0.7, sa_slow_hi=0.88, sa_slow_factor=15.0,
                    sr_max_iter=o.srmaxiter, sr_parameter=o.srparameter, sr_stop_theta=1e-6)
    elif gauge == "u1xu1":
        base.update(sa_mode=2, sa_repeat=1, sa_slow_lo=2.0, sa_slow_hi=2.7, sa_slow_factor=15.0)
    base.update(extra)
    return Schedule(**base)


@dataclass
class ConfigResult:
    filename: str
    functionals: list      # per copy (Coulomb: the mean over the copy's timeslices)
    thetas: list
    best_copy: int
    output: str | None


def run(gauge: str, size, options: ProgramOptions, mixed=False, precision="double", copies="batched",
        **schedule_extra):
    """Fix every configuration of the FileIterator with `gaugecopies` copies each; writes the
    per-copy functional CSV ("copy,functional", 17 digits; Coulomb: "copy,timeslice,functional") and
    the best copy (or, with save_each, every improving copy but the last as <output>_<copy+1>, then
    the best).  Returns one ConfigResult per file."""
    if copies not in ("batched", "reference"):
        raise ValueError("copies must be 'batched' or 'reference'")
    size = tuple(int(v) for v in size)
    ncopies = max(1, int(options.gaugecopies))
    layout = "timeslice" if gauge == "coulomb" else "gpu"
    dtype = np.float64 if precision in ("double", "fp64") else np.float32
    it = FileIterator(options)
    out = []
    for i in it.ids():
        fname = it.filename(i)
        U = np.zeros(72 * int(np.prod(size)), dtype=dtype)
        if options.hotgaugefield:
            from .plugins import CommonKernelsSU3
            import torch

            dU = torch.zeros(U.size, dtype=torch.float64 if dtype == np.float64 else torch.float32, device="cuda")
            CommonKernelsSU3(size, precision).setHot(0, 0, dU, None, options.seed, 0)
            U = dU.cpu().numpy()
        else:
            files.read_config(fname, options.ftype, size, U, precision, options.reinterpret, layout=layout)
        if gauge == "coulomb":
            res = _coulomb_copies(size, options, U, mixed, ncopies, copies, schedule_extra)
        elif copies == "reference":
            res = _sequential_copies(gauge, size, options, U, mixed, ncopies, schedule_extra)
        else:
            res = _batched_copies(gauge, size, options, U, mixed, ncopies, schedule_extra)
        functionals, thetas, fields, best, best_field, lines = res
        Path(it.output_functional(i)).write_text("\n".join(lines) + "\n")
        outname = None
        if options.save_each and not options.hotgaugefield:
            bestF = -np.inf
            for c in range(ncopies):
                if functionals[c] > bestF:
                    bestF = functionals[c]
                    if c < ncopies - 1:
                        _save(gauge, size, options, precision, fname, f"{it.output_filename(i)}_{c + 1}", fields[c],
                              layout)
        elif not options.hotgaugefield:
            outname = it.output_filename(i)
            _save(gauge, size, options, precision, fname, outname, best_field, layout)
        out.append(ConfigResult(fname, list(functionals), list(thetas), best, outname))
    return out


def _export(gf, c, U):
    R = np.zeros_like(U)
    gf.store(c, R)
    return R


def _batched_copies(gauge, size, options, U, mixed, ncopies, extra):
    sched = schedule_for(gauge, options, **extra)
    with GaugeFixer([size] * ncopies, gauge=gauge, mixed=mixed) as gf:
        for c in range(ncopies):
            gf.load(c, U)
        gf.fix(sched)
        g, a = gf.quality()
        fields = [_export(gf, c, U) for c in range(ncopies)]
    best = int(np.argmax(g))  # the first of equal maxima, as the apps' strict '>'
    lines = ["copy,functional"] + [f"{c},{g[c]:.17g}" for c in range(ncopies)]
    return list(g), list(a), fields, best, fields[best], lines


def _sequential_copies(gauge, size, options, U, mixed, ncopies, extra):
    """The apps' copy loop: each copy from the best so far, one counter through all copies."""
    counter = 1 if options.hotgaugefield else 0  # setHot drew counter 0
    start = U.copy()
    best_f, best = 0.0, 0
    best_field = U
    g_all, a_all, fields = [], [], []
    with GaugeFixer([size], gauge=gauge, mixed=mixed) as gf:
        gf.load(0, start)
        for c in range(ncopies):
            if not options.hotgaugefield:
                gf.load(0, start)  # the apps copy their host array, which holds the best copy so far
            sched = schedule_for(gauge, options, rng_counter=counter, **extra)
            rep = gf.fix(sched)[0]
            counter += 2 * sched.random_trafo + 2 * rep.sa_sweeps + 2 * rep.sr_sweeps
            R = _export(gf, 0, U)
            g_all.append(rep.gff)
            a_all.append(rep.theta)
            fields.append(R)
            if rep.gff > best_f:
                best_f, best, best_field = rep.gff, c, R
                start = R
    lines = ["copy,functional"] + [f"{c},{g_all[c]:.17g}" for c in range(ncopies)]
    return g_all, a_all, fields, best, best_field, lines


def _coulomb_copies(size, options, U, mixed, ncopies, copies, extra):
    """Coulomb: every copy a lattice of Nt timeslices in one context; the written configuration takes
    each timeslice from its best copy (gf_export_slices).  One copy in "reference" mode draws the
    app's Philox stream slice by slice (rng_streams = 1)."""
    nt = size[0]
    if copies == "reference" and ncopies == 1:
        extra = dict(extra, rng_streams=1)
    sched = schedule_for("coulomb", options, **extra)
    with GaugeFixer([size] * ncopies, gauge="coulomb", mixed=mixed) as gf:
        for c in range(ncopies):
            gf.load(c, U)
        gf.fix(sched)
        g, a = gf.quality()
        g = np.asarray(g).reshape(ncopies, nt)
        a = np.asarray(a).reshape(ncopies, nt)
        fields = [_export(gf, c, U) for c in range(ncopies)]
        pick = [int(np.argmax(g[:, t])) for t in range(nt)]
        best_field = np.zeros_like(U)
        gf.store_slices(pick, best_field)
    lines = ["copy,timeslice,functional"] + [f"{c},{t},{g[c, t]:.17g}" for c in range(ncopies) for t in range(nt)]
    per_copy = list(g.mean(axis=1))
    return per_copy, list(a.max(axis=1)), fields, int(np.argmax(per_copy)), best_field, lines


def _save(gauge, size, options, precision, template, outname, U, layout):
    files.write_config(outname, options.ftype, size, U, precision, options.reinterpret, template=template,
                       sa_steps=options.sasteps, layout=layout)
