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

Differences, stated: copy c draws its random gauge transformation and SA heat-bath numbers from
Philox key word seed + c (the reference advances one global counter across copies); the
precision is compared as a float, like the reference's ``float precision``; for GF_COULOMB the
lattice's timeslices are fixed together and one copy is supported (the reference keeps the best
copy per timeslice).
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
    functionals: list      # per copy (per timeslice for Coulomb)
    thetas: list
    best_copy: int
    output: str | None


def run(gauge: str, size, options: ProgramOptions, mixed=False, precision="double", **schedule_extra):
    """Fix every configuration of the FileIterator with `gaugecopies` copies each; writes the
    per-copy functional CSV ("copy,functional", 17 digits) and the best copy (or, with save_each,
    every improving copy but the last as <output>_<copy+1>, then the best).  Returns one
    ConfigResult per file."""
    size = tuple(int(v) for v in size)
    copies = max(1, int(options.gaugecopies))
    if gauge == "coulomb" and copies != 1:
        raise ValueError("Coulomb: one gauge copy per configuration (the timeslices are fixed together)")
    layout = "timeslice" if gauge == "coulomb" else "gpu"
    dtype = np.float64 if precision in ("double", "fp64") else np.float32
    it = FileIterator(options)
    out = []
    sched = schedule_for(gauge, options, **schedule_extra)
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
        with GaugeFixer([size] * copies, gauge=gauge, mixed=mixed) as gf:
            for c in range(copies):
                gf.load(c, U)
            gf.fix(sched)
            g, a = gf.quality()
            results = []
            for c in range(copies):
                R = np.zeros_like(U)
                gf.store(c, R)
                results.append(R)
        lines = ["copy,functional"] + [f"{c},{g[c]:.17g}" for c in range(len(g))]
        Path(it.output_functional(i)).write_text("\n".join(lines) + "\n")
        best, bestF = 0, -np.inf
        outname = None
        for c in range(copies):
            if g[c] > bestF:
                bestF, best = g[c], c
                if options.save_each and c < copies - 1 and not options.hotgaugefield:
                    _save(gauge, size, options, precision, fname, f"{it.output_filename(i)}_{c + 1}", results[c],
                          layout)
        if not options.hotgaugefield and not options.save_each:
            outname = it.output_filename(i)
            _save(gauge, size, options, precision, fname, outname, results[best], layout)
        out.append(ConfigResult(fname, list(g), list(a), best, outname))
    return out


def _save(gauge, size, options, precision, template, outname, U, layout):
    files.write_config(outname, options.ftype, size, U, precision, options.reinterpret, template=template,
                       sa_steps=options.sasteps, layout=layout)
