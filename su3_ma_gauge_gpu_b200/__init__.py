"""su3_ma_gauge_gpu_b200 -- B200-native (sm_100a) SU(3) lattice gauge fixing.

A drop-in for the gauge-fixing sweep of cuLGT (ilyakudrov/SU3_MA_gauge_GPU):
red/black SU(2)-subgroup site updates with overrelaxation, simulated annealing,
microcanonical and stochastic-relaxation steps for Landau, Coulomb, maximal
Abelian and U(1)xU(1) gauges, plus the gauge functional and theta.  The compute
path is hand-written CUDA in ``libgfix.so`` behind the C ABI of ``include/gfix.h``;
this package is the Python host side over that ABI.
"""
from ._lib import GaugeFixError, lib  # noqa: F401
from .plugins import (  # noqa: F401
    CommonKernelsSU3,
    CoulombKernelsSU3,
    GaugeFixingStats,
    LandauKernelsSU3,
    MAGKernelsSU3,
    U1xU1KernelsSU3,
)

__all__ = [
    "GaugeFixError",
    "lib",
    "CommonKernelsSU3",
    "CoulombKernelsSU3",
    "GaugeFixingStats",
    "LandauKernelsSU3",
    "MAGKernelsSU3",
    "U1xU1KernelsSU3",
]
