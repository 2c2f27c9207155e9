"""B200-native CSRST per-time-step PIC loop.

The physics runs in hand-written sm_100a kernels in libcsrst_gpu.so behind
the C ABI of include/csrst.h; this package is the host-side mirror of the
reference's TETMSolver / PartBunch / ScatterGatherImpl interfaces.
"""
from ._lib import CsrstError, lib  # noqa: F401
from .pic import (Ensemble, IntCIC, IntS1, IntS2, PartBunch, ScatterGatherImpl, ShapeFunction,  # noqa: F401
                  PoissonSolver, Simulation, TETMSolver, moveMesh)
from .workloads import BunchSpec, RunConfig, bend_config, make_bunch, workload  # noqa: F401
