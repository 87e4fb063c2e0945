"""fvm3d — B200-native explicit residual-and-update path of FVM-3D-F90.

The compute runs in libfvm3d.so (hand-written sm_100a CUDA kernels behind the
C ABI of include/fvm3d.h). This package is the host-side mirror of the
reference's solver interface: scheme ids and namelist names (abi), the
per-case solver object (solver.Solver), seeded case builders (cases), the
namelist front end (namelist), solution output (output), block partitioning
(partition), the tile / z-chunk autotuner (tuning) and the continuous-batching
server (serving).
"""
from . import abi, cases  # noqa: F401
from .abi import make_config, scheme_index  # noqa: F401
from .solver import FvmError, Solver  # noqa: F401

__all__ = ["abi", "cases", "make_config", "scheme_index", "Solver", "FvmError"]
