"""B200-native 3D-RISM solute solver (the hnc3d.c hot path of bgy3d).

The compute path is librism3d.so: hand-written sm_100a CUDA kernels behind
the C ABI of include/rism3d.h.  This package is the Python host mirror of
the reference's solute interface (``hnc3d_run_solute``) plus device-level
access to the residual and Jacobian (``RismContext``).
"""
from ._abi import CLOSURES, RismError, lib  # noqa: F401
from .shard import hnc3d_run_batch_sharded  # noqa: F401
from .sites import MOLECULES, find_molecule, synthetic_solute  # noqa: F401
from .solver import (DEFAULTS, RismContext, hnc3d_run_batch, hnc3d_run_solute, hnc3d_run_solvent,  # noqa: F401
                     hnc3d_solute_grad, problem_data, rism_solvent)
