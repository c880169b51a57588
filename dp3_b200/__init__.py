"""dp3_b200: B200-native drop-in for DP3 DDECal's direction-iterative
diagonal and scalar gain solvers (IterativeDiagonalSolver /
IterativeScalarSolver).

  dp3_b200.ddsolve   ctypes binding of the C ABI (include/ddsolve_b200.h)
  dp3_b200.solvers   mirror of dp3::ddecal::SolverBase and its iterative
                     subclasses
  dp3_b200.synth     seeded synthetic observations of the benchmark configs
  dp3_b200.build     in-tree build of the native libraries
"""
from . import ddsolve, solvers  # noqa: F401
from .solvers import (IterativeDiagonalSolver, IterativeScalarSolver,  # noqa: F401
                      SolveData, SolveResult)
