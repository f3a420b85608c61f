"""B200-native CubismUP_2D timestep pipeline.

The product is the CUDA library ``libcup2d.so`` (C ABI in include/cup2d.h);
this package holds its sources (csrc/), the in-tree build (build.py) and a
ctypes binding that mirrors the reference's Simulation/Operator interface
(abi.py).
"""
from .abi import (Context, Simulation, Operator, PutObjectsOnGrid, advDiff, PressureSingle,
                  PressureIterator_unif, advDiffGrav, PressureVarRho_approx, ComputeForces,
                  Cup2DError, Ensemble, parse_args, lib, LIB_PATH, EXPORTS)

__all__ = ["Context", "Simulation", "Operator", "PutObjectsOnGrid", "advDiff", "PressureSingle",
           "PressureIterator_unif", "advDiffGrav", "PressureVarRho_approx", "ComputeForces",
           "Cup2DError", "Ensemble", "parse_args", "lib", "LIB_PATH", "EXPORTS"]
