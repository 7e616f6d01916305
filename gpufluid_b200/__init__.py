"""B200-native FLIP/PIC/APIC substep for GPUFLUID's FlipSolver3D.

The per-substep hot path (binning, P2G, forces/BC/divergence, Jacobi/GS-RB/PCG
pressure, projection, G2P + advection) runs as hand-written sm_100a CUDA in
libgfb200.so, called through the C ABI declared in include/gfb200.h.
"""
from .solver import (FlipSolver3D, FlipDivergenceError, PressureSolveError, DeviceArray,
                     StepProfiler, cfl_substep_count, cfl_substep_count_gpu)

__all__ = ["FlipSolver3D", "FlipDivergenceError", "PressureSolveError", "DeviceArray",
           "StepProfiler", "cfl_substep_count", "cfl_substep_count_gpu"]
