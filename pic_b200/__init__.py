"""pic_b200 -- B200 (sm_100a) implementation of the electrostatic PIC time step
of dimad285/PIC behind a C ABI (include/picb200.h, libpicb200.so).

Drop-in modules keep the reference's classes and call signatures:
    Particles.Particles2D, Grid.Grid2D, Solvers.Solver, multigrid.MultigridSolver,
    Boundaries.Boundaries, MCC.read_cross_section / null_collision_method
The fused fast path is simulation.PICSimulation.
"""
from . import _lib  # noqa: F401

__all__ = ["Boundaries", "Consts", "Grid", "MCC", "Particles", "Solvers", "multigrid", "simulation", "workloads"]


def library_path() -> str:
    return _lib.LIB_PATH
