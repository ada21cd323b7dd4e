"""fr_learn_b200 -- B200-native flux-reconstruction residual + Runge-Kutta path.

A drop-in for FlurryPP's solver::calcResidual / update / timeStepA / timeStepB /
calcDt path (Alchemist1zaq/fr_learn), running as hand-written sm_100a kernels
behind the C ABI in include/frgpu.h (libfrgpu.so, built in-tree).
"""
from .mesh import BC, Mesh, box2d, box3d, bump2d, concat_meshes  # noqa: F401
from .solver import FRG_FP64, FRG_MIXED, Ensemble, FrgError, Solver, default_params, lib, read_gmsh  # noqa: F401

__all__ = ["BC", "Mesh", "box2d", "box3d", "bump2d", "concat_meshes", "FRG_FP64", "FRG_MIXED", "Ensemble", "FrgError", "Solver",
           "default_params", "lib", "read_gmsh"]
