"""B200-native explicit Godunov step for dimaZloy/2D-DNS-godunov-solver-.

The hot path (reconstruction, face fluxes, viscous source, boundary
conditions and the explicit Euler update of calcOneStageMUSCLcpuFast and its
step loop) runs as hand-written sm_100a CUDA kernels in libgodunov2d.so
behind the C ABI of include/godunov2d.h.  This package is the Python host
side: the mesh schema and generators, case definitions and a ctypes mirror
of the reference's setupSolver/propagate2d call shape.
"""
from . import mesh, cases, solver  # noqa: F401
from .mesh import Mesh2d  # noqa: F401
from .solver import Solver, propagate_until_converged, setupSolver, updateResidualSA  # noqa: F401


def build(force: bool = False, verbose: bool = False) -> str:
    from . import native_build as _b
    return _b.build(force=force, verbose=verbose)
