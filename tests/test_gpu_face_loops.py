"""Face-loop variants of the step against the CPU oracle.

FACE_SLOTS evaluates each face once and stores each side's flux in its
(cell, face) slot; the update sums the slots in face order, so with exactly
antisymmetric geometry (n_j = -n_i, equal lengths, as the generators give)
and the odd, symmetric Minmod limiter it reproduces the cell-centred result
bit for bit.  FACE_COLOURED accumulates into the cells colour by colour, so
its flux sums round in colour order: within the FP64 tolerance.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(pkg, orc, mesh, cfg, prims, nsteps, loop):
    s = pkg.setupSolver(mesh, cfg, loop=loop)
    s.createFields2d(0, *prims)
    s.propagate2d(nsteps)
    o = orc.Oracle(mesh, cfg, nthreads=4)
    o.init_fields(*prims)
    o.run(nsteps)
    return s.get_state(0)["Ucons"], o.field("Uold")


def rel(a, b):
    """Max relative error per variable; rho u and rho v are scaled by the
    momentum magnitude (rho v is zero to round-off in the square case)."""
    scale = np.abs(b).max(axis=0)
    scale[1] = scale[2] = np.sqrt(b[:, 1] ** 2 + b[:, 2] ** 2).max()
    return float((np.abs(a - b).max(axis=0) / scale).max())


def test_face_slots_bit_exact_square(pkg, orc):
    mesh, cfg, prims = pkg.cases.square_inviscid(61)
    U, ref = run(pkg, orc, mesh, cfg, prims, 30, "face")
    assert np.array_equal(U, ref)


@pytest.mark.parametrize("loop", ["face", "coloured"])
def test_face_loops_cylinder_viscous(pkg, orc, loop):
    mesh, cfg, prims = pkg.cases.cylinder_case(65)
    U, ref = run(pkg, orc, mesh, cfg, prims, 40, loop)
    assert rel(U, ref) <= 1e-10


def test_face_coloured_square_step_tolerance(pkg, orc):
    mesh, cfg, prims = pkg.cases.square_inviscid(61)
    U, ref = run(pkg, orc, mesh, cfg, prims, 1, "coloured")
    assert rel(U, ref) <= 1e-12
    U, ref = run(pkg, orc, mesh, cfg, prims, 100, "coloured")
    assert rel(U, ref) <= 1e-10
