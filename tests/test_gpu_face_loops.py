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


def gpu_state(pkg, mesh, cfg, prims, nsteps, **launch):
    s = pkg.setupSolver(mesh, cfg, **launch)
    s.createFields2d(0, *prims)
    h = s.propagate2d(nsteps)[0]
    st = s.get_state(0)
    s.close()
    return st, h


# TILE_FACES: the fused kernel over per-tile face lists must give exactly the
# cell-centred kernel's results, with pairs evaluated once (AUSM+ with
# Minmod / Venkatakrishnan / no limiter) and without (Roe, van Leer).
@pytest.mark.parametrize("case", ["square", "square_venkat", "square_none", "square_roe", "square_vanleer",
                                  "cylinder", "quads", "reference_mesh"])
def test_tile_faces_equal_cell_loop(pkg, orc, case):
    if case.startswith("square"):
        kw = {"square": {}, "square_venkat": {"limiter": "venkat"}, "square_none": {"limiter": "none"},
              "square_roe": {"flux": "roe"}, "square_vanleer": {"limiter": "vanleer"}}[case]
        mesh, cfg, prims = pkg.cases.square_inviscid(61, **kw)
        n = 30
    elif case == "cylinder":
        mesh, cfg, prims = pkg.cases.cylinder_case(129)
        n = 40
    elif case == "quads":
        mesh, cfg, prims = pkg.cases.reference_tgv_case(41, quads=True)
        n = 20
    else:
        from test_gpu_reference_mesh import shock_case
        mesh, cfg, prims = shock_case(pkg)
        n = 25
    ref, href = gpu_state(pkg, mesh, cfg, prims, n, loop="cell")
    got, hgot = gpu_state(pkg, mesh, cfg, prims, n, loop="tile")
    for k in ("Ucons", "prims", "node_prims"):
        assert np.array_equal(ref[k], got[k]), k
    assert href["dt"] == hgot["dt"] and href["residual"] == hgot["residual"]
    if case in ("square", "square_none"):
        o = orc.Oracle(mesh, cfg, nthreads=4)
        o.init_fields(*prims)
        o.run(n)
        assert np.array_equal(got["Ucons"], o.field("Uold"))


def test_tile_faces_batched_and_block128(pkg):
    # one handle: one flux and viscosity model for all of its cases
    items = [pkg.cases.tgv_case(n, mach, 400.0) for n, mach in ((33, 0.3), (47, 0.2), (29, 0.4))]
    meshes = [m for m, _, _ in items]
    cfgs = [c for _, c, _ in items]
    out = []
    for launch in ({"loop": "cell"}, {"loop": "tile"}, {"loop": "tile", "block": 128}):
        s = pkg.solver.Solver(meshes, cfgs, pkg.solver.make_launch(**launch))
        for i, (_, _, p) in enumerate(items):
            s.createFields2d(i, *p)
        s.propagate2d(15)
        out.append([s.get_state(i)["Ucons"] for i in range(len(items))])
        s.close()
    for other in out[1:]:
        for a, b in zip(out[0], other):
            assert np.array_equal(a, b)
