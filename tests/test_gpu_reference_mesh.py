"""The reference's own mesh (oblickShock2dl00F1n.h5: 3,592 triangles and 246
quads, non-unit node_stencils, and the reference generator's tri/quad
up/down node convention) through the CUDA step, against the CPU oracle."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_mesh(pkg):
    return pkg.mesh.Mesh2d.load_npz(os.path.join(HERE, "golden", "oblique_shock_mesh.npz"))


def shock_case(pkg, flux="ausm", limiter="minmod"):
    mesh = reference_mesh(pkg)
    g = 1.4
    cfg = {"thermo": dict(pkg.cases.AIR), "flux": flux, "limiter": limiter, "viscosity": "none", "dt_mode": 2,
           "CFL": 0.4, "beta": 1.0, "ksi": 1.0e-12, "init_nodes": 0,
           # tags of the file: -4 left (x=0), -2 right (x=4.1), -3 bottom, -1 top
           "bc": [{"tag": -4, "kind": "inflow", "rho": 1.0, "u": 2.0, "v": 0.0, "p": 1.0 / g},
                  {"tag": -1, "kind": "inflow", "rho": 1.0, "u": 2.0, "v": 0.0, "p": 1.0 / g},
                  {"tag": -2, "kind": "outflow"}, {"tag": -3, "kind": "slip"}]}
    n = mesh.nCells
    xc, yc = mesh.cell_mid_points[:, 0], mesh.cell_mid_points[:, 1]
    rho = 1.0 + 0.1 * np.sin(3 * xc) * np.cos(5 * yc)
    prims = (rho, np.full(n, 2.0), 0.1 * np.sin(2 * yc), np.full(n, 1.0 / g))
    return mesh, cfg, prims


@pytest.mark.parametrize("order", ["natural", "hilbert"])
def test_reference_mesh_inviscid_bit_exact(pkg, orc, order):
    mesh, cfg, prims = shock_case(pkg)
    s = pkg.setupSolver(mesh, cfg, order=order)
    s.createFields2d(0, *prims)
    o = orc.Oracle(mesh, cfg, nthreads=4)
    o.init_fields(*prims)
    for _ in range(25):
        a = s.propagate2d(1)[0]
        b = o.step()
        assert a["dt"] == b["dt"]
    g = s.get_state(0)
    assert np.array_equal(g["Ucons"], o.field("Uold"))
    assert np.array_equal(g["node_prims"], o.node_prims())


def test_reference_mesh_viscous_and_roe(pkg, orc):
    mesh, cfg, prims = shock_case(pkg, flux="roe", limiter="venkat")
    cfg = dict(cfg, viscosity="constant", mu_ref=1e-3, Pr=0.72, art_viscosity=1)
    s = pkg.setupSolver(mesh, cfg)
    s.createFields2d(0, *prims)
    s.propagate2d(20)
    o = orc.Oracle(mesh, cfg, nthreads=4)
    o.init_fields(*prims)
    o.run(20)
    U = s.get_state(0)["Ucons"]
    ref = o.field("Uold")
    err = (np.abs(U - ref).max(axis=0) / np.abs(ref).max(axis=0)).max()
    assert err <= 1e-10, err
