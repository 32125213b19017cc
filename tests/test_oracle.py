"""CPU checks of the oracle: analytic known answers for the restated
reference formulas (no GPU)."""
import math

import numpy as np
import pytest


def physical_flux(u, nx, ny, gamma):
    """Exact Euler flux F(U).n for primitive state u = (rho, u, v, p)."""
    rho, vx, vy, p = u
    vn = vx * nx + vy * ny
    E = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy)
    return np.array([rho * vn, rho * vx * vn + p * nx, rho * vy * vn + p * ny, (E + p) * vn])


@pytest.mark.parametrize("kind", ["ausm", "roe", "ausm_m2020"])
@pytest.mark.parametrize("state", [(1.0, 0.3, -0.2, 0.8), (1.2, 2.5, 0.4, 0.7), (0.9, -3.0, 1.0, 1.1)])
def test_flux_consistency(orc, kind, state):
    """F(U, U, n) equals minus the physical flux times the face length (the
    reference returns the inward-normal convention -(F.n) L)."""
    g = 1.4
    nx, ny = 0.6, 0.8
    side = 0.37
    f = orc.flux(kind, state, state, nx, ny, side, g)
    ref = -physical_flux(state, nx, ny, g) * side
    assert np.allclose(f, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("kind", ["ausm", "roe"])
def test_flux_antisymmetry_bitwise(orc, kind):
    """F(L, R, n) == -F(R, L, -n) exactly: the two cells of a face add
    opposite fluxes (conservation of the cell-centred scheme)."""
    rng = np.random.default_rng(3)
    for _ in range(200):
        L = np.array([rng.uniform(0.5, 2), rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(0.3, 2)])
        R = np.array([rng.uniform(0.5, 2), rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(0.3, 2)])
        th = rng.uniform(0, 2 * math.pi)
        nx, ny, side = math.cos(th), math.sin(th), rng.uniform(0.01, 1)
        a = orc.flux(kind, L, R, nx, ny, side, 1.4)
        b = orc.flux(kind, R, L, -nx, -ny, side, 1.4)
        if kind == "ausm":
            assert np.array_equal(a, -b)
        else:
            assert np.allclose(a, -b, rtol=1e-13, atol=1e-13 * np.abs(a).max())


def test_ausm_supersonic_upwind(orc):
    """Supersonic flow from L into R (n points from L to R): the AUSM+ flux
    is the physical flux of the upwind (L) state."""
    g = 1.4
    L = (1.0, 3.0, 0.1, 1.0 / g)
    R = (1.3, 2.2, -0.3, 1.2 / g)
    nx, ny = 1.0, 0.0
    f = orc.flux("ausm", L, R, nx, ny, 1.0, g)
    assert np.allclose(f, -physical_flux(L, nx, ny, g), rtol=1e-12)


def test_riemann_pair_golden(orc):
    """The reference's flux test pair (testFluxes2d.jl:10-24) against an
    independent 50-digit evaluation committed in tests/golden."""
    import json
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "riemann_pair.json")
    with open(path) as f:
        gold = json.load(f)
    for case in gold["cases"]:
        f_ = orc.flux(case["flux"], case["left"], case["right"], case["nx"], case["ny"], case["side"], case["gamma"])
        exp = np.array([float(x) for x in case["expected"]])
        assert np.allclose(f_, exp, rtol=case["rtol"], atol=case["rtol"] * np.abs(exp).max()), (case["flux"], f_, exp)


def test_minmod_is_smooth_harmonic(orc):
    L = orc.lib()
    assert L.orc_minmod(1.0, 1.0, 0.0) == 1.0
    assert L.orc_minmod(2.0, -1.0, 0.0) == 0.0
    assert L.orc_minmod(0.0, 5.0, 1e-12) == 0.0
    # (sign x + sign y) |xy| / (|x|+|y|+c): harmonic mean for same signs
    assert L.orc_minmod(1.0, 3.0, 0.0) == pytest.approx(2 * 3 / 4)
    # symmetric and odd
    for x, y in [(0.3, 1.7), (-2.0, -0.1), (1e-9, 3.0)]:
        assert L.orc_minmod(x, y, 1e-12) == L.orc_minmod(y, x, 1e-12)
        assert L.orc_minmod(-x, -y, 1e-12) == -L.orc_minmod(x, y, 1e-12)


def test_venkat_limiter_properties(orc):
    L = orc.lib()
    assert L.orc_venkat(1.0, -1.0, 0.0) == 0.0          # extremum -> first order
    assert L.orc_venkat(1.0, 1e6, 0.0) == pytest.approx(1.0, rel=1e-5)   # limited by the smaller slope
    assert L.orc_venkat(1e6, 1.0, 0.0) == pytest.approx(1.0, rel=1e-5)
    assert L.orc_venkat(1.0, 1.0, 0.0) == pytest.approx(0.75)             # phi(1) = 3/4
    assert L.orc_venkat(1e-3, 1e-3, 1.0) == pytest.approx(1e-3, rel=1e-3) # eps dominates: unlimited
    # continuous across the sign change of the bound (no jump at a local extremum)
    for eps2 in (0.0, 0.1, 10.0):
        assert L.orc_venkat(1.0, 1e-13, eps2) == pytest.approx(L.orc_venkat(1.0, -1e-13, eps2), abs=1e-12)
    # odd in its arguments
    assert L.orc_venkat(-0.3, -0.7, 0.2) == -L.orc_venkat(0.3, 0.7, 0.2)


def test_partition_matches_reference(orc):
    """distibuteCellsInThreadsSA (partMesh2d.jl:2-34): equal ranges, thread 1
    absorbs the remainder."""
    r = orc.partition(4, 10)
    assert r.tolist() == [[1, 4], [5, 6], [7, 8], [9, 10]]
    r = orc.partition(3, 9)
    assert r.tolist() == [[1, 3], [4, 6], [7, 9]]


def test_uniform_flow_preserved(orc, pkg):
    """A uniform state on a jittered periodic mesh stays uniform to
    round-off (free-stream preservation of the cell-centred scheme)."""
    mesh = pkg.mesh.periodic_square_mesh(17)
    cfg = {"thermo": dict(pkg.cases.AIR), "flux": "ausm", "limiter": "minmod", "viscosity": "none",
           "dt_mode": 2, "CFL": 0.5, "bc": [], "init_nodes": 1}
    n = mesh.nCells
    o = orc.Oracle(mesh, cfg, nthreads=2)
    o.init_fields(np.ones(n), np.full(n, 0.5), np.full(n, -0.25), np.full(n, 1.0 / 1.4))
    o.run(5)
    U = o.field("Uold")
    assert np.abs(U[:, 0] - 1.0).max() < 1e-13
    assert np.abs(U[:, 1] - 0.5).max() < 1e-13


def test_green_gauss_exact_for_linear(orc, pkg):
    """On a regular triangulation the unweighted cluster means reproduce a
    linear field at the nodes, so the node-based Green-Gauss gradient
    (calcGradients.jl:36-139) is exact and the twice-applied Laplacian of
    calcDiffTerm vanishes away from the boundary."""
    mesh = pkg.mesh.structured_mesh(21, 21, 0.0, 1.0, 0.0, 1.0)
    n = mesh.nCells
    xc, yc = mesh.cell_mid_points[:, 0], mesh.cell_mid_points[:, 1]
    cfg = {"thermo": dict(pkg.cases.AIR), "flux": "ausm", "limiter": "minmod", "viscosity": "reference",
           "mu_ref": 1.0, "dt_mode": 0, "dt": 1e-9, "init_nodes": 0,
           "bc": [{"tag": -1, "kind": "outflow"}, {"tag": -2, "kind": "outflow"}, {"tag": -3, "kind": "outflow"}]}
    o = orc.Oracle(mesh, cfg, nthreads=2)
    # rho u = 2 + 3x - 5y through u with rho = 1
    o.init_fields(np.ones(n), 2 + 3 * xc - 5 * yc, np.zeros(n), np.full(n, 1.0))
    o.calc_diff_term()
    # interior cells: Laplacian of a linear field is 0
    interior = (xc > 0.15) & (xc < 0.85) & (yc > 0.15) & (yc < 0.85)
    D = o.field("Diff")
    assert np.abs(D[interior, 1]).max() < 1e-7


def test_tgv_energy_decays(orc, pkg):
    """Periodic Taylor-Green vortex: kinetic energy decays monotonically
    at roughly exp(-4 nu t)."""
    mesh, cfg, prims = pkg.cases.tgv_case(33, mach=0.2, re=100.0)
    o = orc.Oracle(mesh, dict(cfg, dt_mode=2, CFL=0.5), nthreads=2)
    o.init_fields(*prims)
    h = o.run(40)
    ek = np.array([s["Ek"] for s in h])
    assert np.all(np.diff(ek) < 0)
    t = h[-1]["flowTime"] + h[-1]["dt"]
    nu = cfg["mu_ref"]
    theory = math.exp(-4.0 * nu * t)
    assert ek[-1] / ek[0] == pytest.approx(theory, rel=0.05)
