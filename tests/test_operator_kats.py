"""The reference's own known-answer operator drivers, restated on the CPU oracle.

The reference checks its viscous operators with three drivers that compare
against analytic answers (it plots them; it records no numbers):

- testDiffOperatorsGrads.jl:3-14,260-355: the node-based Green-Gauss
  gradient (calcScalarFieldGreenGaussNodesBasedGradient, calcGradients.jl:36-139)
  of phi = x^2 y^3 against (2 x y^3, 3 x^2 y^2);
- testDiffOperatorsLaplace.jl:2-8,63-163: that gradient applied twice,
  Lap = d(gradX)/dX + d(gradY)/dY, of phi = (x^4 + y^4)/3 against 4x^2 + 4y^2;
- testViscousFluxesTGV2d.jl:167-205,487-488: the kinetic energy of the
  compressible Taylor-Green vortex (U=40, P=1e5, rho=1, mu=1e-2, L=1) against
  Ek(t)/E0 = exp(-4 mu t / L^2), with E0 = U^2 pi^2 (initfields_TGV2d.jl:2-6).

The reference runs the operator drivers on a 100x100 triangulated square
whose file is not in its repository; the same grid is generated here (the
unit square, every quad cut along one diagonal).  The bounds are the
discretisation error of the scheme, stated per test, with its order of
convergence checked on a refined grid.  Measured values are noted beside
each bound.
"""
import math

import numpy as np
import pytest


def _operator_case(pkg, n_nodes):
    mesh = pkg.mesh.structured_mesh(n_nodes, n_nodes, 0.0, 1.0, 0.0, 1.0)
    cfg = {"thermo": dict(pkg.cases.AIR), "flux": "ausm", "limiter": "minmod", "viscosity": "reference",
           "mu_ref": 1.0, "dt_mode": 0, "dt": 1e-9, "init_nodes": 0,
           "bc": [{"tag": -1, "kind": "outflow"}, {"tag": -2, "kind": "outflow"}, {"tag": -3, "kind": "outflow"}]}
    return mesh, cfg


def _interior(mesh, layers):
    """Cells at least `layers` grid spacings from the boundary (the node means
    of boundary nodes are one-sided, which the reference's drivers also see)."""
    x, y = mesh.cell_mid_points[:, 0], mesh.cell_mid_points[:, 1]
    h = 1.0 / (math.isqrt(mesh.nNodes) - 1)
    return (x > layers * h) & (x < 1 - layers * h) & (y > layers * h) & (y < 1 - layers * h)


def _gradient_error(pkg, orc, n_nodes):
    mesh, cfg = _operator_case(pkg, n_nodes)
    o = orc.Oracle(mesh, cfg, nthreads=4)
    x, y = mesh.cell_mid_points[:, 0], mesh.cell_mid_points[:, 1]
    gx, gy = o.green_gauss_gradient(x * x * y ** 3)
    ddx, ddy = 2.0 * x * y ** 3, 3.0 * x * x * y * y
    inner = _interior(mesh, 2)
    # gradX pairs with -ny (calcGradients.jl:116-126): with inward unit
    # normals it approximates d/dy, and gradY approximates d/dx
    swapped = max(np.abs(gx - ddy)[inner].max(), np.abs(gy - ddx)[inner].max())
    as_named = max(np.abs(gx - ddx)[inner].max(), np.abs(gy - ddy)[inner].max())
    mag = np.abs(np.hypot(gx, gy) - np.hypot(ddx, ddy))[inner].max()
    return swapped, as_named, mag


def test_gradient_x2y3_known_answer(pkg, orc):
    """phi = x^2 y^3 on the 100x100 triangulated unit square (h = 0.01):
    the magnitude of the Green-Gauss gradient matches |grad phi| (what the
    reference's driver plots) within 2h on interior cells (measured 1.19h),
    its components match (d/dy, d/dx) within 4h (measured 2.82h), and the
    error halves when h halves (first order: cell centroids are not the
    centres of the cluster means)."""
    h = 0.01
    swapped, as_named, mag = _gradient_error(pkg, orc, 101)
    assert mag <= 2.0 * h, mag
    assert swapped <= 4.0 * h, swapped
    assert as_named > 0.5, as_named  # not the unswapped pairing
    swapped2, _, mag2 = _gradient_error(pkg, orc, 201)
    assert 1.8 <= swapped / swapped2 <= 2.2, (swapped, swapped2)
    assert 1.8 <= mag / mag2 <= 2.2, (mag, mag2)


def _laplacian(pkg, orc, n_nodes):
    mesh, cfg = _operator_case(pkg, n_nodes)
    o = orc.Oracle(mesh, cfg, nthreads=4)
    x, y = mesh.cell_mid_points[:, 0], mesh.cell_mid_points[:, 1]
    phi = (x ** 4 + y ** 4) / 3.0
    # the driver's composition (testDiffOperatorsLaplace.jl:98-110)
    gx, gy = o.green_gauss_gradient(phi)
    dxx, _ = o.green_gauss_gradient(gx)
    _, dyy = o.green_gauss_gradient(gy)
    lap = dxx + dyy
    # the same operator as calcDiffTerm applies it (calcDiffTerm.jl:88-113,
    # mu = 1): rho = 1 and u = v = phi make rho u = rho v = phi
    n = mesh.nCells
    o.init_fields(np.ones(n), phi, phi, np.full(n, 1.0e5))
    o.calc_diff_term()
    D = o.field("Diff")
    return mesh, lap, D, 4.0 * x * x + 4.0 * y * y


def test_laplacian_x4y4_known_answer(pkg, orc):
    """phi = (x^4 + y^4)/3 on the 100x100 triangulated unit square: the
    twice-applied Green-Gauss Laplacian matches 4x^2 + 4y^2 within 2h on cells
    three spacings from the boundary (measured 1.29h), first order in h, and
    calcDiffTerm's viscous term with mu = 1 is that same Laplacian to 1e-12."""
    h = 0.01
    mesh, lap, D, exact = _laplacian(pkg, orc, 101)
    inner = _interior(mesh, 3)
    err = np.abs(lap - exact)[inner].max()
    assert err <= 2.0 * h, err
    scale = np.abs(lap).max()
    assert np.abs(D[:, 1] - lap).max() <= 1e-12 * scale
    assert np.abs(D[:, 2] - lap).max() <= 1e-12 * scale
    mesh2, lap2, _, exact2 = _laplacian(pkg, orc, 201)
    err2 = np.abs(lap2 - exact2)[_interior(mesh2, 3)].max()
    assert 1.8 <= err / err2 <= 2.2, (err, err2)


def tgv_ek_run(run, pkg, n_nodes, dt, steps):
    """(E0, Ek(t)/E0, theory) for the reference's TGV case on an n_nodes^2
    grid of [0, 2pi]^2, where run(mesh, cfg, prims, steps) returns the step
    statistics."""
    mesh, cfg, prims = pkg.cases.reference_tgv_case(n_nodes)
    cfg = dict(cfg, dt=dt)
    rho, u, v, _ = prims
    e0 = float((0.5 * rho * (u * u + v * v) * mesh.cell_areas).sum())
    hist = run(mesh, cfg, prims, steps)
    t = steps * dt
    mu = cfg["tgv"]["mu"]
    return e0, hist[-1]["Ek"] / e0, math.exp(-4.0 * mu * t)


def test_tgv_kinetic_energy_known_answer(pkg, orc):
    """The reference's TGV (U=40, P=1e5, mu=1e-2; testViscousFluxesTGV2d.jl:167-185):
    E0 equals computeTGV2d_Ek_Theory at t = 0, U^2 pi^2, to 1e-12; Ek(t)/E0
    lies below exp(-4 mu t) (the scheme adds dissipation) and the excess
    shrinks at second order: by at least 3.5x from a 41^2 to an 81^2 grid
    (measured 4.7x), over 500 steps of dt = 2e-5 (t = 0.01, local CFL 0.36 on
    the finer grid; the reference's dt = 1e-7 would need 100,000 steps)."""
    def run(mesh, cfg, prims, steps):
        o = orc.Oracle(mesh, cfg, nthreads=8)
        o.init_fields(*prims)
        return o.run(steps)

    e0, r1, th = tgv_ek_run(run, pkg, 41, 2e-5, 500)
    assert e0 == pytest.approx(40.0 ** 2 * math.pi ** 2, rel=1e-12)
    _, r2, _ = tgv_ek_run(run, pkg, 81, 2e-5, 500)
    assert r1 < th and r2 < th, (r1, r2, th)
    assert (th - r1) / (th - r2) >= 3.5, (r1, r2, th)
