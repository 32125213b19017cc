"""The reference's known-answer operator drivers on the GPU, through the C ABI.

Same cases as tests/test_operator_kats.py (where the CPU oracle is pinned to
them): the twice-applied Green-Gauss Laplacian of phi = (x^4 + y^4)/3
(testDiffOperatorsLaplace.jl:2-8,63-163) through gd2d_calc_diff_term, and the
kinetic-energy decay of the reference's Taylor-Green vortex
(testViscousFluxesTGV2d.jl:167-205,487-488) through gd2d_propagate.
"""
import math

import numpy as np
import pytest

from test_operator_kats import _interior, _operator_case, tgv_ek_run

pytestmark = pytest.mark.gpu


def test_gpu_laplacian_x4y4_known_answer(pkg, orc):
    """calcDiffTerm's viscous term with mu = 1 and rho u = rho v = phi is the
    Laplacian of phi: within 2h of 4x^2 + 4y^2 on cells three spacings from
    the boundary of the 100x100 triangulated square, and within 1e-12 (of the
    largest value) of the oracle's on every cell."""
    h = 0.01
    mesh, cfg = _operator_case(pkg, 101)
    n = mesh.nCells
    x, y = mesh.cell_mid_points[:, 0], mesh.cell_mid_points[:, 1]
    phi = (x ** 4 + y ** 4) / 3.0
    prims = (np.ones(n), phi, phi, np.full(n, 1.0e5))
    s = pkg.setupSolver(mesh, cfg)
    s.createFields2d(0, *prims)
    D = s.calcDiffTerm(0)
    s.close()
    o = orc.Oracle(mesh, cfg, nthreads=4)
    o.init_fields(*prims)
    o.calc_diff_term()
    Do = o.field("Diff")
    exact = 4.0 * x * x + 4.0 * y * y
    inner = _interior(mesh, 3)
    for v in (1, 2):
        assert np.abs(D[:, v] - exact)[inner].max() <= 2.0 * h
        assert np.abs(D[:, v] - Do[:, v]).max() <= 1e-12 * np.abs(Do[:, v]).max()


def test_gpu_tgv_kinetic_energy_known_answer(pkg, orc):
    """The reference's TGV (U=40, P=1e5, mu=1e-2) to t = 0.01 on 41^2, 81^2
    and 161^2 grids: Ek/E0 on the two coarse grids equals the oracle's to
    1e-12, stays below exp(-4 mu t), and the excess dissipation of the scheme
    falls by at least 3.5x per halving of h (second order), reaching below
    0.02% of E0 on the finest grid (oracle: 0.0085%)."""
    def gpu(mesh, cfg, prims, steps):
        s = pkg.setupSolver(mesh, cfg)
        s.createFields2d(0, *prims)
        s.propagate2d(steps)
        h = s.history(0)
        s.close()
        return h

    def cpu(mesh, cfg, prims, steps):
        o = orc.Oracle(mesh, cfg, nthreads=8)
        o.init_fields(*prims)
        return o.run(steps)

    runs = [(41, 2e-5, 500), (81, 2e-5, 500), (161, 1e-5, 1000)]
    ratios = []
    for k, (nn, dt, steps) in enumerate(runs):
        _, r, th = tgv_ek_run(gpu, pkg, nn, dt, steps)
        if k < 2:
            _, ro, _ = tgv_ek_run(cpu, pkg, nn, dt, steps)
            assert r == pytest.approx(ro, rel=1e-12, abs=0), (nn, r, ro)
        assert r < th, (nn, r, th)
        ratios.append(r)
    th = math.exp(-4.0 * 1e-2 * 0.01)
    ex = [th - r for r in ratios]
    assert ex[0] / ex[1] >= 3.5 and ex[1] / ex[2] >= 3.5, ex
    assert ex[2] < 2e-4, ex
