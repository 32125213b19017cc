"""Mixed-precision path (FP32 reconstruction, fluxes and viscous terms; FP64
state update and reductions): error against the FP64 CPU oracle.

Reported as the relative L2 and Linf error of rho, rho u, rho v, E after N
steps and the drift of the conserved totals; the bounds below are the
acceptance thresholds of this path (its target: density L2 error under
1e-5 after 1000 steps on the 2.09M-cell cylinder; here shorter runs on
smaller meshes).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def l2_linf(a, b):
    """Relative L2 and Linf errors of rho, rho u, rho v, E; the momentum
    components are scaled by the momentum magnitude (one of them may be zero
    everywhere)."""
    a = np.asarray(a)
    b = np.asarray(b)
    d = a - b
    mom = np.sqrt(b[:, 1] ** 2 + b[:, 2] ** 2)
    n2 = np.sqrt((b ** 2).sum(axis=0))
    n2[1] = n2[2] = np.sqrt((mom ** 2).sum())
    ninf = np.abs(b).max(axis=0)
    ninf[1] = ninf[2] = mom.max()
    l2 = np.sqrt((d ** 2).sum(axis=0)) / np.maximum(n2, 1e-300)
    linf = np.abs(d).max(axis=0) / np.maximum(ninf, 1e-300)
    return l2, linf


def run(pkg, orc, mesh, cfg, prims, nsteps, **launch):
    s = pkg.setupSolver(mesh, cfg, precision="mixed", **launch)
    s.createFields2d(0, *prims)
    gh = s.propagate2d(nsteps)
    o = orc.Oracle(mesh, cfg, nthreads=4)
    o.init_fields(*prims)
    oh = o.run(nsteps)
    return s, o, s.history(0), oh


@pytest.mark.parametrize("loop", ["cell", "tile"])
def test_mixed_square_100_steps(pkg, orc, loop):
    mesh, cfg, prims = pkg.cases.square_inviscid(101)
    s, o, gh, oh = run(pkg, orc, mesh, cfg, prims, 100, loop=loop)
    U = s.get_state(0)["Ucons"]
    l2, linf = l2_linf(U, o.field("Uold"))
    print("mixed square 100 steps L2", l2, "Linf", linf)
    assert l2[0] < 1e-5 and l2.max() < 1e-4
    # conserved totals follow the FP64 oracle
    for v in range(4):
        assert gh[-1]["totals"][v] == pytest.approx(oh[-1]["totals"][v], rel=1e-5, abs=1e-9)
    assert gh[-1]["dt"] == pytest.approx(oh[-1]["dt"], rel=1e-4)


@pytest.mark.parametrize("loop", ["cell", "tile"])
def test_mixed_cylinder_viscous(pkg, orc, loop):
    mesh, cfg, prims = pkg.cases.cylinder_case(129)
    s, o, gh, oh = run(pkg, orc, mesh, cfg, prims, 100, loop=loop)
    U = s.get_state(0)["Ucons"]
    l2, linf = l2_linf(U, o.field("Uold"))
    print("mixed cylinder 129 100 steps L2", l2, "Linf", linf)
    # measured 1.2e-7 (both loops); the bound leaves a factor of 8
    assert l2[0] < 1e-6
    assert all(h["nonfinite"] == 0 for h in gh)


def test_mixed_cylinder_1000_steps_against_fp64(pkg):
    """The density bound of the mixed path (L2 under 1e-5 after 1000 steps)
    on the viscous cylinder at 129^2: against the FP64 GPU path from the
    same state, which the parity tests hold bit-identical to the oracle
    (the oracle itself would take minutes for 1000 steps here)."""
    mesh, cfg, prims = pkg.cases.cylinder_case(129)
    out = {}
    for prec in ("f64", "mixed"):
        s = pkg.setupSolver(mesh, cfg, precision=prec, loop="tile")
        s.createFields2d(0, *prims)
        s.propagate2d(1000)
        out[prec] = s.get_state(0)["Ucons"]
        assert all(x["nonfinite"] == 0 for x in s.history(0)), prec
        s.close()
    l2, linf = l2_linf(out["mixed"], out["f64"])
    print("mixed vs FP64 cylinder 129, 1000 steps: L2", l2, "Linf", linf)
    # measured 1.0e-6
    assert l2[0] < 1e-5, l2


@pytest.mark.parametrize("flux,loop", [("roe", "cell"), ("ausm", "cell"), ("roe", "tile"), ("ausm", "tile")])
def test_mixed_fluxes_tgv_batch(pkg, orc, flux, loop):
    tg = [pkg.cases.tgv_case(n, 0.2 + 0.1 * k, 400.0 + 300 * k, flux=flux) for k, n in enumerate((33, 49, 41))]
    s = pkg.solver.Solver([m for m, _, _ in tg], [c for _, c, _ in tg],
                          pkg.solver.make_launch(precision="mixed", loop=loop))
    for i, (_, _, p) in enumerate(tg):
        s.createFields2d(i, *p)
    s.propagate2d(50)
    for i, (m, c, p) in enumerate(tg):
        o = orc.Oracle(m, c, nthreads=2)
        o.init_fields(*p)
        oh = o.run(50)
        l2, _ = l2_linf(s.get_state(i)["Ucons"], o.field("Uold"))
        assert l2[0] < 1e-5, (flux, i, l2)
        ek_gpu = s.history(i)[-1]["Ek"]
        assert ek_gpu == pytest.approx(oh[-1]["Ek"], rel=1e-5)


def test_mixed_tile_quads(pkg, orc):
    mesh, cfg, prims = pkg.cases.reference_tgv_case(41, quads=True)
    s, o, gh, oh = run(pkg, orc, mesh, cfg, prims, 20, loop="tile")
    l2, _ = l2_linf(s.get_state(0)["Ucons"], o.field("Uold"))
    assert l2[0] < 1e-5 and l2.max() < 1e-4, l2
