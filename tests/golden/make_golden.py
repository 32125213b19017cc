"""Generate tests/golden/riemann_pair.json.

The reference's only flux test (testFluxes2d.jl:10-24) feeds one Riemann
pair to its Roe kernel but records no expected values.  This script
evaluates the published AUSM+ (Liou 1996, in the reference's variant with
a12 = min of the numerical sound speeds, AUSMflux2dFast.jl:87-175) and Roe
(Roe 1981 with Harten's fix, RoeFlux2dFast.jl:1-197) fluxes for that pair
in 50-digit arithmetic (mpmath), independently of the C oracle, so the
oracle's double-precision restatement can be checked against it.

It also converts the reference's only shipped mesh, oblickShock2dl00F1n.h5
(3,838 cells: 3,592 triangles and 246 quads, non-unit node_stencils), with
the package's HDF5 reader into tests/golden/oblique_shock_mesh.npz so that
the GPU tests can run the reference's own mesh without the reference
checkout, and records a digest of every dataset in
tests/golden/oblique_shock_mesh.json.

Run: GD2D_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py
(without GD2D_REFERENCE_DIR only the Riemann-pair file is written).
"""
import json
import os

import mpmath as mp

mp.mp.dps = 50


def sign(x):
    return mp.mpf(1) if x > 0 else (mp.mpf(-1) if x < 0 else x)


def ausm_plus(L, R, nx, ny, side, g):
    rl, ul, vl, pl = L
    rr, ur, vr, pr = R
    htl = mp.mpf("0.5") * (ul * ul + vl * vl) + pl / rl + pl / rl / (g - 1)
    htr = mp.mpf("0.5") * (ur * ur + vr * vr) + pr / rr + pr / rr / (g - 1)
    k = 2 * (g - 1) / (g + 1)
    sl, sr = mp.sqrt(k * htl), mp.sqrt(k * htr)
    vnl, vnr = ul * nx + vl * ny, ur * nx + vr * ny
    al = sl * min(mp.mpf(1), sl / abs(vnl))
    ar = sr * min(mp.mpf(1), sr / abs(vnr))
    a12 = min(al, ar)
    ML, MR = vnl / a12, vnr / a12
    beta, alfa = mp.mpf(1) / 8, mp.mpf(3) / 16

    def Mp(M):
        return (M + abs(M)) / 2 if abs(M) >= 1 else (M + 1) ** 2 / 4 + beta * (M * M - 1) ** 2

    def Mm(M):
        return (M - abs(M)) / 2 if abs(M) >= 1 else -(M - 1) ** 2 / 4 - beta * (M * M - 1) ** 2

    def Pp(M):
        return (1 + sign(M)) / 2 if abs(M) >= 1 else (M + 1) ** 2 * (2 - M) / 4 + alfa * M * (M * M - 1) ** 2

    def Pm(M):
        return (1 - sign(M)) / 2 if abs(M) >= 1 else (M - 1) ** 2 * (2 + M) / 4 - alfa * M * (M * M - 1) ** 2

    m = Mp(ML) + Mm(MR)
    p12 = Pp(ML) * pl + Pm(MR) * pr
    mp_, mm_ = (m + abs(m)) / 2, (m - abs(m)) / 2
    return [-(a12 * (mp_ * rl + mm_ * rr)) * side,
            -(a12 * (mp_ * rl * ul + mm_ * rr * ur) + p12 * nx) * side,
            -(a12 * (mp_ * rl * vl + mm_ * rr * vr) + p12 * ny) * side,
            -(a12 * (mp_ * rl * htl + mm_ * rr * htr)) * side]


def roe(L, R, nx, ny, side, g):
    rl, ul, vl, pl = L
    rr, ur, vr, pr = R
    mx, my = -ny, nx
    unl, uml = ul * nx + vl * ny, ul * mx + vl * my
    unr, umr = ur * nx + vr * ny, ur * mx + vr * my
    al, ar = mp.sqrt(g * pl / rl), mp.sqrt(g * pr / rr)
    Hl = al * al / (g - 1) + (ul * ul + vl * vl) / 2
    Hr = ar * ar / (g - 1) + (ur * ur + vr * vr) / 2
    RT = mp.sqrt(rr / rl)
    rho = RT * rl
    u = (ul + RT * ur) / (1 + RT)
    v = (vl + RT * vr) / (1 + RT)
    H = (Hl + RT * Hr) / (1 + RT)
    a = mp.sqrt((g - 1) * (H - (u * u + v * v) / 2))
    un, um = u * nx + v * ny, u * mx + v * my
    drho, dp, dun, dum = rr - rl, pr - pl, unr - unl, umr - uml
    LdU = [(dp - rho * a * dun) / (2 * a * a), rho * dum, drho - dp / (a * a), (dp + rho * a * dun) / (2 * a * a)]
    ws = [abs(un - a), abs(un), abs(un), abs(un + a)]
    d = mp.mpf(1) / 5
    for i in (0, 3):
        if ws[i] < d:
            ws[i] = (ws[i] * ws[i] / d + d) / 2
    Rv = [[1, 0, 1, 1],
          [u - a * nx, mx, u, u + a * nx],
          [v - a * ny, my, v, v + a * ny],
          [H - un * a, um, (u * u + v * v) / 2, H + un * a]]
    diss = [sum(ws[j] * LdU[j] * Rv[i][j] for j in range(4)) for i in range(4)]
    fl = [rl * unl, rl * unl * ul + pl * nx, rl * unl * vl + pl * ny, rl * unl * Hl]
    fr = [rr * unr, rr * unr * ur + pr * nx, rr * unr * vr + pr * ny, rr * unr * Hr]
    return [-(fl[i] + fr[i] - diss[i]) * side / 2 for i in range(4)]


def main():
    # testFluxes2d.jl:10-24
    left = [mp.mpf(1.0), mp.mpf(290.0), mp.mpf(0.0), mp.mpf(7143)]
    right = [mp.mpf("1.7"), mp.mpf("263.72"), mp.mpf("-51.62"), mp.mpf(15282.0)]
    # use the double values the reference stores
    left = [mp.mpf(float(x)) for x in left]
    right = [mp.mpf(float(x)) for x in right]
    nx, ny, side, g = mp.mpf(1), mp.mpf(0), mp.mpf(1), mp.mpf(float(1.4))
    cases = []
    for name, fn in (("ausm", ausm_plus), ("roe", roe)):
        for L, R, tag in ((left, right, "L->R"), (right, left, "R->L")):
            out = fn(L, R, nx, ny, side, g)
            cases.append({"flux": name, "order": tag, "left": [float(x) for x in L], "right": [float(x) for x in R],
                          "nx": 1.0, "ny": 0.0, "side": 1.0, "gamma": 1.4,
                          "expected": [mp.nstr(x, 30) for x in out], "rtol": 1e-12})
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "riemann_pair.json")
    with open(path, "w") as f:
        json.dump({"source": "testFluxes2d.jl:10-24 pair, 50-digit evaluation (make_golden.py)", "cases": cases}, f,
                  indent=1)
    print("wrote", path)
    convert_reference_mesh()


def convert_reference_mesh(src=None):
    """Convert the reference repository's mesh file, found in the checkout
    named by GD2D_REFERENCE_DIR (skipped when that is unset)."""
    import hashlib
    import sys
    import numpy as np
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(os.path.dirname(here))
    sys.path.insert(0, root)
    import __graft_entry__ as graft
    pkg = graft.load_package()
    from importlib import import_module
    h5 = import_module(graft.PKG_NAME + ".hdf5mesh")
    if src is None:
        ref_dir = os.environ.get("GD2D_REFERENCE_DIR")
        if not ref_dir:
            print("GD2D_REFERENCE_DIR not set; reference mesh conversion skipped")
            return
        src = os.path.join(ref_dir, "oblickShock2dl00F1n.h5")
    if not os.path.exists(src):
        print("reference mesh not found; skipped", src)
        return
    ds = h5.read_datasets(src)
    mesh = h5.readMesh2dHDF5(src)
    mesh.save_npz(os.path.join(here, "oblique_shock_mesh.npz"))
    digest = {k: hashlib.sha256(np.ascontiguousarray(np.asarray(v)).tobytes()).hexdigest() for k, v in
              sorted(ds.items())}
    meta = {"source": "oblickShock2dl00F1n.h5 (reference repository), read by hdf5mesh.read_datasets",
            "nCells": int(mesh.nCells), "nNodes": int(mesh.nNodes), "sha256": digest}
    with open(os.path.join(here, "oblique_shock_mesh.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("wrote oblique_shock_mesh.npz/.json", mesh.nCells, mesh.nNodes)


if __name__ == "__main__":
    main()
