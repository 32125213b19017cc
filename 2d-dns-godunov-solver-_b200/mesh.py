"""Mesh schema of the reference solver and synthetic mesh generators.

``Mesh2d`` holds exactly the arrays of the reference's ``mesh2d_Int32``
(primeObjects.jl:109-135) as read by ``readMesh2dHDF5`` (utilsIO.jl:107-252):
column-major (Fortran-order) numpy arrays with 1-based Int32 indices and
negative boundary tags in ``cell_stiffness``.  The conventions were checked
on the reference's own mesh file (oblickShock2dl00F1n.h5):

* cell nodes are counter-clockwise; edge k joins nodes (k, k+1);
* ``cells2nodes[:, 2k-2:2k]`` is edge k's node pair;
* ``cell_edges_Nx/Ny`` are unit INWARD normals ``(-ey, ex)/L``;
* ``cell_areas`` is the shoelace area, ``cell_mid_points`` the vertex mean,
  ``HX`` the longest edge;
* ``node2cellL2down[:, 2k-2]`` is the own vertex opposite edge k and
  ``node2cellL2up[:, 2k-2]`` the neighbour's far vertex (quads: the node
  pair of the opposite edge in slots 2k-2, 2k-1); 0 on boundary faces;
* ``cell_clusters`` lists each node's cells in ascending order, 0-padded to
  ``nNeibCells`` (8), with weights ``node_stencils``.

The generators build structured triangulations (each grid quad cut along its
(x0,y0)->(x1,y1) diagonal), optionally periodic, jittered or with cells
removed inside a circle (a staircase cylinder), and structured quad meshes.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Dict, Optional

import numpy as np

TAG_INFLOW = -1
TAG_OUTFLOW = -2
TAG_SLIP = -3
TAG_WALL = -4

MESH_INT_FIELDS = ("mesh_connectivity", "cell_stiffness", "cells2nodes", "cell_clusters",
                   "node2cellL2up", "node2cellL2down", "bc_data", "bc_indexes")
MESH_FLOAT_FIELDS = ("xNodes", "yNodes", "cell_nodes_X", "cell_nodes_Y", "cell_mid_points",
                     "cell_areas", "HX", "cell_edges_Nx", "cell_edges_Ny", "cell_edges_length",
                     "node_stencils")


@dataclasses.dataclass
class Mesh2d:
    """mesh2d_Int32 (primeObjects.jl:109-135)."""

    nCells: int
    nNodes: int
    nNeibCells: int
    nBSets: int
    xNodes: np.ndarray
    yNodes: np.ndarray
    mesh_connectivity: np.ndarray  # (nCells, 7) int32
    bc_data: np.ndarray
    bc_indexes: np.ndarray
    cell_nodes_X: np.ndarray  # (nCells, 4)
    cell_nodes_Y: np.ndarray
    cell_mid_points: np.ndarray  # (nCells, 2)
    cell_areas: np.ndarray
    HX: np.ndarray
    cell_edges_Nx: np.ndarray  # (nCells, 4)
    cell_edges_Ny: np.ndarray
    cell_edges_length: np.ndarray
    cell_stiffness: np.ndarray  # (nCells, 4) int32
    cell_clusters: np.ndarray  # (nNodes, nNeibCells) int32
    node_stencils: np.ndarray  # (nNodes, nNeibCells)
    node2cellL2up: np.ndarray  # (nCells, 8) int32
    node2cellL2down: np.ndarray
    cells2nodes: np.ndarray  # (nCells, 8) int32

    def __post_init__(self):
        for name in MESH_INT_FIELDS:
            setattr(self, name, np.asfortranarray(getattr(self, name), dtype=np.int32))
        for name in MESH_FLOAT_FIELDS:
            setattr(self, name, np.asfortranarray(getattr(self, name), dtype=np.float64))
        self.nCells = int(self.nCells)
        self.nNodes = int(self.nNodes)
        self.nNeibCells = int(self.nNeibCells)

    @property
    def has_quads(self) -> bool:
        return bool((self.mesh_connectivity[:, 2] == 4).any())

    def arrays(self) -> Dict[str, np.ndarray]:
        return {f.name: getattr(self, f.name) for f in dataclasses.fields(self)}

    def save_npz(self, path: str) -> None:
        d = {k: (np.asarray(v) if isinstance(v, np.ndarray) else np.asarray(v))
             for k, v in self.arrays().items()}
        np.savez_compressed(path, **d)

    @classmethod
    def from_arrays(cls, d) -> "Mesh2d":
        kw = {}
        for f in dataclasses.fields(cls):
            v = d[f.name]
            kw[f.name] = np.asarray(v) if np.ndim(v) else int(np.asarray(v))
        return cls(**kw)

    @classmethod
    def load_npz(cls, path: str) -> "Mesh2d":
        with np.load(path) as z:
            return cls.from_arrays({k: z[k] for k in z.files})

    def validate(self) -> None:
        """Structural invariants the step relies on; raises ValueError."""
        nc, nn = self.nCells, self.nNodes
        mc = self.mesh_connectivity
        if mc.shape != (nc, 7):
            raise ValueError("mesh_connectivity must be (nCells, 7)")
        nf = mc[:, 2]
        if not np.isin(nf, (3, 4)).all():
            raise ValueError("cells must have 3 or 4 nodes")
        typ = mc[:, 1]
        if not ((typ == 3) == (nf == 3)).all():
            raise ValueError("cell type code (3 tri / 2 quad) disagrees with node count")
        cs = self.cell_stiffness
        for k in range(4):
            live = nf > k
            nb = cs[live, k]
            if ((nb > nc) | (nb == 0)).any():
                raise ValueError("cell_stiffness holds an out-of-range neighbour or 0 on a live face")
        if (self.cell_areas <= 0).any():
            raise ValueError("non-positive cell area")
        cl = self.cell_clusters
        if cl.shape != (nn, self.nNeibCells) or (cl < 0).any() or (cl > nc).any():
            raise ValueError("cell_clusters out of range")
        for arr, name in ((self.node2cellL2up, "node2cellL2up"), (self.node2cellL2down, "node2cellL2down"),
                          (self.cells2nodes, "cells2nodes")):
            if (arr < 0).any() or (arr > nn).any():
                raise ValueError(name + " out of range")


# --------------------------------------------------------------------------
# generators


def _finish_mesh(cell_nodes: np.ndarray, nnodes_per_cell: np.ndarray, vx: np.ndarray, vy: np.ndarray,
                 node_x: np.ndarray, node_y: np.ndarray, boundary_tag: Callable) -> Mesh2d:
    """Build every derived array from cells given as merged 0-based node ids
    ``cell_nodes (nCells, 4)`` (-1 padded), per-cell unwrapped vertex
    coordinates ``vx, vy (nCells, 4)`` and ``boundary_tag(ex0, ey0, ex1, ey1)``
    returning a negative tag per boundary edge."""
    nc = cell_nodes.shape[0]
    nn = node_x.shape[0]
    nf = nnodes_per_cell.astype(np.int64)
    quad = nf == 4
    kk = np.arange(4)
    nxt = np.where(quad[:, None], (kk[None, :] + 1) % 4, np.array([1, 2, 0, 0])[None, :])
    live = kk[None, :] < nf[:, None]
    rows = np.arange(nc)[:, None]
    a_id = cell_nodes
    b_id = cell_nodes[rows, nxt]
    ax, ay = vx, vy
    bx, by = vx[rows, nxt], vy[rows, nxt]
    ex, ey = bx - ax, by - ay
    L = np.sqrt(ex * ex + ey * ey)
    with np.errstate(invalid="ignore", divide="ignore"):
        Nx = np.where(live, -ey / np.where(live, L, 1.0), 0.0)
        Ny = np.where(live, ex / np.where(live, L, 1.0), 0.0)
    L = np.where(live, L, 0.0)
    # shoelace area and vertex mean
    cross = np.where(live, ax * by - bx * ay, 0.0)
    area = 0.5 * cross.sum(axis=1)
    sx = np.where(live, vx, 0.0).sum(axis=1)
    sy = np.where(live, vy, 0.0).sum(axis=1)
    mid = np.stack([sx / nf, sy / nf], axis=1)
    hx = L.max(axis=1)

    # neighbours across edges: match unordered node pairs
    ci, ck = np.nonzero(live)
    ka = a_id[ci, ck].astype(np.int64)
    kb = b_id[ci, ck].astype(np.int64)
    key = np.minimum(ka, kb) * (nn + 1) + np.maximum(ka, kb)
    order = np.argsort(key, kind="stable")
    ks = key[order]
    same_next = np.zeros(len(ks), dtype=bool)
    same_next[:-1] = ks[1:] == ks[:-1]
    if (same_next[:-1] & same_next[1:]).any():
        raise ValueError("non-manifold mesh: an edge is shared by more than two cells")
    nb_cell = np.full(len(ks), -1, dtype=np.int64)
    nb_k = np.full(len(ks), -1, dtype=np.int64)
    idx = np.nonzero(same_next)[0]
    o1, o2 = order[idx], order[idx + 1]
    nb_cell[o1], nb_k[o1] = ci[o2], ck[o2]
    nb_cell[o2], nb_k[o2] = ci[o1], ck[o1]

    stiff = np.zeros((nc, 4), dtype=np.int64)
    interior = nb_cell >= 0
    stiff[ci[interior], ck[interior]] = nb_cell[interior] + 1
    bnd = ~interior
    tags = boundary_tag(ax[ci[bnd], ck[bnd]], ay[ci[bnd], ck[bnd]], bx[ci[bnd], ck[bnd]], by[ci[bnd], ck[bnd]])
    stiff[ci[bnd], ck[bnd]] = tags

    # up / down nodes (1-based)
    up = np.zeros((nc, 8), dtype=np.int64)
    dn = np.zeros((nc, 8), dtype=np.int64)
    ii, kk_i = ci[interior], ck[interior]
    jj, kj = nb_cell[interior], nb_k[interior]
    tri_i = ~quad[ii]
    # triangle: down = own vertex opposite edge k = vertex (k+2)%3
    dn[ii[tri_i], 2 * kk_i[tri_i]] = cell_nodes[ii[tri_i], (kk_i[tri_i] + 2) % 3] + 1
    quad_i = quad[ii]
    dn[ii[quad_i], 2 * kk_i[quad_i]] = cell_nodes[ii[quad_i], (kk_i[quad_i] + 2) % 4] + 1
    dn[ii[quad_i], 2 * kk_i[quad_i] + 1] = cell_nodes[ii[quad_i], (kk_i[quad_i] + 3) % 4] + 1
    tri_j = ~quad[jj]
    up[ii[tri_j], 2 * kk_i[tri_j]] = cell_nodes[jj[tri_j], (kj[tri_j] + 2) % 3] + 1
    quad_j = quad[jj]
    up[ii[quad_j], 2 * kk_i[quad_j]] = cell_nodes[jj[quad_j], (kj[quad_j] + 2) % 4] + 1
    up[ii[quad_j], 2 * kk_i[quad_j] + 1] = cell_nodes[jj[quad_j], (kj[quad_j] + 3) % 4] + 1

    c2n = np.zeros((nc, 8), dtype=np.int64)
    c2n[:, 0::2] = np.where(live, a_id + 1, 0)
    c2n[:, 1::2] = np.where(live, b_id + 1, 0)

    # clusters: ascending cell ids per node
    pc, pk = np.nonzero(live)
    pn = cell_nodes[pc, pk].astype(np.int64)
    o = np.lexsort((pc, pn))
    pn, pc = pn[o], pc[o]
    counts = np.bincount(pn, minlength=nn)
    if counts.max(initial=0) > 8:
        raise ValueError("a node belongs to more than 8 cells")
    start = np.concatenate([[0], np.cumsum(counts)[:-1]])
    slot = np.arange(len(pn)) - start[pn]
    clusters = np.zeros((nn, 8), dtype=np.int64)
    clusters[pn, slot] = pc + 1
    stencils = np.ones((nn, 8))

    conn = np.zeros((nc, 7), dtype=np.int64)
    conn[:, 0] = np.arange(1, nc + 1)
    conn[:, 1] = np.where(quad, 2, 3)
    conn[:, 2] = nf
    conn[:, 3:7] = np.where(live, cell_nodes + 1, 0)

    bcells, bk = ci[bnd], ck[bnd]
    bc_data = np.stack([bcells + 1, nf[bcells], bk + 1], axis=1) if bnd.any() else np.zeros((0, 3))
    bc_idx = tags.astype(np.int64) if bnd.any() else np.zeros(0)
    return Mesh2d(
        nCells=nc, nNodes=nn, nNeibCells=8, nBSets=int(len(np.unique(bc_idx))),
        xNodes=node_x, yNodes=node_y, mesh_connectivity=conn, bc_data=bc_data, bc_indexes=bc_idx,
        cell_nodes_X=np.where(live, vx, 0.0), cell_nodes_Y=np.where(live, vy, 0.0),
        cell_mid_points=mid, cell_areas=area, HX=hx,
        cell_edges_Nx=Nx, cell_edges_Ny=Ny, cell_edges_length=L, cell_stiffness=stiff,
        cell_clusters=clusters, node_stencils=stencils, node2cellL2up=up, node2cellL2down=dn,
        cells2nodes=c2n)


def structured_mesh(nx_nodes: int, ny_nodes: int, x0: float, x1: float, y0: float, y1: float, *,
                    quads: bool = False, jitter: float = 0.0, seed: int = 0, periodic: bool = False,
                    tags: Optional[Dict[str, int]] = None,
                    remove: Optional[Callable[[np.ndarray, np.ndarray], np.ndarray]] = None,
                    hole_tag: int = TAG_WALL) -> Mesh2d:
    """Structured (nx_nodes x ny_nodes) grid on [x0,x1]x[y0,y1].

    Triangles (default): every grid quad (a,b,c,d) is cut along a-c into
    (a,b,c) and (a,c,d).  ``quads=True`` keeps the quads.  ``jitter`` moves
    interior nodes uniformly by up to +-jitter*h (seeded).  ``periodic``
    merges opposite sides (a torus; cell geometry uses unwrapped vertices).
    ``remove(xc, yc)`` drops cells whose centroid it flags; the new
    boundary is tagged ``hole_tag``.  ``tags`` maps 'left','right','bottom',
    'top' to boundary tags (default -1, -2, -3, -3).
    """
    t = {"left": TAG_INFLOW, "right": TAG_OUTFLOW, "bottom": TAG_SLIP, "top": TAG_SLIP}
    if tags:
        t.update(tags)
    hx = (x1 - x0) / (nx_nodes - 1)
    hy = (y1 - y0) / (ny_nodes - 1)
    gi, gj = np.meshgrid(np.arange(nx_nodes), np.arange(ny_nodes), indexing="xy")
    X = x0 + gi * hx
    Y = y0 + gj * hy
    # exact boundary coordinates
    X[:, -1] = x1
    Y[-1, :] = y1
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        dx = rng.uniform(-jitter * hx, jitter * hx, size=X.shape)
        dy = rng.uniform(-jitter * hy, jitter * hy, size=Y.shape)
        inner = np.zeros(X.shape, dtype=bool)
        inner[1:-1, 1:-1] = True
        X = np.where(inner, X + dx, X)
        Y = np.where(inner, Y + dy, Y)
    if periodic:
        mx, my = nx_nodes - 1, ny_nodes - 1
        node_id = (gi % mx) + (gj % my) * mx
        node_x = X[:my, :mx].ravel().copy()
        node_y = Y[:my, :mx].ravel().copy()
    else:
        node_id = gi + gj * nx_nodes
        node_x = X.ravel().copy()
        node_y = Y.ravel().copy()

    qi, qj = np.meshgrid(np.arange(nx_nodes - 1), np.arange(ny_nodes - 1), indexing="xy")
    qi, qj = qi.ravel(), qj.ravel()
    a = (qj, qi)
    b = (qj, qi + 1)
    c = (qj + 1, qi + 1)
    d = (qj + 1, qi)
    if quads:
        corners = [a, b, c, d]
        ids = np.stack([node_id[p] for p in corners], axis=1)
        vx = np.stack([X[p] for p in corners], axis=1)
        vy = np.stack([Y[p] for p in corners], axis=1)
        nper = np.full(len(qi), 4)
    else:
        t1 = [a, b, c]
        t2 = [a, c, d]
        ids1 = np.stack([node_id[p] for p in t1], axis=1)
        ids2 = np.stack([node_id[p] for p in t2], axis=1)
        ids = np.stack([ids1, ids2], axis=1).reshape(-1, 3)
        vx = np.stack([np.stack([X[p] for p in t1], 1), np.stack([X[p] for p in t2], 1)], 1).reshape(-1, 3)
        vy = np.stack([np.stack([Y[p] for p in t1], 1), np.stack([Y[p] for p in t2], 1)], 1).reshape(-1, 3)
        pad = np.full((ids.shape[0], 1), -1)
        ids = np.concatenate([ids, pad], axis=1)
        vx = np.concatenate([vx, np.zeros((vx.shape[0], 1))], axis=1)
        vy = np.concatenate([vy, np.zeros((vy.shape[0], 1))], axis=1)
        nper = np.full(ids.shape[0], 3)
    if remove is not None:
        cx = np.where(np.arange(4)[None, :] < nper[:, None], vx, 0.0).sum(1) / nper
        cy = np.where(np.arange(4)[None, :] < nper[:, None], vy, 0.0).sum(1) / nper
        keep = ~np.asarray(remove(cx, cy), dtype=bool)
        ids, vx, vy, nper = ids[keep], vx[keep], vy[keep], nper[keep]
        # Drop, repeatedly, cells left with two or more faces on the cut
        # boundary (notches of the staircase with a single neighbour).
        while True:
            nfc = nper.max()
            k = np.arange(nfc)
            nxt = np.where(nper[:, None] == 4, (k[None, :] + 1) % 4, np.array([1, 2, 0, 0])[None, :nfc])
            live = k[None, :] < nper[:, None]
            a = ids[:, :nfc].astype(np.int64)
            b = ids[np.arange(len(ids))[:, None], nxt].astype(np.int64)
            key = np.minimum(a, b) * (node_x.shape[0] + 1) + np.maximum(a, b)
            kl = key[live]
            uniq, cnt = np.unique(kl, return_counts=True)
            single = np.zeros(key.shape, dtype=bool)
            single[live] = np.isin(kl, uniq[cnt == 1])
            ax_, ay_ = vx[:, :nfc], vy[:, :nfc]
            bx_, by_ = vx[np.arange(len(ids))[:, None], nxt], vy[np.arange(len(ids))[:, None], nxt]
            outer = (((ax_ == x0) & (bx_ == x0)) | ((ax_ == x1) & (bx_ == x1)) |
                     ((ay_ == y0) & (by_ == y0)) | ((ay_ == y1) & (by_ == y1)))
            cut = (single & ~outer).sum(axis=1)
            drop = cut >= 2
            if not drop.any():
                break
            ids, vx, vy, nper = ids[~drop], vx[~drop], vy[~drop], nper[~drop]
        used = np.zeros(node_x.shape[0], dtype=bool)
        used[ids[ids >= 0]] = True
        remap = np.full(node_x.shape[0], -1, dtype=np.int64)
        remap[used] = np.arange(int(used.sum()))
        ids = np.where(ids >= 0, remap[np.maximum(ids, 0)], -1)
        node_x, node_y = node_x[used], node_y[used]

    def boundary_tag(ax, ay, bx, by):
        out = np.full(ax.shape, hole_tag, dtype=np.int64)
        out[(ax == x0) & (bx == x0)] = t["left"]
        out[(ax == x1) & (bx == x1)] = t["right"]
        out[(ay == y0) & (by == y0)] = t["bottom"]
        out[(ay == y1) & (by == y1)] = t["top"]
        return out

    return _finish_mesh(ids, nper, vx, vy, node_x, node_y, boundary_tag)


def unit_square_mesh(n_nodes: int = 101, jitter: float = 0.1, seed: int = 1) -> Mesh2d:
    """Unit square, n x n nodes, triangulated, interior nodes jittered by
    +-jitter*h; left inflow (-1), right outflow (-2), top/bottom slip (-3)."""
    return structured_mesh(n_nodes, n_nodes, 0.0, 1.0, 0.0, 1.0, jitter=jitter, seed=seed)


def cylinder_mesh(n_nodes: int = 1025, radius: float = 0.5, xlim=(-5.0, 15.0), ylim=(-8.0, 8.0),
                  wall_tag: int = TAG_WALL) -> Mesh2d:
    """[-5,15]x[-8,8] triangulated grid with the cells whose centroid lies
    inside the circle of the given radius removed (staircase wall tagged
    ``wall_tag``); left inflow, right/top/bottom extrapolated outflow."""
    r2 = radius * radius
    return structured_mesh(n_nodes, n_nodes, xlim[0], xlim[1], ylim[0], ylim[1],
                           tags={"left": TAG_INFLOW, "right": TAG_OUTFLOW, "bottom": TAG_OUTFLOW,
                                 "top": TAG_OUTFLOW},
                           remove=lambda xc, yc: xc * xc + yc * yc < r2, hole_tag=wall_tag)


def periodic_square_mesh(n_nodes: int, length: float = 2.0 * np.pi, quads: bool = False) -> Mesh2d:
    """Periodic [0,length]^2 with n x n grid points per side (n-1 distinct)."""
    return structured_mesh(n_nodes, n_nodes, 0.0, length, 0.0, length, periodic=True, quads=quads)


def concat_meshes(meshes) -> Mesh2d:
    """Disjoint union of meshes (indices shifted); used to run several
    independent cases on the CPU oracle as one mesh."""
    cell_off = np.cumsum([0] + [m.nCells for m in meshes])
    node_off = np.cumsum([0] + [m.nNodes for m in meshes])

    def shift(arr, off, keep_negative=False):
        a = np.asarray(arr, dtype=np.int64)
        if keep_negative:
            return np.where(a > 0, a + off, a)
        return np.where(a > 0, a + off, 0)

    out = {}
    out["nCells"] = int(cell_off[-1])
    out["nNodes"] = int(node_off[-1])
    out["nNeibCells"] = 8
    out["nBSets"] = max(m.nBSets for m in meshes)
    cat = lambda name: np.concatenate([getattr(m, name) for m in meshes], axis=0)
    out["xNodes"] = cat("xNodes")
    out["yNodes"] = cat("yNodes")
    conn = []
    for m, co, no in zip(meshes, cell_off, node_off):
        c = np.asarray(m.mesh_connectivity, dtype=np.int64).copy()
        c[:, 0] += co
        c[:, 3:7] = np.where(c[:, 3:7] > 0, c[:, 3:7] + no, 0)
        conn.append(c)
    out["mesh_connectivity"] = np.concatenate(conn)
    out["cell_stiffness"] = np.concatenate([shift(m.cell_stiffness, co, True) for m, co in zip(meshes, cell_off)])
    for name in ("cells2nodes", "node2cellL2up", "node2cellL2down"):
        out[name] = np.concatenate([shift(getattr(m, name), no) for m, no in zip(meshes, node_off)])
    out["cell_clusters"] = np.concatenate([shift(m.cell_clusters, co) for m, co in zip(meshes, cell_off)])
    bcd = []
    for m, co in zip(meshes, cell_off):
        b = np.asarray(m.bc_data, dtype=np.int64).reshape(-1, 3).copy()
        b[:, 0] += co
        bcd.append(b)
    out["bc_data"] = np.concatenate(bcd)
    out["bc_indexes"] = np.concatenate([np.asarray(m.bc_indexes).ravel() for m in meshes])
    for name in ("cell_nodes_X", "cell_nodes_Y", "cell_mid_points", "cell_areas", "HX", "cell_edges_Nx",
                 "cell_edges_Ny", "cell_edges_length", "node_stencils"):
        out[name] = cat(name)
    return Mesh2d(**out)
