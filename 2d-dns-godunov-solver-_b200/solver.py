"""Host-side mirror of the reference's solver interface over the C ABI.

The reference drives one explicit step from Julia (testInviscidFluxesGPUx32.jl,
testViscousFluxesTGV2d.jl): ``readMesh2dHDF5`` -> ``setupSolver_*.jl`` globals
-> ``createFields2d`` -> a loop of ``calcDiffTerm`` /
``calcOneStageMUSCLcpuFast`` / ``updateVariablesSA`` /
``cells2nodesSolutionReconstructionWithStencils`` / residuals.  Here the same
call shape maps onto libgodunov2d.so:

  setupSolver(meshes, cfgs)            -> Solver (gd2d_setup)
  Solver.createFields2d(i, rho,u,v,p)  -> gd2d_set_state
  Solver.propagate2d(nsteps)           -> gd2d_propagate (the whole loop body)
  Solver.calcOneStageMUSCLcpuFast(...) -> gd2d_calc_one_stage
  Solver.updateVariablesSA(i)          -> gd2d_update_variables
  Solver.cells2nodesSolutionReconstructionWithStencils() -> gd2d_cells_to_nodes
  Solver.calcDiffTerm(i)               -> gd2d_calc_diff_term

Every call runs on the GPU; there is no CPU fallback.  Arrays are numpy in
the reference's column-major layout.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .mesh import Mesh2d


def mesh_view(mesh: Mesh2d) -> N.MeshView:
    v = N.MeshView()
    v.n_cells, v.n_nodes, v.n_neib_cells = mesh.nCells, mesh.nNodes, mesh.nNeibCells
    v.x_nodes = mesh.xNodes.ctypes.data
    v.y_nodes = mesh.yNodes.ctypes.data
    for name in ("mesh_connectivity", "cell_stiffness", "cells2nodes", "cell_edges_Nx", "cell_edges_Ny",
                 "cell_edges_length", "cell_areas", "HX", "cell_mid_points", "cell_clusters", "node_stencils",
                 "node2cellL2up", "node2cellL2down"):
        setattr(v, name, getattr(mesh, name).ctypes.data)
    return v


def make_params(cfg: Dict) -> N.Params:
    """gd2d_params from a case configuration dict (see cases.py)."""
    p = N.Params()
    th = cfg["thermo"]
    p.RGAS, p.Gamma = th["RGAS"], th["Gamma"]
    p.Cp, p.mu, p.kGas = th.get("Cp", 1000.0), th.get("mu", 0.0), th.get("kGas", 0.0)
    p.CFL = cfg.get("CFL", 0.5)
    # the reference steps with the fixed solControls.dt
    # (testInviscidFluxesGPUx32.jl:324 only reports the CFL-based tau);
    # the CFL-driven modes are opt-in
    p.dt_mode = int(cfg.get("dt_mode", 0))
    if p.dt_mode == 0 and not cfg.get("dt", 0.0) > 0.0:
        raise ValueError("dt_mode 0 (fixed time step, the reference's solControls.dt) needs a positive 'dt'")
    p.dt = cfg.get("dt", 0.0)
    p.beta = cfg.get("beta", 1.0)
    p.ksi = cfg.get("ksi", 1.0e-12)
    p.venkat_K = cfg.get("venkat_K", 5.0)
    p.mu_ref = cfg.get("mu_ref", 0.0)
    p.T_ref = cfg.get("T_ref", 300.0)
    p.Pr = cfg.get("Pr", 0.72)
    tgv = cfg.get("tgv", {})
    p.tgv_U0, p.tgv_P0 = tgv.get("U0", 40.0), tgv.get("P0", 100000.0)
    p.tgv_L, p.tgv_mu = tgv.get("L", 1.0), tgv.get("mu", 1.0e-2)
    p.start_time = cfg.get("start_time", 0.0)
    p.density_constrained = int(cfg.get("densityConstrained", 0))
    p.min_density = cfg.get("minDensityConstrained", 0.01)
    p.max_density = cfg.get("maxDensityConstrained", 10.0)
    p.flux = N.FLUX[cfg.get("flux", "ausm")]
    p.limiter = N.LIMITER[cfg.get("limiter", "minmod")]
    p.viscosity = N.VISC[cfg.get("viscosity", "none")]
    p.art_viscosity = int(cfg.get("art_viscosity", 0))
    p.init_nodes = int(cfg.get("init_nodes", 0))
    bcs = cfg.get("bc", [])
    if len(bcs) > N.GD2D_MAX_BC:
        raise ValueError("too many boundary kinds")
    p.n_bc = len(bcs)
    for i, b in enumerate(bcs):
        p.bc[i].tag, p.bc[i].kind = b["tag"], N.BC_KIND[b["kind"]]
        p.bc[i].rho, p.bc[i].u, p.bc[i].v, p.bc[i].p = (b.get("rho", 0.0), b.get("u", 0.0), b.get("v", 0.0),
                                                        b.get("p", 0.0))
        p.bc[i].Tw = b.get("Tw", 0.0)
    return p


def make_launch(precision="f64", order="hilbert", loop="tile", block=0, node_block=0, persistent=0,
                graph_steps=0, stream=None, min_blocks=0, device=0) -> N.Launch:
    l = N.Launch()
    l.device = int(device)
    l.precision = N.PRECISION[precision] if isinstance(precision, str) else int(precision)
    l.order = N.ORDER[order] if isinstance(order, str) else int(order)
    l.loop = N.LOOP[loop] if isinstance(loop, str) else int(loop)
    l.block, l.node_block, l.persistent, l.graph_steps = block, node_block, persistent, graph_steps
    l.min_blocks = min_blocks
    l.stream = stream
    return l


class Solver:
    """One gd2d handle: several independent cases advancing together."""

    def __init__(self, meshes: Sequence[Mesh2d], cfgs: Sequence[Dict], launch: Optional[N.Launch] = None):
        self.L = N.load()
        self.meshes = list(meshes)
        self.cfgs = [dict(c) for c in cfgs]
        n = len(self.meshes)
        self._views = (N.MeshView * n)(*[mesh_view(m) for m in self.meshes])
        self._params = (N.Params * n)(*[make_params(c) for c in self.cfgs])
        self._launch = launch if launch is not None else make_launch()
        self._t0 = [0.0] * n
        h = C.c_void_p()
        N.check(self.L.gd2d_setup(C.byref(h), n, self._views, self._params, C.byref(self._launch)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.gd2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ncases(self):
        return len(self.meshes)

    def _chk(self, code):
        return N.check(code, self.h)

    # -- initial / restart state -------------------------------------------
    def createFields2d(self, icase: int, rho, ux, uy, p):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, ux, uy, p)]
        for a in arrs:
            if a.shape != (self.meshes[icase].nCells,):
                raise ValueError("field size does not match the mesh")
        dp = C.POINTER(C.c_double)
        self._chk(self.L.gd2d_set_state(self.h, icase, *[a.ctypes.data_as(dp) for a in arrs]))
        self._t0[icase] = float(self.cfgs[icase].get("start_time", 0.0))

    set_state = createFields2d

    def set_conservative(self, icase: int, ucons, flow_time: float, rebuild_nodes: bool = True):
        u = np.asfortranarray(ucons, dtype=np.float64)
        self._chk(self.L.gd2d_set_conservative(self.h, icase, u.ctypes.data_as(C.POINTER(C.c_double)),
                                               float(flow_time), int(rebuild_nodes)))
        self._t0[icase] = float(flow_time)

    def flow_time(self, icase: int) -> float:
        """Current flowTime of a case: its start (set_state / restart) plus
        the dt of every step taken since."""
        h = self.history(icase, 1)
        return h[-1]["flowTime"] + h[-1]["dt"] if h else self._t0[icase]

    def save_snapshot(self, icase: int, path: str) -> None:
        """Solution snapshot of one case as a raw .npz (no VTK): the
        reference's solutionCellsT fields (flowTime, dt, densityCells,
        UxCells, UyCells, pressureCells; primeObjects.jl:197-205,
        evaluate2d.jl:187-203) plus the conservative state, which makes a
        restart continue bit for bit."""
        st = self.get_state(icase)
        h = self.history(icase, 1)
        P = st["prims"]
        np.savez(path, flowTime=self.flow_time(icase), dt=(h[-1]["dt"] if h else 0.0),
                 densityCells=P[:, 0], UxCells=P[:, 1], UyCells=P[:, 2], pressureCells=P[:, 3],
                 Ucons=st["Ucons"], nCells=self.meshes[icase].nCells)

    def load_snapshot(self, icase: int, path: str) -> float:
        """Restart a case from save_snapshot's file (loadPrevResults.jl:3-38
        reads the primitives; here the conservatives are restored exactly and
        the node values rebuilt from them).  Returns the restored flowTime."""
        d = np.load(path)
        if int(d["nCells"]) != self.meshes[icase].nCells:
            raise ValueError("snapshot does not match the case's mesh")
        t = float(d["flowTime"])
        self.set_conservative(icase, np.asfortranarray(d["Ucons"]), t, rebuild_nodes=True)
        return t

    # -- stepping ------------------------------------------------------------
    def propagate2d(self, nsteps: int) -> List[Dict]:
        st = (N.Stats * self.ncases)()
        self._chk(self.L.gd2d_propagate(self.h, int(nsteps), st))
        return [s.as_dict() for s in st]

    propagate = propagate2d

    def history(self, icase: int, capacity: int = 1 << 20) -> List[Dict]:
        buf = (N.Stats * capacity)()
        n = self._chk(self.L.gd2d_get_history(self.h, icase, buf, capacity))
        return [buf[i].as_dict() for i in range(n)]

    def get_state(self, icase: int) -> Dict[str, np.ndarray]:
        m = self.meshes[icase]
        U = np.zeros((m.nCells, 4), order="F")
        P = np.zeros((m.nCells, 4), order="F")
        Nd = np.zeros((m.nNodes, 4), order="F")
        dp = C.POINTER(C.c_double)
        self._chk(self.L.gd2d_get_state(self.h, icase, U.ctypes.data_as(dp), P.ctypes.data_as(dp),
                                        Nd.ctypes.data_as(dp)))
        return {"Ucons": U, "prims": P, "node_prims": Nd}

    def autotune(self, steps_per_trial: int = 64) -> dict:
        """Time candidate launch shapes on this handle's own state (which is
        saved and restored, so the run continues as if nothing happened) and
        keep the fastest: cell-kernel register budget and persistence,
        node-pass block, steps per CUDA graph.  Returns the chosen shape and
        its device ms per step."""
        ch = N.Launch()
        self._chk(self.L.gd2d_autotune(self.h, int(steps_per_trial), C.byref(ch)))
        t, _, _ = self.last_timing()
        return {"min_blocks": ch.min_blocks, "persistent": ch.persistent, "node_block": ch.node_block,
                "graph_steps": ch.graph_steps, "ms_per_step": t}

    def last_timing(self) -> Tuple[float, float, int]:
        t, c, n = C.c_double(), C.c_double(), C.c_int64()
        self._chk(self.L.gd2d_last_timing(self.h, C.byref(t), C.byref(c), C.byref(n)))
        return t.value, c.value, n.value

    # -- the reference's functions one at a time ---------------------------------
    def calcOneStageMUSCLcpuFast(self, icase: int, beta: float, dt: float, flow_time: float):
        m = self.meshes[icase]
        F = np.zeros((m.nCells, 4), order="F")
        Un = np.zeros((m.nCells, 4), order="F")
        dp = C.POINTER(C.c_double)
        self._chk(self.L.gd2d_calc_one_stage(self.h, icase, beta, dt, flow_time, F.ctypes.data_as(dp),
                                             Un.ctypes.data_as(dp)))
        return F, Un

    def updateVariablesSA(self, icase: int):
        m = self.meshes[icase]
        D = np.zeros((m.nCells, 4), order="F")
        self._chk(self.L.gd2d_update_variables(self.h, icase, D.ctypes.data_as(C.POINTER(C.c_double))))
        return D

    def cells2nodesSolutionReconstructionWithStencils(self):
        self._chk(self.L.gd2d_cells_to_nodes(self.h))

    def calcDiffTerm(self, icase: int):
        m = self.meshes[icase]
        D = np.zeros((m.nCells, 4), order="F")
        self._chk(self.L.gd2d_calc_diff_term(self.h, icase, D.ctypes.data_as(C.POINTER(C.c_double))))
        return D


def updateResidualSA(history: Sequence[Dict], convergence_criteria: Sequence[float]) -> Tuple[List[float], int]:
    """The reference's residual bookkeeping (updateResidualSA,
    evaluate2d.jl:1-41) over a case's step history, step 1 first.

    residualsVectorMax starts at ones and is the running max of the first
    curIter residuals while 1 < curIter < 6 (curIter = the 1-based step);
    the solution is converged at the first curIter > 5 where every
    residual divided by its max is <= its criterion.  Returns
    (residualsVectorMax, converged step or 0)."""
    rmax = [1.0, 1.0, 1.0, 1.0]
    crit = [float(c) for c in convergence_criteria]
    for it in range(1, len(history) + 1):
        if 1 < it < 6:
            rmax = [max(h["residual"][v] for h in history[:it]) for v in range(4)]
        if it > 5 and all(history[it - 1]["residual"][v] / rmax[v] <= crit[v] for v in range(4)):
            return rmax, it
    return rmax, 0


def propagate_until_converged(solver: "Solver", icase: int, max_steps: int, convergence_criteria: Sequence[float],
                              chunk: int = 256) -> int:
    """The reference's run loop (testInviscidFluxesGPUx32.jl:314-447): step
    until the residual criterion of updateResidualSA holds or max_steps
    steps have run, in chunks of `chunk` steps (one CUDA graph replay per
    32 steps; the convergence test runs on the host between chunks, so up
    to chunk-1 steps past convergence may run).  Returns the converged step
    (1-based, since the case's state was set) or 0."""
    done = 0
    while done < max_steps:
        n = min(chunk, max_steps - done)
        solver.propagate2d(n)
        done += n
        _, conv = updateResidualSA(solver.history(icase), convergence_criteria)
        if conv:
            return conv
    return 0


def autotune_layout(meshes: Sequence[Mesh2d], cfgs: Sequence[Dict], prims: Sequence[Sequence[np.ndarray]],
                    orders: Sequence[str] = ("hilbert", "rcm", "natural"), blocks: Sequence[int] = (256, 128),
                    steps: int = 64, **launch_kw) -> Tuple[Dict, List[Dict]]:
    """Pick the mesh ordering and the tile size (cells per block of the cell
    kernel) by timing them.  Both are fixed when a handle is set up (they
    decide the device layout and the tile face lists), so, unlike
    Solver.autotune, each candidate is a handle of its own: set up, given
    the cases' initial primitives `prims[i] = (rho, u, v, p)`, warmed up for
    one CUDA graph, timed over `steps` steps (device time, CUDA events) and
    destroyed before the next.  Returns the fastest candidate's make_launch
    keywords (ready for setupSolver / Solver, and for Solver.autotune to
    tune the rest on the chosen layout) and every trial's ms per step."""
    trials = []
    best = None
    for order in orders:
        for block in blocks:
            kw = dict(launch_kw, order=order, block=block)
            s = Solver(meshes, cfgs, make_launch(**kw))
            try:
                for i, p in enumerate(prims):
                    s.createFields2d(i, *p)
                s.propagate2d(max(32, launch_kw.get("graph_steps", 0) or 32))
                s.propagate2d(steps)
                total, cell, _ = s.last_timing()
            finally:
                s.close()
            rec = {"order": order, "block": block, "ms_per_step": total / steps, "cell_kernel_ms": cell}
            trials.append(rec)
            if best is None or rec["ms_per_step"] < best[1]:
                best = (kw, rec["ms_per_step"])
    return best[0], trials


def setupSolver(meshes, cfgs, **launch_kw) -> Solver:
    """setupSolver_*.jl + device setup for one or more cases."""
    if isinstance(meshes, Mesh2d):
        meshes, cfgs = [meshes], [cfgs]
    return Solver(meshes, cfgs, make_launch(**launch_kw))
