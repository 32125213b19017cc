"""ctypes wrapper of the CPU oracle (godunov2d_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline arm of bench.py to check the CUDA path.  The product path never imports
this module.  Parity of the oracle itself is unpinned by reference-produced
vectors (the reference is Julia and records none); see the C file header.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
SRC = os.path.join(HERE, "godunov2d_oracle.c")

FLUX = {"ausm": 1, "roe": 2, "ausm_m2020": 3}
LIMITER = {"none": 0, "minmod": 1, "venkat": 2, "vanleer": 3, "vanalbada": 4}
BC_KIND = {"inflow": 1, "outflow": 2, "slip": 3, "noslip_isothermal": 4, "tgv": 5}
VISC = {"none": 0, "reference": 1, "sutherland": 2, "constant": 3}


def build(force: bool = False) -> str:
    """Compile the oracle with the recipe of oracle/Makefile."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(SRC):
        os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB_PATH


class OrcMesh(C.Structure):
    _fields_ = [("nCells", C.c_int64), ("nNodes", C.c_int64), ("nNeibCells", C.c_int32), ("pad_", C.c_int32),
                ("xNodes", C.c_void_p), ("yNodes", C.c_void_p), ("mesh_connectivity", C.c_void_p),
                ("cell_stiffness", C.c_void_p), ("cells2nodes", C.c_void_p), ("cell_edges_Nx", C.c_void_p),
                ("cell_edges_Ny", C.c_void_p), ("cell_edges_length", C.c_void_p), ("cell_areas", C.c_void_p),
                ("HX", C.c_void_p), ("cell_mid_points", C.c_void_p), ("cell_clusters", C.c_void_p),
                ("node_stencils", C.c_void_p), ("node2cellL2up", C.c_void_p), ("node2cellL2down", C.c_void_p)]


class OrcBC(C.Structure):
    _fields_ = [("tag", C.c_int32), ("kind", C.c_int32), ("rho", C.c_double), ("u", C.c_double),
                ("v", C.c_double), ("p", C.c_double), ("Tw", C.c_double)]


class OrcParams(C.Structure):
    _fields_ = [("RGAS", C.c_double), ("Gamma", C.c_double), ("Cp", C.c_double), ("mu", C.c_double),
                ("kGas", C.c_double), ("CFL", C.c_double), ("dt", C.c_double), ("beta", C.c_double),
                ("ksi", C.c_double), ("venkat_K", C.c_double), ("mu_ref", C.c_double), ("T_ref", C.c_double),
                ("Pr", C.c_double), ("tgv_U0", C.c_double), ("tgv_P0", C.c_double), ("tgv_L", C.c_double),
                ("tgv_mu", C.c_double), ("minDensityConstrained", C.c_double),
                ("maxDensityConstrained", C.c_double), ("flux", C.c_int32), ("limiter", C.c_int32),
                ("viscosity", C.c_int32), ("art_viscosity", C.c_int32), ("dt_mode", C.c_int32),
                ("init_nodes", C.c_int32), ("nthreads", C.c_int32), ("n_bc", C.c_int32),
                ("densityConstrained", C.c_int32), ("pad2_", C.c_int32), ("bc", OrcBC * 8)]


class OrcStats(C.Structure):
    _fields_ = [("dt", C.c_double), ("flowTime", C.c_double), ("tau", C.c_double), ("velmax", C.c_double),
                ("residual", C.c_double * 4), ("rhoMin", C.c_double), ("rhoMax", C.c_double),
                ("totals", C.c_double * 4), ("Ek", C.c_double), ("step", C.c_int64), ("nonfinite", C.c_int32),
                ("pad_", C.c_int32)]

    def as_dict(self):
        return {"dt": self.dt, "flowTime": self.flowTime, "tau": self.tau, "velmax": self.velmax,
                "residual": list(self.residual), "rhoMin": self.rhoMin, "rhoMax": self.rhoMax,
                "totals": list(self.totals), "Ek": self.Ek, "step": self.step, "nonfinite": self.nonfinite}


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcParams)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_init_fields.argtypes = [C.c_void_p, dp, dp, dp, dp]
        L.orc_step.argtypes = [C.c_void_p, C.POINTER(OrcStats)]
        L.orc_run.argtypes = [C.c_void_p, C.c_int32, C.POINTER(OrcStats)]
        L.orc_calc_one_stage.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.orc_update_variables.argtypes = [C.c_void_p, C.POINTER(OrcStats)]
        L.orc_cells2nodes.argtypes = [C.c_void_p]
        L.orc_calc_diff_term.argtypes = [C.c_void_p]
        L.orc_green_gauss_gradient.argtypes = [C.c_void_p, dp, dp, dp]
        L.orc_field.restype = dp
        L.orc_field.argtypes = [C.c_void_p, C.c_int32]
        L.orc_flow_time.restype = C.c_double
        L.orc_flow_time.argtypes = [C.c_void_p]
        L.orc_max_edge.restype = C.c_double
        L.orc_max_edge.argtypes = [C.c_void_p]
        L.orc_set_time.argtypes = [C.c_void_p, C.c_double]
        for nm in ("orc_minmod", "orc_vanleer", "orc_vanalbada", "orc_venkat"):
            getattr(L, nm).restype = C.c_double
            getattr(L, nm).argtypes = [C.c_double, C.c_double, C.c_double]
        L.orc_flux.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, C.c_double, C.c_double, dp]
        L.orc_air_conductivity.restype = C.c_double
        L.orc_air_conductivity.argtypes = [C.c_double]
        L.orc_sutherland.restype = C.c_double
        L.orc_sutherland.argtypes = [C.c_double]
        L.orc_partition.argtypes = [C.c_int32, C.c_int64, C.POINTER(C.c_int32)]
        for nm in ("orc_sizeof_params", "orc_sizeof_mesh", "orc_sizeof_stats"):
            getattr(L, nm).restype = C.c_int32
        assert L.orc_sizeof_params() == C.sizeof(OrcParams)
        assert L.orc_sizeof_mesh() == C.sizeof(OrcMesh)
        assert L.orc_sizeof_stats() == C.sizeof(OrcStats)
        _lib = L
    return _lib


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def flux(kind: str, uL, uR, nx, ny, side, gamma):
    out = np.zeros(4)
    a = np.ascontiguousarray(uL, dtype=np.float64)
    b = np.ascontiguousarray(uR, dtype=np.float64)
    lib().orc_flux(FLUX[kind], _dptr(a), _dptr(b), nx, ny, side, gamma, _dptr(out))
    return out


def partition(nthreads: int, n: int) -> np.ndarray:
    r = np.zeros((max(nthreads, 1), 2), dtype=np.int32)
    lib().orc_partition(nthreads, n, r.ctypes.data_as(C.POINTER(C.c_int32)))
    return r


def make_params(cfg) -> OrcParams:
    """OrcParams from the plain-dict case configuration shared with the product."""
    p = OrcParams()
    th = cfg["thermo"]
    p.RGAS, p.Gamma, p.Cp, p.mu, p.kGas = th["RGAS"], th["Gamma"], th.get("Cp", 1000.0), th.get("mu", 0.0), th.get("kGas", 0.0)
    p.CFL = cfg.get("CFL", 0.5)
    p.dt = cfg.get("dt", 0.0)
    p.beta = cfg.get("beta", 1.0)
    p.ksi = cfg.get("ksi", 1.0e-12)
    p.venkat_K = cfg.get("venkat_K", 5.0)
    p.mu_ref = cfg.get("mu_ref", 0.0)
    p.T_ref = cfg.get("T_ref", 300.0)
    p.Pr = cfg.get("Pr", 0.72)
    tgv = cfg.get("tgv", {})
    p.tgv_U0, p.tgv_P0, p.tgv_L, p.tgv_mu = (tgv.get("U0", 40.0), tgv.get("P0", 100000.0), tgv.get("L", 1.0),
                                              tgv.get("mu", 1.0e-2))
    p.densityConstrained = int(cfg.get("densityConstrained", 0))
    p.minDensityConstrained = cfg.get("minDensityConstrained", 0.01)
    p.maxDensityConstrained = cfg.get("maxDensityConstrained", 10.0)
    p.flux = FLUX[cfg.get("flux", "ausm")]
    p.limiter = LIMITER[cfg.get("limiter", "minmod")]
    p.viscosity = VISC[cfg.get("viscosity", "none")]
    p.art_viscosity = int(cfg.get("art_viscosity", 0))
    p.dt_mode = int(cfg.get("dt_mode", 0))
    p.init_nodes = int(cfg.get("init_nodes", 0))
    p.nthreads = int(cfg.get("nthreads", os.cpu_count() or 1))
    bcs = cfg.get("bc", [])
    p.n_bc = len(bcs)
    for i, b in enumerate(bcs):
        p.bc[i].tag = b["tag"]
        p.bc[i].kind = BC_KIND[b["kind"]]
        p.bc[i].rho, p.bc[i].u, p.bc[i].v, p.bc[i].p = b.get("rho", 0.0), b.get("u", 0.0), b.get("v", 0.0), b.get("p", 0.0)
        p.bc[i].Tw = b.get("Tw", 0.0)
    return p


class Oracle:
    """One reference-ordered FP64 solver state on the CPU."""

    FIELD = {"rho": 0, "ux": 1, "uy": 2, "p": 3, "a": 4, "vmax": 5, "rhoN": 6, "uxN": 7, "uyN": 8, "pN": 9,
             "Uold": 10, "Unew": 11, "UN": 12, "Diff": 13, "Delta": 14, "FLUXES": 15, "muArt": 16}

    def __init__(self, mesh, cfg, nthreads=None):
        L = lib()
        self.mesh = mesh
        self.cfg = dict(cfg)
        if nthreads is not None:
            self.cfg["nthreads"] = nthreads
        m = OrcMesh()
        m.nCells, m.nNodes, m.nNeibCells = mesh.nCells, mesh.nNodes, mesh.nNeibCells
        for name in ("xNodes", "yNodes", "mesh_connectivity", "cell_stiffness", "cells2nodes", "cell_edges_Nx",
                     "cell_edges_Ny", "cell_edges_length", "cell_areas", "HX", "cell_mid_points", "cell_clusters",
                     "node_stencils", "node2cellL2up", "node2cellL2down"):
            setattr(m, name, getattr(mesh, name).ctypes.data)
        self._m = m
        self._p = make_params(self.cfg)
        self.h = L.orc_create(C.byref(self._m), C.byref(self._p))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_destroy(h)
            self.h = None

    def init_fields(self, rho, ux, uy, p):
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (rho, ux, uy, p)]
        lib().orc_init_fields(self.h, *[_dptr(a) for a in arrs])

    def step(self):
        st = OrcStats()
        lib().orc_step(self.h, C.byref(st))
        return st.as_dict()

    def run(self, nsteps):
        hist = []
        for _ in range(nsteps):
            hist.append(self.step())
        return hist

    def calc_one_stage(self, beta, dt, t):
        lib().orc_calc_one_stage(self.h, beta, dt, t)

    def update_variables(self):
        st = OrcStats()
        lib().orc_update_variables(self.h, C.byref(st))
        return st.as_dict()

    def cells2nodes(self):
        lib().orc_cells2nodes(self.h)

    def calc_diff_term(self):
        lib().orc_calc_diff_term(self.h)

    def green_gauss_gradient(self, field):
        """calcScalarFieldGreenGaussNodesBasedGradient (calcGradients.jl:36-139)
        of a cell field: (gradX, gradY), gradX paired with -ny as in the
        reference, so gradX approximates d/dy and gradY d/dx for the mesh's
        inward unit normals."""
        f = np.ascontiguousarray(field, dtype=np.float64)
        if f.shape != (self.mesh.nCells,):
            raise ValueError("field size does not match the mesh")
        gx = np.zeros_like(f)
        gy = np.zeros_like(f)
        lib().orc_green_gauss_gradient(self.h, _dptr(f), _dptr(gx), _dptr(gy))
        return gx, gy

    def field(self, name):
        n = self.mesh.nNodes if name in ("rhoN", "uxN", "uyN", "pN", "UN") else self.mesh.nCells
        width = 4 if name in ("Uold", "Unew", "UN", "Diff", "Delta", "FLUXES") else 1
        ptr = lib().orc_field(self.h, self.FIELD[name])
        a = np.ctypeslib.as_array(ptr, shape=(n * width,)).copy()
        return a.reshape((n, 4), order="F") if width == 4 else a

    def prims(self):
        return np.stack([self.field(k) for k in ("rho", "ux", "uy", "p")], axis=1)

    def node_prims(self):
        return np.stack([self.field(k) for k in ("rhoN", "uxN", "uyN", "pN")], axis=1)

    @property
    def flow_time(self):
        return lib().orc_flow_time(self.h)

    def set_time(self, t):
        lib().orc_set_time(self.h, t)
