"""ctypes binding of include/godunov2d.h (libgodunov2d.so).

The structures below mirror the C declarations field for field; the
library checks nothing about Python, so any change to the header must be
reflected here (tests/test_abi.py compares the exported symbol list and
struct sizes against the header).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgodunov2d.so")

GD2D_MAX_BC = 8
STATUS = {0: "OK", -1: "ERR_ARG", -2: "ERR_MESH", -3: "ERR_CUDA", -4: "ERR_NONFINITE", -5: "ERR_TIMEOUT",
          -6: "ERR_OOM", -7: "ERR_STATE"}
FLUX = {"ausm": 1, "roe": 2, "ausm_m2020": 3}
LIMITER = {"none": 0, "minmod": 1, "venkat": 2, "vanleer": 3, "vanalbada": 4}
BC_KIND = {"inflow": 1, "outflow": 2, "slip": 3, "noslip_isothermal": 4, "tgv": 5}
VISC = {"none": 0, "reference": 1, "sutherland": 2, "constant": 3}
PRECISION = {"f64": 0, "mixed": 1}
ORDER = {"natural": 0, "hilbert": 1, "rcm": 2}
LOOP = {"cell": 0, "coloured": 1, "face": 2, "tile": 3}

EXPORTS = ("gd2d_abi_version", "gd2d_last_error", "gd2d_setup", "gd2d_set_state", "gd2d_set_conservative",
           "gd2d_propagate", "gd2d_get_history", "gd2d_get_state", "gd2d_calc_one_stage", "gd2d_update_variables",
           "gd2d_cells_to_nodes", "gd2d_calc_diff_term", "gd2d_autotune", "gd2d_last_timing", "gd2d_destroy",
           "gd2d_update_variables_noalloc")


class MeshView(C.Structure):
    _fields_ = [("n_cells", C.c_int64), ("n_nodes", C.c_int64), ("n_neib_cells", C.c_int32),
                ("reserved0", C.c_int32), ("x_nodes", C.c_void_p), ("y_nodes", C.c_void_p),
                ("mesh_connectivity", C.c_void_p), ("cell_stiffness", C.c_void_p), ("cells2nodes", C.c_void_p),
                ("cell_edges_Nx", C.c_void_p), ("cell_edges_Ny", C.c_void_p), ("cell_edges_length", C.c_void_p),
                ("cell_areas", C.c_void_p), ("HX", C.c_void_p), ("cell_mid_points", C.c_void_p),
                ("cell_clusters", C.c_void_p), ("node_stencils", C.c_void_p), ("node2cellL2up", C.c_void_p),
                ("node2cellL2down", C.c_void_p)]


class BC(C.Structure):
    _fields_ = [("tag", C.c_int32), ("kind", C.c_int32), ("rho", C.c_double), ("u", C.c_double),
                ("v", C.c_double), ("p", C.c_double), ("Tw", C.c_double)]


class Params(C.Structure):
    _fields_ = [("RGAS", C.c_double), ("Gamma", C.c_double), ("Cp", C.c_double), ("mu", C.c_double),
                ("kGas", C.c_double), ("CFL", C.c_double), ("dt", C.c_double), ("beta", C.c_double),
                ("ksi", C.c_double), ("venkat_K", C.c_double), ("mu_ref", C.c_double), ("T_ref", C.c_double),
                ("Pr", C.c_double), ("tgv_U0", C.c_double), ("tgv_P0", C.c_double), ("tgv_L", C.c_double),
                ("tgv_mu", C.c_double), ("start_time", C.c_double), ("min_density", C.c_double),
                ("max_density", C.c_double), ("flux", C.c_int32), ("limiter", C.c_int32),
                ("viscosity", C.c_int32), ("art_viscosity", C.c_int32), ("dt_mode", C.c_int32),
                ("init_nodes", C.c_int32), ("n_bc", C.c_int32), ("density_constrained", C.c_int32),
                ("bc", BC * GD2D_MAX_BC)]


class Launch(C.Structure):
    _fields_ = [("precision", C.c_int32), ("order", C.c_int32), ("loop", C.c_int32), ("block", C.c_int32),
                ("node_block", C.c_int32), ("persistent", C.c_int32), ("graph_steps", C.c_int32),
                ("min_blocks", C.c_int32), ("device", C.c_int32), ("reserved0", C.c_int32), ("stream", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("dt", C.c_double), ("flow_time", C.c_double), ("tau", C.c_double), ("velmax", C.c_double),
                ("residual", C.c_double * 4), ("rho_min", C.c_double), ("rho_max", C.c_double),
                ("totals", C.c_double * 4), ("kinetic_energy", C.c_double), ("step", C.c_int64),
                ("nonfinite", C.c_int32), ("reserved0", C.c_int32)]

    def as_dict(self):
        return {"dt": self.dt, "flowTime": self.flow_time, "tau": self.tau, "velmax": self.velmax,
                "residual": list(self.residual), "rhoMin": self.rho_min, "rhoMax": self.rho_max,
                "totals": list(self.totals), "Ek": self.kinetic_energy, "step": self.step,
                "nonfinite": self.nonfinite}


class NativeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load(path: str = LIB_PATH):
    """Load libgodunov2d.so; raises if it is missing (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"libgodunov2d.so not built at {path}; run __graft_entry__.build()")
    L = C.CDLL(path)
    vp, i32, i64, dp = C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_double)
    L.gd2d_abi_version.restype = C.c_int
    L.gd2d_last_error.restype = C.c_char_p
    L.gd2d_last_error.argtypes = [vp]
    L.gd2d_setup.argtypes = [C.POINTER(vp), i32, C.POINTER(MeshView), C.POINTER(Params), C.POINTER(Launch)]
    L.gd2d_set_state.argtypes = [vp, i32, dp, dp, dp, dp]
    L.gd2d_set_conservative.argtypes = [vp, i32, dp, C.c_double, i32]
    L.gd2d_propagate.argtypes = [vp, i32, C.POINTER(Stats)]
    L.gd2d_get_history.argtypes = [vp, i32, C.POINTER(Stats), i32]
    L.gd2d_get_state.argtypes = [vp, i32, dp, dp, dp]
    L.gd2d_calc_one_stage.argtypes = [vp, i32, C.c_double, C.c_double, C.c_double, dp, dp]
    L.gd2d_update_variables.argtypes = [vp, i32, dp]
    L.gd2d_cells_to_nodes.argtypes = [vp]
    L.gd2d_calc_diff_term.argtypes = [vp, i32, dp]
    L.gd2d_autotune.argtypes = [vp, i32, C.POINTER(Launch)]
    L.gd2d_last_timing.argtypes = [vp, dp, dp, C.POINTER(i64)]
    L.gd2d_destroy.argtypes = [vp]
    L.gd2d_update_variables_noalloc.argtypes = [vp, vp, vp, i64, C.c_double, vp, vp]
    for name in EXPORTS:
        if name not in ("gd2d_last_error",):
            getattr(L, name).restype = C.c_int
    if L.gd2d_abi_version() != 1:
        raise OSError("ABI version mismatch")
    _lib = L
    return L


def check(code: int, handle=None):
    if code < 0:
        msg = load().gd2d_last_error(handle)
        raise NativeError(code, msg.decode() if msg else "")
    return code
