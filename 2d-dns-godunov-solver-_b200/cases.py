"""Case definitions: mesh + parameters + initial state for the benchmark and
test workloads.

A case configuration is a plain dict shared by the CUDA solver and the CPU
oracle (same keys, same meaning):

  thermo      {"RGAS", "Gamma", "Cp", "mu", "kGas"} (THERMOPHYSICS, thermo.jl:4-10)
  flux        "ausm" | "roe" | "ausm_m2020"
  limiter     "minmod" | "venkat" | "vanleer" | "vanalbada" | "none"
  viscosity   "none" | "reference" | "sutherland" | "constant"
  art_viscosity 0/1, mu_ref, T_ref, Pr, venkat_K, ksi
  dt_mode     0 fixed ``dt`` (the reference's solControls.dt, testInviscidFluxesGPUx32.jl:301;
              the default) | 1 step with the CFL-based ``tau`` the reference only
              reports (testInviscidFluxesGPUx32.jl:299,324) | 2 local CFL (extension)
  CFL, dt, beta
  init_nodes  0 reference behaviour (node primitives zero in step 1) | 1
  bc          list of {"tag", "kind", rho/u/v/p, Tw}
  tgv         {"U0", "P0", "L", "mu"} for the analytic Taylor-Green ghost state

The reference's own drivers hard-code these as globals in
setupSolver_*.jl (e.g. setupSolver_step2d.jl:5-68).
"""
from __future__ import annotations

import math
from typing import Dict, List, Tuple

import numpy as np

from . import mesh as meshmod

AIR = {"RGAS": 287.058, "Gamma": 1.4, "Cp": 1000.0, "mu": 0.0, "kGas": 0.0}


def square_inviscid(n_nodes: int = 101, seed: int = 1, flux: str = "ausm", limiter: str = "minmod"):
    """Plain FP64 inviscid step on the jittered unit square.

    Mach 2 along +x with rho=1, p=1/gamma (a=1), a Gaussian density bump
    (amplitude 0.2, sigma 0.05 at (0.3,0.5)) and 1% seeded noise on rho;
    left supersonic inflow, right outflow, slip walls top and bottom;
    AUSM+ / MUSCL / Minmod, CFL 0.5."""
    mesh = meshmod.unit_square_mesh(n_nodes, jitter=0.1, seed=seed)
    g = AIR["Gamma"]
    cfg = {"thermo": dict(AIR), "flux": flux, "limiter": limiter, "viscosity": "none", "dt_mode": 2,
           "CFL": 0.5, "beta": 1.0, "ksi": 1.0e-12, "init_nodes": 0,
           "bc": [{"tag": -1, "kind": "inflow", "rho": 1.0, "u": 2.0, "v": 0.0, "p": 1.0 / g},
                  {"tag": -2, "kind": "outflow"}, {"tag": -3, "kind": "slip"}]}
    xc, yc = mesh.cell_mid_points[:, 0], mesh.cell_mid_points[:, 1]
    rng = np.random.default_rng(seed + 1000)
    rho = 1.0 + 0.2 * np.exp(-((xc - 0.3) ** 2 + (yc - 0.5) ** 2) / (2.0 * 0.05 ** 2))
    rho = rho * (1.0 + rng.uniform(-0.01, 0.01, size=rho.shape))
    prims = (rho, np.full_like(rho, 2.0), np.zeros_like(rho), np.full_like(rho, 1.0 / g))
    return mesh, cfg, prims


# Freestream of the reference's supersonic-cylinder inlet
# (boundaryConditions2d.jl:36-39): rho=1.1766, u=1232.6445, p=101325 -> T~300 K, M~3.55.
CYL_RHO, CYL_P = 1.1766, 101325.0


def cylinder_case(n_nodes: int = 1025, mach: float = 3.5, re_d: float = 1.0e4, radius: float = 0.5,
                  flux: str = "ausm", limiter: str = "venkat", viscous: bool = True, art_viscosity: bool = True,
                  cfl: float = 0.4):
    """Viscous supersonic cylinder: [-5,15]x[-8,8], cells with centroid
    inside r<radius removed, no-slip isothermal staircase wall (Tw = T_inf);
    Sutherland viscosity scaled to mu_inf = rho U D / Re_D, Pr = 0.72,
    artificial viscosity, Venkatakrishnan limiter, CFL 0.4."""
    mesh = meshmod.cylinder_mesh(n_nodes, radius=radius)
    th = dict(AIR)
    g, R = th["Gamma"], th["RGAS"]
    T_inf = CYL_P / (CYL_RHO * R)
    a_inf = math.sqrt(g * CYL_P / CYL_RHO)
    u_inf = mach * a_inf
    D = 2.0 * radius
    mu_inf = CYL_RHO * u_inf * D / re_d
    cfg = {"thermo": th, "flux": flux, "limiter": limiter,
           "viscosity": "sutherland" if viscous else "none", "art_viscosity": int(art_viscosity and viscous),
           "mu_ref": mu_inf, "T_ref": T_inf, "Pr": 0.72, "venkat_K": 5.0, "dt_mode": 2, "CFL": cfl,
           "beta": 1.0, "ksi": 1.0e-12, "init_nodes": 0,
           # the reference's density constraint with its default bounds
           # (setupSolver_step2d.jl:167-169): the base region behind the
           # cylinder expands towards vacuum after the impulsive start
           "densityConstrained": 1, "minDensityConstrained": 0.01, "maxDensityConstrained": 10.0,
           "bc": [{"tag": -1, "kind": "inflow", "rho": CYL_RHO, "u": u_inf, "v": 0.0, "p": CYL_P},
                  {"tag": -2, "kind": "outflow"},
                  {"tag": -4, "kind": "noslip_isothermal", "Tw": T_inf}],
           "case_info": {"mach": mach, "re_d": re_d, "radius": radius, "nodes_per_side": n_nodes}}
    nc = mesh.nCells
    prims = (np.full(nc, CYL_RHO), np.full(nc, u_inf), np.zeros(nc), np.full(nc, CYL_P))
    return mesh, cfg, prims


def tgv_case(n_nodes: int, mach: float, re: float, flux: str = "ausm", limiter: str = "minmod", cfl: float = 0.4):
    """Periodic Taylor-Green vortex on [0,2pi]^2: rho0=1, p0=1/gamma (a0=1),
    U0=Mach, u=U0 sin x cos y, v=-U0 cos x sin y,
    p=p0+rho0 U0^2/4 (cos 2x + cos 2y); constant mu = rho0 U0 L / Re, L=1."""
    mesh = meshmod.periodic_square_mesh(n_nodes)
    th = dict(AIR)
    g = th["Gamma"]
    U0 = mach
    p0 = 1.0 / g
    mu = 1.0 * U0 * 1.0 / re
    cfg = {"thermo": th, "flux": flux, "limiter": limiter, "viscosity": "constant", "art_viscosity": 0,
           "mu_ref": mu, "T_ref": 1.0, "Pr": 0.72, "dt_mode": 2, "CFL": cfl, "beta": 1.0, "ksi": 1.0e-12,
           "init_nodes": 0, "bc": [], "case_info": {"mach": mach, "re": re, "nodes_per_side": n_nodes}}
    x, y = mesh.cell_mid_points[:, 0], mesh.cell_mid_points[:, 1]
    u = U0 * np.sin(x) * np.cos(y)
    v = -U0 * np.cos(x) * np.sin(y)
    p = p0 + 1.0 * U0 * U0 / 4.0 * (np.cos(2 * x) + np.cos(2 * y))
    prims = (np.ones_like(x), u, v, p)
    return mesh, cfg, prims


def reference_tgv_case(n_nodes: int = 101, quads: bool = False):
    """The reference's own compressible TGV test (testViscousFluxesTGV2d.jl,
    setupSolver_TGV2d.jl): [0,2pi]^2 box, analytic TGV ghost state on every
    boundary face (boundaryConditions_TGV2d.jl:16-30), U=40, P=1e5, rho=1,
    constant mu=1e-2 with the reference's Laplacian viscous term
    (calcDiffTerm.jl), fixed dt = 1e-7."""
    tag = -5
    mesh = meshmod.structured_mesh(n_nodes, n_nodes, 0.0, 2.0 * math.pi, 0.0, 2.0 * math.pi, quads=quads,
                                   tags={"left": tag, "right": tag, "bottom": tag, "top": tag})
    th = dict(AIR)
    cfg = {"thermo": th, "flux": "ausm", "limiter": "minmod", "viscosity": "reference", "art_viscosity": 0,
           "mu_ref": 1.0e-2, "dt_mode": 0, "dt": 1.0e-7, "CFL": 0.1, "beta": 1.0, "ksi": 1.0e-12, "init_nodes": 0,
           "tgv": {"U0": 40.0, "P0": 100000.0, "L": 1.0, "mu": 1.0e-2},
           "bc": [{"tag": tag, "kind": "tgv"}]}
    x, y = mesh.cell_mid_points[:, 0], mesh.cell_mid_points[:, 1]
    P, U, R = 100000.0, 40.0, th["RGAS"]
    T = P / R
    rho = np.full_like(x, P / R / T)
    u = U * np.sin(x) * np.cos(y)
    v = -U * np.cos(x) * np.sin(y)
    p = P + 0.25 * U * U * (np.cos(2 * x) + np.cos(2 * y))
    return mesh, cfg, (rho, u, v, p)


def shard_cases(sizes, world: int, rank: int) -> List[int]:
    """Indices of the independent cases rank `rank` of `world` advances:
    greedy longest-processing-time assignment by cell count (largest case to
    the least-loaded rank, ties to the lower rank), so every rank gets a
    deterministic, nearly equal share with no data exchange between ranks."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad world/rank")
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * world
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += sizes[i]
    return [i for i in range(len(sizes)) if owner[i] == rank]


def batched_tgv(n_cases: int = 64, seed: int = 4, n_min: int = 64, n_max: int = 512) -> List[Tuple]:
    """Seeded TGV batch: nodes per side U{n_min..n_max}, Mach U(0.1,0.5), Re U(100,1600)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_cases):
        n = int(rng.integers(n_min, n_max + 1))
        out.append(tgv_case(n, float(rng.uniform(0.1, 0.5)), float(rng.uniform(100.0, 1600.0))))
    return out


def batched_cylinders(n_cases: int = 16, seed: int = 5, n_min: int = 257, n_max: int = 1025) -> List[Tuple]:
    """Seeded cylinder sweep: nodes per side U{n_min..n_max}, Mach U(2,4),
    Re_D U(2e3,2e4), radius U(0.3,0.7)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_cases):
        n = int(rng.integers(n_min, n_max + 1))
        out.append(cylinder_case(n, mach=float(rng.uniform(2.0, 4.0)), re_d=float(rng.uniform(2.0e3, 2.0e4)),
                                 radius=float(rng.uniform(0.3, 0.7))))
    return out
