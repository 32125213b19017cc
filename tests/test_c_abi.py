"""The C ABI from plain C: tests/c_abi_demo.c runs setup -> set_state ->
propagate -> get_state through libgodunov2d with gcc, on a case whose mesh
and state this test writes into a generated header.  On the CPU the program
must compile and link against the header and the library; on a GPU its
result must equal the Python binding's bit for bit."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NSTEPS = 5


def _c_array(ctype, name, a):
    flat = np.asarray(a).ravel(order="F")
    if ctype == "double":
        body = ", ".join(repr(float(x)) for x in flat)
    else:
        body = ", ".join(str(int(x)) for x in flat)
    return f"static const {ctype} {name}[{max(len(flat), 1)}] = {{{body}}};\n"


def _write_header(pkg, path):
    mesh, cfg, prims = pkg.cases.square_inviscid(6)
    th = cfg["thermo"]
    inflow = [b for b in cfg["bc"] if b["kind"] == "inflow"][0]
    out = [f"#define N_CELLS {mesh.nCells}\n#define N_NODES {mesh.nNodes}\n#define N_NEIB {mesh.nNeibCells}\n",
           f"#define NSTEPS {NSTEPS}\n#define CASE_RGAS {th['RGAS']!r}\n#define CASE_GAMMA {th['Gamma']!r}\n",
           f"#define CASE_CFL {cfg['CFL']!r}\n#define IN_RHO {inflow['rho']!r}\n#define IN_U {inflow['u']!r}\n",
           f"#define IN_P {inflow['p']!r}\n"]
    for name in ("xNodes", "yNodes"):
        out.append(_c_array("double", "x_nodes" if name == "xNodes" else "y_nodes", getattr(mesh, name)))
    for name in ("mesh_connectivity", "cell_stiffness", "cells2nodes", "cell_clusters", "node2cellL2up",
                 "node2cellL2down"):
        out.append(_c_array("int32_t", name, getattr(mesh, name)))
    for name in ("cell_edges_Nx", "cell_edges_Ny", "cell_edges_length", "cell_areas", "HX", "cell_mid_points",
                 "node_stencils"):
        out.append(_c_array("double", name, getattr(mesh, name)))
    for name, a in zip(("rho0", "ux0", "uy0", "p0"), prims):
        out.append(_c_array("double", name, a))
    with open(path, "w") as f:
        f.write("".join(out))
    assert cfg["flux"] == "ausm" and cfg["limiter"] == "minmod" and cfg["viscosity"] == "none"
    return mesh, cfg, prims


def _build(pkg, tmp_path):
    _write_header(pkg, tmp_path / "case_data.h")
    libdir = os.path.dirname(pkg._native.LIB_PATH)
    exe = tmp_path / "c_abi_demo"
    subprocess.run(["gcc", "-O2", "-std=c11", "-I", os.path.join(ROOT, "include"), "-I", str(tmp_path),
                    os.path.join(ROOT, "tests", "c_abi_demo.c"), "-o", str(exe), "-L", libdir, "-lgodunov2d",
                    f"-Wl,-rpath,{libdir}"], check=True, capture_output=True, text=True)
    return exe


def test_c_caller_compiles_and_links(pkg, tmp_path):
    exe = _build(pkg, tmp_path)
    assert exe.exists()


@pytest.mark.gpu
def test_c_caller_matches_python_binding(pkg, tmp_path):
    exe = _build(pkg, tmp_path)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.split("\n")
    mesh, cfg, prims = pkg.cases.square_inviscid(6)
    n = mesh.nCells
    got = np.array([float(x) for x in lines[:4 * n]]).reshape((n, 4), order="F")
    s = pkg.setupSolver(mesh, cfg)
    s.createFields2d(0, *prims)
    st = s.propagate2d(NSTEPS)[0]
    ref = s.get_state(0)["Ucons"]
    s.close()
    assert np.array_equal(got, ref)
    tail = lines[4 * n].split()
    assert int(tail[1]) == NSTEPS and float(tail[3]) == st["dt"]
