"""CPU checks of the C ABI: the library loads, exports every entry point
declared in include/godunov2d.h, its structs have the header's layout, and
argument/mesh validation answers with error codes before any device work."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "godunov2d.h")


def header_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char \*)\s*(gd2d_\w+)\s*\(", src, flags=re.M)))


def test_header_exports_match(native, pkg):
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(native, n), n
    assert sorted(pkg._native.EXPORTS) == names
    out = subprocess.run(["nm", "-D", "--defined-only", native._name], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (gd2d_\w+)", out))
    assert set(names) <= exported


def test_struct_layout_matches_header(pkg, tmp_path):
    probe = tmp_path / "probe.c"
    probe.write_text('#include "godunov2d.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                     "int main(void){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(gd2d_mesh_view),"
                     " sizeof(gd2d_params), sizeof(gd2d_launch), sizeof(gd2d_stats), sizeof(gd2d_bc),"
                     " offsetof(gd2d_params, bc));return 0;}\n")
    exe = tmp_path / "probe"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(probe), "-o", str(exe)])
    sizes = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    N = pkg._native
    assert sizes == [C.sizeof(N.MeshView), C.sizeof(N.Params), C.sizeof(N.Launch), C.sizeof(N.Stats),
                     C.sizeof(N.BC), N.Params.bc.offset]


def _setup(native, pkg, mesh, cfg, ncases=1, launch=None):
    N = pkg._native
    views = (N.MeshView * ncases)(*[pkg.solver.mesh_view(mesh)] * ncases)
    params = (N.Params * ncases)(*[pkg.solver.make_params(cfg)] * ncases)
    h = C.c_void_p()
    rc = native.gd2d_setup(C.byref(h), ncases, views, params, C.byref(launch) if launch is not None else None)
    return rc, native.gd2d_last_error(None).decode()


def test_validation_errors_before_device_work(native, pkg):
    mesh, cfg, _ = pkg.cases.square_inviscid(9)
    h = C.c_void_p()
    assert native.gd2d_setup(C.byref(h), 0, None, None, None) == -1
    # a boundary tag without an entry in the table
    bad = dict(cfg, bc=[b for b in cfg["bc"] if b["tag"] != -3])
    rc, msg = _setup(native, pkg, mesh, bad)
    assert rc == -2 and "tag -3" in msg
    # neighbour index out of range
    m2 = pkg.mesh.Mesh2d.from_arrays({k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v)
                                      for k, v in mesh.arrays().items()})
    m2.cell_stiffness[3, 0] = mesh.nCells + 5
    rc, msg = _setup(native, pkg, m2, cfg)
    assert rc == -2 and "out of range" in msg
    # zero area
    m3 = pkg.mesh.Mesh2d.from_arrays({k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v)
                                      for k, v in mesh.arrays().items()})
    m3.cell_areas[7] = 0.0
    rc, msg = _setup(native, pkg, m3, cfg)
    assert rc == -2 and "area" in msg
    # inconsistent flux across cases of one handle
    rc, msg = _setup(native, pkg, mesh, dict(cfg, CFL=-1.0))
    assert rc == -1
    assert native.gd2d_propagate(None, 1, None) == -1
    assert native.gd2d_autotune(None, 8, None) == -1
    assert native.gd2d_destroy(None) == 0


@pytest.mark.parametrize("shape,text", [({"block": 64}, "block"), ({"node_block": 512}, "node_block"),
                                        ({"min_blocks": 5}, "min_blocks"), ({"precision": 7}, "precision")])
def test_launch_shape_validation(native, pkg, shape, text):
    mesh, cfg, _ = pkg.cases.square_inviscid(9)
    rc, msg = _setup(native, pkg, mesh, cfg, launch=pkg.solver.make_launch(**shape))
    assert rc == -1 and text in msg, (rc, msg)


def test_missing_library_fails_loudly(pkg, tmp_path):
    with pytest.raises(OSError):
        pkg._native.load(str(tmp_path / "nope.so")) if pkg._native._lib is None else pkg._native.C.CDLL(
            str(tmp_path / "nope.so"))
