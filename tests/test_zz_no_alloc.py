"""gd2d_update_variables_noalloc: the allocation-free entry point for callers
that own all device memory (their own pool or an allocation-free step loop).

The caller allocates every input and output (here with torch); the entry
point must give the same primitives, residuals and Uold <- Unew update as
the handle-based step (gd2d_propagate + gd2d_get_state), on two calls in a
row, since calls share the library's fixed scratch array.  This file is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64).reshape(-1, 4, order="F") if np.ndim(a) == 1 else np.asarray(a)
    b = np.asarray(b, dtype=np.float64)
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    return float((np.abs(a - b).max(axis=0) / scale).max())


def test_noalloc_update_matches_handle_step(pkg):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    N = pkg._native
    L = N.load()
    mesh, cfg, prims = pkg.cases.square_inviscid(61)
    s = pkg.setupSolver(mesh, cfg)
    s.createFields2d(0, *prims)
    n = mesh.nCells
    U_prev = s.get_state(0)["Ucons"]
    stream = torch.cuda.current_stream()
    for call in range(2):
        st = s.propagate2d(1)[0]
        g = s.get_state(0)
        U_new, P_new = g["Ucons"], g["prims"]
        d_unew = torch.from_numpy(U_new.ravel(order="F").copy()).cuda()
        d_uold = torch.from_numpy(U_prev.ravel(order="F").copy()).cuda()
        d_prims = torch.zeros(4 * n, dtype=torch.float64, device="cuda")
        d_stats = torch.zeros(6, dtype=torch.float64, device="cuda")
        rc = L.gd2d_update_variables_noalloc(d_unew.data_ptr(), d_uold.data_ptr(), d_prims.data_ptr(), n,
                                             cfg["thermo"]["Gamma"], d_stats.data_ptr(),
                                             C.c_void_p(stream.cuda_stream))
        assert rc == 0, L.gd2d_last_error(None)
        torch.cuda.synchronize()
        prims_out = d_prims.cpu().numpy().reshape(n, 4, order="F")
        uold_out = d_uold.cpu().numpy().reshape(n, 4, order="F")
        stats = d_stats.cpu().numpy()
        assert _rel(prims_out, P_new) <= TOL, call
        assert np.array_equal(uold_out, U_new), call
        for v in range(4):
            assert stats[v] == pytest.approx(st["residual"][v], rel=TOL, abs=1e-300), (call, v)
        rho, ux, uy, p = P_new[:, 0], P_new[:, 1], P_new[:, 2], P_new[:, 3]
        vmax = np.sqrt(ux * ux + uy * uy) + np.sqrt(1.4 * p / rho)
        assert stats[4] == pytest.approx(vmax.max(), rel=TOL)
        assert stats[5] == 0.0
        U_prev = U_new
    s.close()


def test_noalloc_rejects_oversize_and_null(pkg):
    L = pkg._native.load()
    rc = L.gd2d_update_variables_noalloc(C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), (1 << 24) + 1, 1.4,
                                         C.c_void_p(16), None)
    assert rc == -1
    assert b"16777216" in L.gd2d_last_error(None)
    assert L.gd2d_update_variables_noalloc(None, None, None, 10, 1.4, None, None) == -1
