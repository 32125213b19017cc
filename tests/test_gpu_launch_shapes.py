"""Launch shapes do not change results, and the autotuner leaves no trace.

Every launch-shape knob of gd2d_launch (register budget, persistent grid,
node-pass block, steps per graph, cell block) must give bit-identical FP64
states: the per-tile reductions are ordered by tile, not by block, and each
cell's arithmetic does not depend on where it runs.  gd2d_autotune runs
trial steps on the handle's own state and must restore it exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _viscous_case(pkg):
    return pkg.cases.cylinder_case(129)


def _run(pkg, mesh, cfg, prims, nsteps, **launch):
    s = pkg.setupSolver(mesh, cfg, **launch)
    s.createFields2d(0, *prims)
    s.propagate2d(nsteps)
    st = s.get_state(0)
    h = s.history(0)
    s.close()
    return st, h


@pytest.mark.parametrize("shape", [
    {"min_blocks": 2}, {"min_blocks": 4}, {"persistent": 1}, {"persistent": 1, "min_blocks": 4},
    {"node_block": 64}, {"node_block": 128}, {"node_block": 256}, {"block": 128}, {"graph_steps": 1},
    {"graph_steps": 128},
    {"loop": "cell"}, {"loop": "cell", "min_blocks": 2}, {"loop": "tile", "min_blocks": 2},
    {"loop": "tile", "persistent": 1, "min_blocks": 4},
])
def test_launch_shape_is_bit_exact(pkg, shape):
    mesh, cfg, prims = _viscous_case(pkg)
    ref, href = _run(pkg, mesh, cfg, prims, 40)
    got, hgot = _run(pkg, mesh, cfg, prims, 40, **shape)
    for k in ("Ucons", "prims", "node_prims"):
        assert np.array_equal(ref[k], got[k]), (shape, k)
    assert [h["dt"] for h in href] == [h["dt"] for h in hgot]
    if "block" not in shape:
        # the step statistics too: each tile folds its 256 cells in a fixed
        # order, and the node pass folds the tile records in an order that
        # depends neither on its block size nor on which warp finishes last
        assert href == hgot, shape


@pytest.mark.parametrize("precision,loop", [("f64", "cell"), ("f64", "tile"), ("mixed", "cell"), ("mixed", "tile")])
def test_autotune_restores_state(pkg, precision, loop):
    """The trials leave no trace: the state right after gd2d_autotune is the
    state before it, and the run continues from there (FP64: bit-identical
    to a run that never tuned; mixed: its FP32 arithmetic may round
    differently under another register budget, so within 1e-6)."""
    mesh, cfg, prims = _viscous_case(pkg)
    ref, href = _run(pkg, mesh, cfg, prims, 30, precision=precision, loop=loop)
    s = pkg.setupSolver(mesh, cfg, precision=precision, loop=loop)
    s.createFields2d(0, *prims)
    s.propagate2d(10)
    before = s.get_state(0)
    chosen = s.autotune(steps_per_trial=16)
    after = s.get_state(0)
    for k in ("Ucons", "prims", "node_prims"):
        assert np.array_equal(before[k], after[k]), k
    assert chosen["min_blocks"] in (2, 3, 4) and chosen["persistent"] in (0, 1)
    assert chosen["node_block"] in (64, 128, 256) and chosen["graph_steps"] in (8, 32, 128)
    assert chosen["ms_per_step"] > 0.0
    s.propagate2d(20)
    got = s.get_state(0)
    h = s.history(0)
    s.close()
    assert len(h) == 30 and h[-1]["step"] == 30
    if precision == "f64":
        for k in ("Ucons", "prims", "node_prims"):
            assert np.array_equal(ref[k], got[k]), k
        assert [x["dt"] for x in h] == [x["dt"] for x in href]
    else:
        U, R = got["Ucons"], ref["Ucons"]
        assert (np.abs(U - R).max(axis=0) / np.abs(R).max(axis=0)).max() <= 1e-6
        assert h[-1]["flowTime"] == pytest.approx(href[-1]["flowTime"], rel=1e-6)


def test_autotune_keeps_a_set_graph_length(pkg):
    """A graph length set in the launch record (as the batched Taylor-Green
    workload sets 100 steps) is not searched: the autotuner keeps it and
    tunes the rest."""
    mesh, cfg, prims = _viscous_case(pkg)
    s = pkg.setupSolver(mesh, cfg, graph_steps=16)
    s.createFields2d(0, *prims)
    chosen = s.autotune(steps_per_trial=16)
    assert chosen["graph_steps"] == 16
    s.propagate2d(40)
    assert s.history(0)[-1]["step"] == 40
    s.close()


def test_autotune_layout_picks_a_timed_candidate(pkg):
    """Ordering and tile size are chosen among timed handles of their own;
    the chosen layout steps to the same FP64 state as any other (results do
    not depend on the layout)."""
    mesh, cfg, prims = _viscous_case(pkg)
    kw, trials = pkg.solver.autotune_layout([mesh], [cfg], [prims], orders=("hilbert", "natural"),
                                            blocks=(256, 128), steps=16)
    assert len(trials) == 4 and all(t["ms_per_step"] > 0.0 for t in trials)
    best = min(trials, key=lambda t: t["ms_per_step"])
    assert (kw["order"], kw["block"]) == (best["order"], best["block"])
    out = []
    for launch in (kw, {"order": "natural", "block": 256}):
        s = pkg.setupSolver(mesh, cfg, **launch)
        s.createFields2d(0, *prims)
        s.propagate2d(12)
        out.append(s.get_state(0)["Ucons"])
        s.close()
    assert np.array_equal(out[0], out[1])


def test_autotune_needs_state(pkg):
    mesh, cfg, prims = _viscous_case(pkg)
    s = pkg.setupSolver(mesh, cfg)
    with pytest.raises(pkg._native.NativeError):
        s.autotune(8)
    s.close()


def test_device_out_of_range(pkg):
    """The handle's device is named in the launch record (the library links
    its own CUDA runtime); a device the process cannot see is an argument
    error, not a CUDA failure."""
    mesh, cfg, prims = pkg.cases.square_inviscid(9)
    with pytest.raises(pkg._native.NativeError) as ei:
        pkg.setupSolver(mesh, cfg, device=999)
    assert "device 999" in str(ei.value)
