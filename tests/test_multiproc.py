"""Multi-rank host logic on CPU (gloo, world size 2).

The batched workloads shard independent cases across ranks with no data
exchange; only the statistics are reduced at the end.  This checks that
the shards are disjoint, complete and balanced, and that two ranks each
stepping their own cases (on the CPU oracle) reproduce a single-process
run of all cases bit for bit.
"""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, queue):
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import __graft_entry__ as graft
    from oracle import oracle as orc
    pkg = graft.load_package()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        cases = [pkg.cases.tgv_case(n, 0.2 + 0.05 * k, 300.0 + 50 * k) for k, n in enumerate((9, 13, 11, 17, 7))]
        sizes = [m.nCells for m, _, _ in cases]
        mine = pkg.cases.shard_cases(sizes, world, rank)
        res = {}
        for i in mine:
            m, c, p = cases[i]
            o = orc.Oracle(m, c, nthreads=1)
            o.init_fields(*p)
            h = o.run(5)
            res[i] = (float(o.field("Uold").sum()), h[-1]["Ek"])
        gathered = [None] * world
        dist.all_gather_object(gathered, res)
        if rank == 0:
            queue.put((gathered, sizes))
    finally:
        dist.destroy_process_group()


def test_case_sharding_two_ranks_matches_single_process(pkg, orc):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, sizes = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    owned = [set(g.keys()) for g in gathered]
    assert owned[0].isdisjoint(owned[1]) and owned[0] | owned[1] == set(range(len(sizes)))
    loads = [sum(sizes[i] for i in o) for o in owned]
    assert max(loads) - min(loads) <= max(sizes)
    # single-process reference run of every case
    cases = [pkg.cases.tgv_case(n, 0.2 + 0.05 * k, 300.0 + 50 * k) for k, n in enumerate((9, 13, 11, 17, 7))]
    merged = {}
    for g in gathered:
        merged.update(g)
    for i, (m, c, p) in enumerate(cases):
        o = orc.Oracle(m, c, nthreads=1)
        o.init_fields(*p)
        h = o.run(5)
        assert merged[i] == (float(o.field("Uold").sum()), h[-1]["Ek"])


def test_shard_cases_properties(pkg):
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        sizes = [int(x) for x in rng.integers(1000, 500000, size=64)]
        shards = [pkg.cases.shard_cases(sizes, world, r) for r in range(world)]
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(64))
        loads = [sum(sizes[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(sizes)
