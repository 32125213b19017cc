"""Benchmark of the explicit Godunov step on B200.

Default workload (one GPU): the plain-FP64 viscous supersonic cylinder,
[-5,15]x[-8,8] on a 1025^2 node grid, triangulated, cells inside r<0.5
removed (~2.09M cells), M=3.5, Re_D=1e4, Sutherland + artificial viscosity,
Venkatakrishnan limiter, AUSM+, local-CFL 0.4.  A "step" is one explicit
time step over all cells.  Synthetic, seeded inputs (no dataset exists).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--config cylinder|square|tgv_batch|cyl_batch] [--precision f64|mixed]

value: cell-steps/s (Mcell-steps/s) with state resident in HBM, device
time from CUDA events on the solver's stream, max over ranks.  The working
set (~0.9 GB) is far larger than L2, so no flush is needed between steps.
e2e: the same metric through the C ABI with host buffers: set_state of
every case from page-locked host arrays (copied to the device directly),
K x gd2d_propagate(h, 1, stats) (per-step stats read back), gd2d_get_state
of every case's final conservatives.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import platform
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import __graft_entry__ as graft  # noqa: E402

# Algorithmic bytes per cell-step (compulsory traffic of the reference
# dataflow: state read+write, face geometry, connectivity, node-average
# cluster data; intermediates counted zero) for the whole step ...
ALG_BYTES = {("f64", False): 216, ("f64", True): 248, ("mixed", False): 164, ("mixed", True): 192}
# ... and for the fused cell kernel alone: the same without the node pass's
# cluster ids and weights, 0.5 nodes per cell x 6 cells x (4 + weight bytes)
# = 36 B in FP64 and 24 B in the mixed path.
CELL_ALG_BYTES = {("f64", False): 180, ("f64", True): 212, ("mixed", False): 140, ("mixed", True): 168}

# DRAM bytes per cell of one cell-kernel launch on the viscous cylinder,
# measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum of one
# launch; FP64 cell-centred on 1025^2 nodes, the others on 513^2 nodes, the
# traffic growing in proportion to the cells); None where not captured.
CELL_KERNEL_TRAFFIC = {("f64", "cell"): 337.0, ("f64", "tile"): 282.0, ("mixed", "cell"): 233.0,
                       ("mixed", "tile"): 149.0}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def build_workload(pkg, config: str, precision: str, size: int = 1025):
    C = pkg.cases
    if config == "square":
        mesh, cfg, prims = C.square_inviscid(101)
        cfg = dict(cfg, dt_mode=2)
        items = [(mesh, cfg, prims)]
        desc = {"workload": "square_inviscid_fp64", "mesh": "unit square 101x101 nodes, jittered tris",
                "cells": mesh.nCells}
    elif config == "tgv_batch":
        items = C.batched_tgv(64)
        desc = {"workload": "batched_tgv_64", "cases": 64, "cells": sum(m.nCells for m, _, _ in items)}
    elif config == "cyl_batch":
        items = C.batched_cylinders(16)
        desc = {"workload": "batched_cylinders_16", "cases": 16, "cells": sum(m.nCells for m, _, _ in items)}
    else:
        mesh, cfg, prims = C.cylinder_case(size)
        cfg = dict(cfg, dt_mode=2)
        items = [(mesh, cfg, prims)]
        desc = {"workload": "cylinder_viscous_fp64" if precision == "f64" else "cylinder_viscous_mixed",
                "mesh": "[-5,15]x[-8,8] %d^2 nodes, tris, r<0.5 removed" % size, "cells": mesh.nCells,
                "mach": 3.5, "re_d": 1.0e4, "limiter": "venkatakrishnan", "viscosity": "sutherland+artificial"}
    viscous = items[0][1].get("viscosity", "none") != "none"
    return items, desc, viscous


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
        dist = td
    return world, rank, local, dist


def dist_max(dist, x):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_sum(dist, x):
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def dist_barrier(dist):
    if dist is not None:
        dist.barrier()


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def cpu_reference(pkg, items, steps, warmup, budget_s=25.0, single_thread_s=8.0):
    """Time the CPU restatement of the reference step (oracle) on a bounded
    sample of the workload: all host threads, `warmup` untimed steps (at
    least 3, at most ~10 s of them), then five timed repeats of equal length
    (median reported); plus a one-thread figure on a step or two."""
    from oracle import oracle as orc
    orc.build()
    nthreads = os.cpu_count() or 1
    mesh, cfg, prims = items[0]
    cells = mesh.nCells
    o = orc.Oracle(mesh, cfg, nthreads=nthreads)
    o.init_fields(*prims)
    t0 = time.perf_counter()
    o.step()
    t1 = time.perf_counter() - t0
    n_warm = max(3, min(warmup, int(10.0 / max(t1, 1e-6))))
    for _ in range(n_warm - 1):
        o.step()
    reps = 5
    per_rep = max(1, min(steps, int(budget_s / reps / max(t1, 1e-6))))
    rates = []
    for _ in range(reps):
        t0 = time.perf_counter()
        for _ in range(per_rep):
            o.step()
        rates.append(cells * per_rep / (time.perf_counter() - t0) / 1e6)
    rates.sort()
    single = None
    if single_thread_s > 0:
        o1 = orc.Oracle(mesh, cfg, nthreads=1)
        o1.init_fields(*prims)
        t0 = time.perf_counter()
        o1.step()
        ts = time.perf_counter() - t0
        n1 = max(1, min(3, int(single_thread_s / max(ts, 1e-6))))
        t0 = time.perf_counter()
        for _ in range(n1):
            o1.step()
        single = cells * n1 / (time.perf_counter() - t0) / 1e6
    return {"value": rates[len(rates) // 2], "unit": "Mcell-steps/s", "cores": nthreads, "kind": "port",
            "sample": f"median of {reps} repeats of {per_rep} steps of case 0 ({cells} cells) after {n_warm} "
                      f"warm-up steps, {nthreads} threads", "warmup": n_warm,
            "repeats": [round(r, 4) for r in rates], "single_thread_value": single, "host": cpu_model()}


def parity_block(pkg, items, s, steps=100):
    """The FP64 GPU step against the CPU oracle on the full workload (case 0),
    both from the same initial state: per-variable max|gpu - oracle| / max|oracle|
    of the conservative state after step 1 and after `steps` steps, and
    whether the states are equal bit for bit.  Tolerances: 1e-12 per step,
    1e-10 after 100 steps."""
    from oracle import oracle as orc
    orc.build()
    mesh, cfg, prims = items[0]
    nthreads = os.cpu_count() or 1
    o = orc.Oracle(mesh, cfg, nthreads=nthreads)
    o.init_fields(*prims)
    s.createFields2d(0, *prims)
    out = {"cells": mesh.nCells, "oracle_threads": nthreads, "vars": ["rho", "rho_u", "rho_v", "E"],
           "tolerance": {"1": 1e-12, str(steps): 1e-10}}
    t0 = time.perf_counter()
    done = 0
    for k in (1, steps):
        s.propagate2d(k - done)
        for _ in range(k - done):
            o.step()
        done = k
        g = s.get_state(0)["Ucons"]
        r = o.field("Uold")
        scale = np.maximum(np.abs(r).max(axis=0), 1e-300)
        err = (np.abs(g - r).max(axis=0) / scale)
        out["after_%d" % k] = {"max_rel_err": [float(x) for x in err], "bit_equal": bool(np.array_equal(g, r))}
    out["seconds"] = round(time.perf_counter() - t0, 1)
    out["pass"] = bool(max(out["after_1"]["max_rel_err"]) <= 1e-12 and
                       max(out["after_%d" % steps]["max_rel_err"]) <= 1e-10)
    return out


def mixed_variant(pkg, items, s64, args, peak):
    """The same workload on the mixed-precision path: device-timed
    throughput, and the error after --error-steps steps against the FP64 path
    (bit-identical to the CPU oracle in the parity tests) from the same
    initial state."""
    mesh, cfg, prims = items[0]
    sm = pkg.solver.Solver([mesh], [cfg], pkg.solver.make_launch(precision="mixed", order=args.order, loop=args.loop,
                                                                device=args.device))
    sm.createFields2d(0, *prims)
    sm.propagate2d(args.gpu_warmup)
    sm.propagate2d(args.steps)
    tot, cell_ms, _ = sm.last_timing()
    value = mesh.nCells * args.steps / (tot / 1e3) / 1e6
    visc = cfg.get("viscosity", "none") != "none"
    alg, calg = ALG_BYTES[("mixed", visc)], CELL_ALG_BYTES[("mixed", visc)]
    # error run: both paths from the initial state
    n_err = args.error_steps
    sm.createFields2d(0, *prims)
    s64.createFields2d(0, *prims)
    hm = sm.propagate2d(n_err)[0]
    h64 = s64.propagate2d(n_err)[0]
    Um = sm.get_state(0)["Ucons"]
    U64 = s64.get_state(0)["Ucons"]
    # relative errors per variable; the momentum components are scaled by
    # the momentum magnitude (one of them may be zero everywhere)
    d = Um - U64
    mom = np.sqrt(U64[:, 1] ** 2 + U64[:, 2] ** 2)
    n2 = np.sqrt((U64 ** 2).sum(axis=0))
    n2[1] = n2[2] = np.sqrt((mom ** 2).sum())
    ninf = np.abs(U64).max(axis=0)
    ninf[1] = ninf[2] = mom.max()
    l2 = np.sqrt((d ** 2).sum(axis=0)) / np.maximum(n2, 1e-300)
    linf = np.abs(d).max(axis=0) / np.maximum(ninf, 1e-300)
    hist_m = sm.history(0)
    hist_64 = s64.history(0)
    t0m, t064 = hist_m[0]["totals"], hist_64[0]["totals"]
    tscale = [abs(t064[0]), math.hypot(t064[1], t064[2]), math.hypot(t064[1], t064[2]), abs(t064[3])]
    drift = [abs((hm["totals"][v] - t0m[v]) - (h64["totals"][v] - t064[v])) / max(tscale[v], 1e-300)
             for v in range(4)]
    # the densityConstrained clamp (evaluate2d.jl:63-77): cells sitting at
    # the lower bound after the error run, and their share of the mass
    clamp = None
    if cfg.get("densityConstrained", 0):
        lo = cfg.get("minDensityConstrained", 0.01)
        A = mesh.cell_areas
        clamp = {"bound": lo}
        for tag, U in (("fp64", U64), ("mixed", Um)):
            at = U[:, 0] <= lo
            clamp[tag] = {"cells_at_bound": int(at.sum()), "cell_fraction": float(at.mean()),
                          "mass_fraction": float((U[at, 0] * A[at]).sum() / (U[:, 0] * A).sum())}
    sm.close()
    return {"value": value, "unit": "Mcell-steps/s", "ms_per_step": tot / args.steps, "cell_kernel_ms": cell_ms,
            "roofline": {"achieved": calg * mesh.nCells / (cell_ms / 1e3) / 1e9 if cell_ms else None, "peak": peak,
                         "frac": (calg * mesh.nCells / (cell_ms / 1e3) / 1e9 / peak) if cell_ms else None,
                         "alg_bytes_per_cell": calg, "step_alg_bytes_per_cell": alg,
                         "step_frac": alg * mesh.nCells / (tot / args.steps / 1e3) / 1e9 / peak},
            "error_vs_fp64": {"steps": n_err, "momentum_scaled_by": "momentum magnitude",
                              "l2_rel": [float(x) for x in l2], "linf_rel": [float(x) for x in linf],
                              "vars": ["rho", "rho_u", "rho_v", "E"], "totals_drift_rel": drift},
            "density_clamp": clamp}


def batched_mixed(pkg, items, s64, args, peak, kind):
    """Configs 4 and 5: every case of the batch on the mixed-precision path in
    one handle (one launch per kernel per step for all cases), launch shapes
    picked by gd2d_autotune starting from a 100-step CUDA graph; device-timed
    aggregate throughput and roofline, then a per-case error after
    `--error-steps` steps against the FP64 path from the same initial states
    (the FP64 path is bit-identical to the CPU oracle in the parity tests, so
    it stands in for the oracle at these sizes).  TGV: the relative error of
    the kinetic energy Ek(t) and of its decay E0 - Ek(t); cylinders: the
    relative L2 error of the density."""
    meshes = [m for m, _, _ in items]
    cfgs = [c for _, c, _ in items]
    cells = sum(m.nCells for m in meshes)
    # ordering and tile size first (each a handle of its own), then the
    # launch shape on the chosen layout; the step loop is a 100-step graph
    kw, layout_trials = pkg.solver.autotune_layout(meshes, cfgs, [p for _, _, p in items], precision="mixed",
                                                   loop=args.loop, device=args.device, graph_steps=100)
    sm = pkg.solver.Solver(meshes, cfgs, pkg.solver.make_launch(**kw))
    for i, (_, _, p) in enumerate(items):
        sm.createFields2d(i, *p)
    tuned = dict(sm.autotune(64), order=kw["order"], block=kw["block"])
    sm.propagate2d(args.gpu_warmup)
    sm.propagate2d(args.steps)
    tot, cell_ms, launches = sm.last_timing()
    value = cells * args.steps / (tot / 1e3) / 1e6
    visc = cfgs[0].get("viscosity", "none") != "none"
    alg, calg = ALG_BYTES[("mixed", visc)], CELL_ALG_BYTES[("mixed", visc)]
    n_err = args.error_steps
    for i, (_, _, p) in enumerate(items):
        sm.createFields2d(i, *p)
        s64.createFields2d(i, *p)

    def run_all(h, n):
        # cases are independent: one that leaves the admissible set (the
        # call reports GD2D_ERR_NONFINITE after its chunk) does not touch
        # the others, which keep stepping
        done = 0
        while done < n:
            k = min(500, n - done)
            try:
                h.propagate2d(k)
            except pkg._native.NativeError as e:
                if e.code != -4:
                    raise
            done += k

    def first_bad(h, i):
        for st in h.history(i):
            if st["nonfinite"]:
                return st["step"]
        return None

    run_all(sm, n_err)
    run_all(s64, n_err)
    per_case = []
    for i, (m, c, p) in enumerate(items):
        rec = dict({"case": i, "cells": m.nCells}, **c.get("case_info", {}))
        bad64, badm = first_bad(s64, i), first_bad(sm, i)
        if bad64 or badm:
            # the FP64 path is the oracle's scheme bit for bit: a case it
            # cannot step is a limit of the scheme, reported, not compared
            rec.update({"left_admissible_set_at_step": {"fp64": bad64, "mixed": badm}})
            per_case.append(rec)
            continue
        if kind == "tgv":
            rho, u, v, _ = p
            e0 = float((0.5 * rho * (u * u + v * v) * m.cell_areas).sum())
            ekm, ek64 = sm.history(i, 1)[-1]["Ek"], s64.history(i, 1)[-1]["Ek"]
            rec.update({"ek_over_e0_fp64": ek64 / e0,
                        "ek_rel_err": abs(ekm - ek64) / ek64,
                        "decay_rel_err": abs((e0 - ekm) - (e0 - ek64)) / max(e0 - ek64, 1e-300)})
        else:
            rm = sm.get_state(i)["Ucons"][:, 0]
            r64 = s64.get_state(i)["Ucons"][:, 0]
            rec["rho_l2_rel_err"] = float(np.sqrt(((rm - r64) ** 2).sum() / (r64 ** 2).sum()))
            rec["rho_linf_rel_err"] = float(np.abs(rm - r64).max() / np.abs(r64).max())
        per_case.append(rec)
    sm.close()
    key = "decay_rel_err" if kind == "tgv" else "rho_l2_rel_err"
    compared = [r for r in per_case if key in r]
    achieved = calg * cells / (cell_ms / 1e3) / 1e9 if cell_ms else None
    return {"value": value, "unit": "Mcell-steps/s", "cells": cells, "ms_per_step": tot / args.steps,
            "cell_kernel_ms": cell_ms, "gpu_launches": int(launches), "autotuned_launch": tuned,
            "layout_trials": layout_trials,
            "roofline": {"achieved": achieved, "peak": peak, "frac": achieved / peak if achieved else None,
                         "alg_bytes_per_cell": calg, "step_alg_bytes_per_cell": alg,
                         "step_achieved_gbs": alg * cells / (tot / args.steps / 1e3) / 1e9},
            "error_vs_fp64": {"steps": n_err, "cases_compared": len(compared),
                              "max_" + key: max(r[key] for r in compared) if compared else None,
                              "per_case": per_case}}


def roe_from_developed_flow(pkg, items, args):
    """Config 3 with the Roe flux on the cylinder.  An impulsive start takes
    the Roe flux out of the admissible set at the wall, so the comparison
    starts from a developed flow: `--roe-restart` FP64 AUSM+ steps from the
    freestream, then that conservative state and flowTime restart an FP64 and
    a mixed-precision handle with the Roe flux (gd2d_set_conservative), which
    run `--error-steps` steps each.  Reports the mixed-vs-FP64 errors as
    mixed_variant does, or where the FP64 Roe run left the admissible set."""
    mesh, cfg, prims = items[0]
    mk = pkg.solver.make_launch
    base = pkg.solver.Solver([mesh], [dict(cfg, flux="ausm")], mk(precision="f64", order=args.order, loop=args.loop,
                                                                   device=args.device))
    base.createFields2d(0, *prims)
    base.propagate2d(args.roe_restart)
    U0 = base.get_state(0)["Ucons"]
    t0 = base.flow_time(0)
    base.close()
    roe = dict(cfg, flux="roe")
    out = {"restart_steps_ausm": args.roe_restart, "restart_flow_time": t0, "steps": args.error_steps}
    runs = {}
    for prec in ("f64", "mixed"):
        h = pkg.solver.Solver([mesh], [roe], mk(precision=prec, order=args.order, loop=args.loop, device=args.device))
        h.set_conservative(0, U0, t0)
        done, failed = 0, None
        while done < args.error_steps:
            n = min(500, args.error_steps - done)
            try:
                h.propagate2d(n)
            except pkg._native.NativeError as e:
                failed = {"after_steps": done + n, "error": str(e)}
                break
            done += n
        runs[prec] = (h, failed)
        out[prec + "_failed"] = failed
    if runs["f64"][1] is None and runs["mixed"][1] is None:
        Um = runs["mixed"][0].get_state(0)["Ucons"]
        U64 = runs["f64"][0].get_state(0)["Ucons"]
        d = Um - U64
        mom = np.sqrt(U64[:, 1] ** 2 + U64[:, 2] ** 2)
        n2 = np.sqrt((U64 ** 2).sum(axis=0))
        n2[1] = n2[2] = np.sqrt((mom ** 2).sum())
        ninf = np.abs(U64).max(axis=0)
        ninf[1] = ninf[2] = mom.max()
        out["l2_rel"] = [float(x) for x in np.sqrt((d ** 2).sum(axis=0)) / np.maximum(n2, 1e-300)]
        out["linf_rel"] = [float(x) for x in np.abs(d).max(axis=0) / np.maximum(ninf, 1e-300)]
        hm, h64 = runs["mixed"][0].history(0), runs["f64"][0].history(0)
        tm0, t640 = hm[0]["totals"], h64[0]["totals"]
        tscale = [abs(t640[0]), math.hypot(t640[1], t640[2]), math.hypot(t640[1], t640[2]), abs(t640[3])]
        out["totals_drift_rel"] = [abs((hm[-1]["totals"][v] - tm0[v]) - (h64[-1]["totals"][v] - t640[v]))
                                   / max(tscale[v], 1e-300) for v in range(4)]
    for h, _ in runs.values():
        h.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=32)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="cylinder", choices=["cylinder", "square", "tgv_batch", "cyl_batch"])
    ap.add_argument("--precision", default="f64", choices=["f64", "mixed"])
    ap.add_argument("--order", default="hilbert")
    ap.add_argument("--graph-steps", type=int, default=0)
    ap.add_argument("--loop", default="tile", choices=["cell", "tile"],
                    help="cell-centred kernel or the tile-face kernel (same results)")
    ap.add_argument("--min-blocks", type=int, default=0, help="cell-kernel register budget (0: library default)")
    ap.add_argument("--node-block", type=int, default=0)
    ap.add_argument("--size", type=int, default=1025, help="cylinder: nodes per side")
    ap.add_argument("--flux", default=None, choices=["ausm", "roe", "ausm_m2020"],
                    help="override the workload's face flux (cylinder: AUSM+)")
    ap.add_argument("--autotune", action="store_true",
                    help="let gd2d_autotune pick the launch shape before the warm-up")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision comparison")
    ap.add_argument("--no-parity", action="store_true", help="skip the FP64 GPU-vs-oracle parity check")
    ap.add_argument("--parity-steps", type=int, default=100, help="steps of the parity check")
    ap.add_argument("--roe-restart", type=int, default=0,
                    help="cylinder: compare Roe mixed vs FP64 from the state after this many AUSM+ steps")
    ap.add_argument("--error-steps", type=int, default=0,
                    help="steps of the mixed-vs-FP64 error measurement (0: 1000; cyl_batch 2000)")
    args = ap.parse_args()
    if args.error_steps <= 0:
        args.error_steps = 2000 if args.config == "cyl_batch" else 1000
    # at least 3 warm-up steps, and at least one CUDA graph's worth
    args.warmup = max(args.warmup, 3)
    # the GPU arm warms up at least one CUDA graph's worth of steps
    gpu_warmup = max(args.warmup, args.graph_steps if args.graph_steps > 0 else 32)
    args.gpu_warmup = gpu_warmup

    world, rank, local, dist = dist_setup(args)
    # one process per GPU: this rank's GPU (device 0 when the launcher
    # already restricted each process to its own GPU)
    args.device = local
    if world > 1:
        import torch
        if local >= torch.cuda.device_count():
            args.device = 0
    pkg = graft.load_package()
    items, desc, viscous = build_workload(pkg, args.config, args.precision, args.size)
    if args.flux:
        items = [(m, dict(c, flux=args.flux), p) for m, c, p in items]
        desc = dict(desc, flux=args.flux)
    sharded = world > 1 and len(items) > 1
    if sharded:
        # independent cases split across ranks (no data exchange), balanced by cells
        mine = pkg.cases.shard_cases([m.nCells for m, _, _ in items], world, rank)
        items = [items[i] for i in mine]
    metric = "Mcell-steps/s"
    cfg_line = dict(desc, precision=args.precision, loop=args.loop,
                    parallelism=(("cases-sharded%d" if sharded else "replicas%d") % world), l2_flush="inputs > L2")

    if args.impl == "reference":
        if rank != 0:
            dist_barrier(dist)
            return
        cb = cpu_reference(pkg, items, args.steps, args.warmup, budget_s=60.0)
        line = {"impl": "reference", "metric": metric, "value": cb["value"], "unit": cb["unit"], "n_gpus": world,
                "steps": args.steps, "warmup": cb["warmup"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg_line,
                "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "repeats",
                                                    "single_thread_value", "host")},
                "e2e": {"value": cb["value"], "unit": cb["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        dist_barrier(dist)
        return

    meshes = [m for m, _, _ in items]
    cfgs = [c for _, c, _ in items]
    launch = pkg.solver.make_launch(precision=args.precision, order=args.order, graph_steps=args.graph_steps,
                                    device=args.device,
                                    loop=args.loop, min_blocks=args.min_blocks, node_block=args.node_block)
    s = pkg.solver.Solver(meshes, cfgs, launch)
    for i, (_, _, p) in enumerate(items):
        s.createFields2d(i, *p)
    cells = sum(m.nCells for m in meshes)
    if args.autotune:
        cfg_line["launch"] = s.autotune(64)

    # warm-up: at least one full CUDA graph of steps, so that the graph is
    # captured and instantiated before the timed region; the clock sampler
    # starts first, its start-up away from the timed region
    with ClockSampler(local) as clk:
        s.propagate2d(gpu_warmup)
        dist_barrier(dist)
        s.propagate2d(args.steps)
        total_ms, cell_ms, launches = s.last_timing()
    dist_barrier(dist)
    total_ms = dist_max(dist, total_ms)
    clocks = clk.summary()
    # whole-job cells: replicas each run the full mesh; shards add up
    job_cells = dist_sum(dist, cells) if sharded else cells * world
    value = job_cells * args.steps / (total_ms / 1e3) / 1e6
    ms_per_step = total_ms / args.steps

    # end to end through the C ABI with host buffers: every case's state
    # uploaded from the host, K single-step calls with the statistics read
    # back each step, every case's conservatives read back at the end
    import ctypes as C
    N = pkg._native
    L = N.load()
    # host buffers in page-locked memory (allocated before the timed
    # region), which the library's copies read and write directly
    import torch
    pinned = []

    def pinned_array(shape_c):
        t = torch.zeros(shape_c, dtype=torch.float64, pin_memory=True)
        pinned.append(t)
        return t.numpy()

    host_prims = []
    for it in items:
        cols = []
        for x in it[2]:
            a = pinned_array(len(x))
            a[:] = x
            cols.append(a)
        host_prims.append(cols)
    # (n, 4) column-major matrices: the transpose of a (4, n) C-order buffer
    ucons = [pinned_array((4, m.nCells)).T for m in meshes]
    dp = C.POINTER(C.c_double)
    # warm-up: the copy engine's first write into fresh page-locked pages
    # costs ~1.3 ms more than the next ones (an application reuses its
    # buffers), so each output buffer is written once before the timing
    for i, u in enumerate(ucons):
        N.check(L.gd2d_get_state(s.h, i, u.ctypes.data_as(dp), None, None), s.h)
    st = (N.Stats * len(meshes))()
    dist_barrier(dist)
    e2e_steps = args.steps
    tick = time.perf_counter
    call_s, call_dev_ms = [], []
    tdev = C.c_double()
    t0 = tick()
    for i, hp in enumerate(host_prims):
        N.check(L.gd2d_set_state(s.h, i, *[a.ctypes.data_as(dp) for a in hp]), s.h)
    t1 = tick()
    for _ in range(e2e_steps):
        ta = tick()
        N.check(L.gd2d_propagate(s.h, 1, st), s.h)
        call_s.append(tick() - ta)
        L.gd2d_last_timing(s.h, C.byref(tdev), None, None)
        call_dev_ms.append(tdev.value)
    t2 = tick()
    for i, u in enumerate(ucons):
        N.check(L.gd2d_get_state(s.h, i, u.ctypes.data_as(dp), None, None), s.h)
    t3 = tick()
    e2e_s = t3 - t0
    e2e_s = dist_max(dist, e2e_s)
    e2e_val = job_cells * e2e_steps / e2e_s / 1e6
    h2d = 4 * 8 * cells / e2e_steps
    d2h = C.sizeof(N.Stats) * len(meshes) + 4 * 8 * cells / e2e_steps
    # where the end-to-end time goes: host clock around each call, and the
    # device time (CUDA events on the stream) of each one-step propagate
    e2e_breakdown = {"set_state_ms": (t1 - t0) * 1e3, "get_state_ms": (t3 - t2) * 1e3,
                     "propagate_calls_ms": (t2 - t1) * 1e3,
                     "propagate_call_median_ms": statistics.median(call_s) * 1e3,
                     "propagate_call_device_median_ms": statistics.median(call_dev_ms),
                     "propagate_call_host_overhead_median_us":
                         (statistics.median(call_s) * 1e3 - statistics.median(call_dev_ms)) * 1e3,
                     "timed_region_device_ms_per_step": None}

    peak, peak_kind = load_peaks()
    alg, calg = ALG_BYTES[(args.precision, viscous)], CELL_ALG_BYTES[(args.precision, viscous)]
    achieved = calg * cells / (cell_ms / 1e3) / 1e9 if cell_ms > 0 else None
    step_achieved = alg * cells / (ms_per_step / 1e3) / 1e9
    tpc = CELL_KERNEL_TRAFFIC.get((args.precision, args.loop)) if args.config == "cylinder" else None
    traffic = tpc * cells if tpc else None
    traffic_src = ("ncu dram bytes per cell of one launch x cells (%.0f B/cell)" % tpc) if tpc else None
    line = {"metric": metric, "value": value, "unit": "Mcell-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": gpu_warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "f64" else "f32+f64",
            "data": "synthetic (seeded generated meshes and initial states)", "config": cfg_line,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "traffic_source": traffic_src,
                         "kernel": ("k_cell_step_tf" if args.loop == "tile" else "k_cell_step")
                                   + (" (mixed)" if args.precision == "mixed" else "")
                                   + " (fused reconstruction+flux+viscous+update)",
                         "alg_bytes_per_cell": calg, "step_alg_bytes_per_cell": alg, "cell_kernel_ms": cell_ms,
                         "peak_kind": peak_kind,
                         "step_achieved_gbs": step_achieved, "step_frac": step_achieved / peak},
            "e2e": {"value": e2e_val, "unit": "Mcell-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps, "breakdown": dict(e2e_breakdown, timed_region_device_ms_per_step=ms_per_step)},
            "gpu_launches": int(launches), "clocks": clocks}
    if args.config in ("cylinder", "square") and args.precision == "f64" and rank == 0 and world == 1 \
            and not args.no_parity:
        line["parity"] = parity_block(pkg, items, s, args.parity_steps)
    if args.config in ("cylinder", "square") and args.precision == "f64" and not args.no_mixed:
        line["mixed"] = mixed_variant(pkg, items, s, args, peak)
    if args.config in ("tgv_batch", "cyl_batch") and args.precision == "f64" and not args.no_mixed:
        line["mixed"] = batched_mixed(pkg, items, s, args, peak, "tgv" if args.config == "tgv_batch" else "cyl")
    if args.config == "cylinder" and args.roe_restart > 0 and world == 1:
        line["roe_from_developed_flow"] = roe_from_developed_flow(pkg, items, args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_reference(pkg, items, args.steps, args.warmup)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "repeats",
                                                   "single_thread_value", "host")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    s.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
