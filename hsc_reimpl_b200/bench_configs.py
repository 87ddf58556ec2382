"""Measurements of the other configurations of the HSC workload (one B200).

    python -m hsc_reimpl_b200.bench_configs [--only c1,c3,c4,c5] [--out report.json]

c1  the 1,331-node cube with one affine plate (error against a sparse direct solve)
c3  64 uneven systems in one persistent launch replayed as a CUDA graph, FP32
    values with FP64 residual replacement every 50 iterations, after the
    autotuner (tile width x ACA rank cap 4-256; omega 0.6)
c4  the learned polynomial preconditioner on held-out vehicle trajectories:
    PCG iterations and time to 1e-6 against plain order-2 Neumann (FP64 and FP32)
vehicle  two solves of the vehicle system in --vehicle-precision (default FP64; a short, fixed command
         for profilers)
assembly GPU assembly of the vehicle's 78,120-tet log-NH Hessian (hsc_fem_assemble) per call,
         the line-search feasible step of a rough direction (hsc_fem_feasible_step) and the
         ABD-FEM contact coupling with its E (hsc_coupling_assemble, 40,000 contacts)
c5  the 1 M-tet torus (12 bodies, 30 % contact-active tread): FP64 / FP32 /
    BF16 solves with their error against a tight FP64 reference, ACA rank sweep
    8-64, Neumann order sweep 1-4, HBM GB/s of the full-H SpMV

The vehicle system itself is bench.py's workload.  Times are CUDA-event times
on the solving stream; L2 is flushed between timed solves.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def log(msg):
    print(msg, flush=True)


def _timed_solves(ctx, ds, reps, flush):
    import torch
    x = torch.empty_like(ds.b)
    ctx.solve(ds, x=x, raise_on_error=False)
    ms, stats = [], None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        e0.record()
        _, stats = ctx.solve(ds, x=x, raise_on_error=False)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return statistics.median(ms), stats, x


def c1(flush):
    import scipy.sparse.linalg as spla
    from .solver import DeviceSystem, HSCContext, HSCOptions
    from .systems import make_cube_system
    s = make_cube_system(seed=0)
    opts = dict(neumann_order=2, omega=2 / 3, aca_rtol=1e-4, tol=1e-6)
    ds = DeviceSystem.from_system(s)
    ctx = HSCContext(HSCOptions(abd_inverse="exact", **opts))
    ms, st, x = _timed_solves(ctx, ds, 20, flush)
    xd = spla.splu(s.H.tocsc()).solve(s.b)
    xs = x.cpu().numpy()
    return {"workload": "cube_1331_nodes_5000_tets", "gpu_ms_per_solve": ms, "gpu_solves_per_s": 1000 / ms,
            "pcg_iterations": st["pcg_iterations"], "rank": st["rank"],
            "full_relative_residual": st["full_relative_residual"],
            "error_vs_direct": float(np.linalg.norm(xs - xd) / np.linalg.norm(xd))}


def c3(flush, count=64):
    import torch
    from .autotune import autotune, time_batch
    from .solver import DeviceSystem, HSCContext, HSCOptions
    from .systems import make_batch_systems
    t = time.time()
    systems = make_batch_systems(seed=0, count=count)
    gen_s = time.time() - t
    devs = [DeviceSystem.from_system(s) for s in systems]
    base = HSCOptions(precision="fp32", residual_replacement=50, omega=0.6)
    best, table = autotune(devs, base=base, log=log)
    out = {"workload": f"batch_{count}_uneven", "systems": count, "generation_s": gen_s,
           "tets": [int(s.meta["tets"]) for s in systems], "bodies": [int(s.meta["bodies"]) for s in systems],
           "autotune": table}
    if best is not None:
        ctx = HSCContext(best)
        xs = [torch.empty_like(d.b) for d in devs]
        ms_graph, stats = time_batch(ctx, devs, xs, reps=5, use_graph=True)
        ms_plain, _ = time_batch(ctx, devs, xs, reps=5, use_graph=False)
        out.update(best={"threads_per_row": best.threads_per_row, "max_rank": best.max_rank},
                   ms_per_batch_graph=ms_graph, ms_per_batch_no_graph=ms_plain,
                   solves_per_s=count * 1000 / ms_graph,
                   iterations=[s["pcg_iterations"] for s in stats],
                   max_full_relative_residual=max(s["full_relative_residual"] for s in stats))
    return out


def c4(steps=40):
    from . import learned as L
    if not L.MODEL_PATH.exists():
        return {"skipped": "no trained model file"}
    bits, meta = L.load_model()
    base = L.VehicleBase(meta.get("eval_variant", 4))
    out = {"model": meta}
    for prec in ("fp64", "fp32"):
        trajs = [L.VehicleTrajectory(base, seed=s, steps=steps) for s in meta.get("eval_seeds", [9001, 9002])]
        res = L.evaluate(bits, trajs, precision=prec)
        out[prec] = {k: {"mean_iterations": float(v["iters"].mean()), "mean_pcg_ms": float(v["pcg_ms"].mean()),
                         "mean_total_ms": float(v["total_ms"].mean()), "fallbacks": int(v["fallback"].sum()),
                         "max_full_relative_residual": float(v["full"].max())} for k, v in res.items()}
        log(json.dumps({prec: out[prec]}))
    return out


def c5(flush):
    import torch
    from .solver import DeviceSystem, HSCContext, HSCOptions
    from .systems import make_stress_system
    t = time.time()
    s = make_stress_system(seed=0)
    out = {"workload": "stress_torus_1M_tets", "generation_s": time.time() - t, "meta": s.meta}
    ds = DeviceSystem.from_system(s)
    del s
    # the coupling to 12 bodies has rank up to 144: caps below it leave an ACA
    # error that makes the approximate Schur complement indefinite (the sweep
    # below shows it), so the precision runs use an uncapped rank
    # the tight reference replaces the recursive residual by the true one every 50 iterations: at
    # tol 1e-10 on this conditioning the plain recurrence drifts away from the true residual
    ref_ctx = HSCContext(HSCOptions(neumann_order=2, tol=1e-10, max_rank=256, max_iter=50000,
                                    residual_replacement=50))
    xr, sr = ref_ctx.solve(ds, raise_on_error=False)
    xr = xr.clone()
    out["reference"] = {"pcg_iterations": sr["pcg_iterations"], "full_relative_residual": sr["full_relative_residual"]}
    modes = {}
    for prec in ("fp64", "fp32", "bf16"):
        o = HSCOptions(neumann_order=2, tol=1e-6, max_rank=256, precision=prec,
                       residual_replacement=0 if prec == "fp64" else 50)
        ctx = HSCContext(o)
        ms, st, x = _timed_solves(ctx, ds, 3, flush)
        modes[prec] = {"ms_per_solve": ms, "pcg_iterations": st["pcg_iterations"], "status": st["status"],
                       "full_relative_residual": st["full_relative_residual"], "pcg_ms": st["pcg_ms"],
                       "error_vs_fp64_reference": float(torch.linalg.vector_norm(x - xr) / torch.linalg.vector_norm(xr)),
                       "stage_ms": st["stage_ms"], "rank": st["rank"], "active_fem_dofs": st["active_fem_dofs"]}
        log(json.dumps({prec: modes[prec]}))
    out["precision"] = modes
    ranks = {}
    for r in (8, 16, 32, 64, 256):
        ctx = HSCContext(HSCOptions(neumann_order=2, tol=1e-6, max_rank=r))
        ms, st, _ = _timed_solves(ctx, ds, 2, flush)
        ranks[r] = {"ms_per_solve": ms, "pcg_iterations": st["pcg_iterations"], "rank": st["rank"],
                    "aca_relative_error": st["aca_relative_error"], "aca_ms": st["stage_ms"][1],
                    "full_relative_residual": st["full_relative_residual"]}
        log(json.dumps({"rank": r, **ranks[r]}))
    out["rank_sweep"] = ranks
    orders = {}
    for k in (1, 2, 3, 4):
        ctx = HSCContext(HSCOptions(neumann_order=k, tol=1e-6, max_rank=256, omega=0.5))
        ms, st, _ = _timed_solves(ctx, ds, 2, flush)
        orders[k] = {"ms_per_solve": ms, "pcg_iterations": st["pcg_iterations"], "status": st["status"],
                     "pcg_us_per_iteration": 1000 * st["pcg_ms"] / max(1, st["pcg_iterations"])}
        log(json.dumps({"order": k, **orders[k]}))
    out["order_sweep"] = orders
    # full-H SpMV: algorithmic bytes / event time
    ctx = HSCContext(HSCOptions())
    xv = torch.randn_like(ds.b)
    y = ctx.spmv(ds, xv)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for _ in range(10):
        flush.zero_()
        torch.cuda.synchronize()
        e0.record()
        ctx.spmv(ds, xv, y)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    nnzb = int(ds.rows.numel())
    n = ds.nblock
    full_blocks = 2 * nnzb - n  # both triangles (about: diagonal blocks once)
    # per stored-or-mirrored block: its 72 B of values (read once per direction), column index, plan entry
    alg_bytes = full_blocks * (72 + 4 + 4) + 4 * (n + 1) + 2 * 3 * n * 8
    ms = statistics.median(times)
    out["spmv"] = {"ms": ms, "algorithmic_bytes": alg_bytes, "achieved_gbs": alg_bytes / (ms / 1000) / 1e9,
                   "note": "hsc_spmv: gather + row-owner SpMV reading the BCOO blocks + coupling + scatter, FP64"}
    log(json.dumps(out["spmv"]))
    return out


def assembly(reps=10):
    import torch
    from .assembly import FemAssembler
    from .systems import annulus_mesh
    xs, ts, off = [], [], 0
    for t in range(7):
        x, tets, _ = annulus_mesh(center=(1.2 * (t % 4), 0.5 * (t // 4), 0.0))
        xs.append(x)
        ts.append(tets + off)
        off += len(x)
    x = np.concatenate(xs)
    tets = np.concatenate(ts)
    rng = np.random.default_rng(0)
    h = np.cbrt((np.abs(np.linalg.det(x[tets[:, 1:]] - x[tets[:, :1]])) / 6.0).mean())
    xp = torch.from_numpy(x + 0.02 * h * rng.standard_normal(x.shape)).cuda()
    E = torch.full((len(tets),), 1e8, dtype=torch.float64, device="cuda")
    asm = FemAssembler(tets, x)
    vals = asm.assemble(xp, E)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for _ in range(reps):
        e0.record()
        asm.assemble(xp, E, values=vals, check=False)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    m = statistics.median(ms)
    # line-search feasibility of a rough direction (about half the tets limit the step)
    dx = torch.from_numpy(0.5 * h * rng.standard_normal(x.shape)).cuda()
    feas = asm.feasible_step(xp, dx)
    fs = []
    for _ in range(reps):
        e0.record()
        asm.feasible_step(xp, dx)  # includes the read of (alpha, halvings) to the host
        e1.record()
        torch.cuda.synchronize()
        fs.append(e0.elapsed_time(e1))
    # ABD-FEM contact coupling: 12 bodies x 400 vertices, 40,000 contacts on the 19,530 FEM nodes
    from .assembly import CouplingAssembler
    nb, nv, ncon = 12, 400, 40_000
    v2b = np.repeat(np.arange(nb), nv).astype(np.int32)
    xbar = rng.uniform(-1, 1, (nb * nv, 3))
    av = rng.integers(0, nb * nv, ncon).astype(np.int32)
    fv = rng.integers(0, len(x), ncon).astype(np.int32)
    nrm = rng.standard_normal((ncon, 3))
    Hc = -(nrm[:, :, None] * nrm[:, None, :]).reshape(-1, 9)
    ca = CouplingAssembler(v2b, xbar, nb, len(x))
    avd, fvd, Hd = (torch.from_numpy(a).cuda() for a in (av, fv, Hc))
    cp = ca.assemble(avd, fvd, Hd)
    cs = []
    for _ in range(reps):
        e0.record()
        ca.assemble(avd, fvd, Hd)  # includes its one stream sync (sizes E) and the copies out
        e1.record()
        torch.cuda.synchronize()
        cs.append(e0.elapsed_time(e1))
    return {"tets": int(len(tets)), "nodes": int(len(x)), "blocks": int(asm.nnzb), "ms": m,
            "tets_per_s": len(tets) / (m / 1000),
            "coupling": {"bodies": nb, "contacts": ncon, "blocks": int(cp["rows"].numel()),
                         "active_dofs": int(cp["active"].numel()), "ms": statistics.median(cs)},
            "feasible_step": {"alpha": feas[0], "halvings": feas[1], "limiting_tets": feas[2],
                              "ms": statistics.median(fs)}}


def vehicle(prec="fp64"):
    from .solver import DeviceSystem, HSCContext, HSCOptions
    from .systems import make_vehicle_system
    s = make_vehicle_system(seed=0)
    ds = DeviceSystem.from_system(s)
    ctx = HSCContext(HSCOptions(neumann_order=2, precision=prec, residual_replacement=0 if prec == "fp64" else 50))
    out = []
    for _ in range(2):
        _, st = ctx.solve(ds)
        out.append({"status": st["status"], "pcg_iterations": st["pcg_iterations"], "pcg_ms": st["pcg_ms"],
                    "total_ms": st["total_ms"]})
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--only", default="c1,c3,c4,c5")
    ap.add_argument("--out", default=None)
    ap.add_argument("--batch-count", type=int, default=64)
    ap.add_argument("--vehicle-precision", default="fp64", choices=("fp64", "fp32", "bf16"))
    a = ap.parse_args(argv)
    import torch
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    want = a.only.split(",")
    rep = {}
    if "assembly" in want:
        rep["assembly"] = assembly(); log(json.dumps({"assembly": rep["assembly"]}))
    if "vehicle" in want:
        rep["vehicle"] = vehicle(a.vehicle_precision); log(json.dumps({"vehicle": rep["vehicle"]}))
    if "c1" in want:
        rep["c1"] = c1(flush); log(json.dumps({"c1": rep["c1"]}))
    if "c3" in want:
        rep["c3"] = c3(flush, a.batch_count); log(json.dumps({"c3": {k: v for k, v in rep["c3"].items() if k != "autotune"}}))
    if "c4" in want:
        rep["c4"] = c4()
    if "c5" in want:
        rep["c5"] = c5(flush)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(rep, f, indent=1, default=float)
    return 0


if __name__ == "__main__":
    sys.exit(main())
