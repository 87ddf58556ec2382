#!/usr/bin/env python
"""HSC solves/s on the vehicle-scale synthetic Newton system, one B200.

Workload (the configuration the metric is quoted on): the vehicle scene's own
Tet4 tire mesh placed seven times (78,197 tets, 24,836 nodes, 74,508 FEM dofs,
149,513 stored upper FEM blocks) and 12 affine bodies (144 dofs), E=1e10
mounted / 1e6 ground tires, each tire's 39 rim-connection nodes stitched to
its rim body and 5-15 % tread contacts to the ground body, made by
``hsc_reimpl_b200.systems.make_reference_vehicle_system`` from a seed.  On this
mesh lambda_max(Dd^-1 D) = 3.89, so the Neumann step is omega = 0.5 (the
reference's 0.7 makes the order-2 polynomial indefinite here: PCG breaks down
at iteration 3).  A step is one full HSC solve through the public API: BCOO->BSR fill, Dd^-1,
coupling extraction, ACA, ABD inverse, reduced core, the persistent Schur PCG to a relative Schur
residual of 1e-6, back-substitution and the FP64 full-system residual check, which every timed
solve must pass at |b - H x| / |b| <= 1e-6.  The timed solves replay the solve's captured CUDA
graph (``HSCContext.solve_batch(use_graph=True)`` -> ``hsc_solve_batch``: one capture per pattern,
as a Newton loop with a fixed pattern would use it; ``--no-graph`` times ``hsc_solve``'s direct
launches); per-stage device times and the kernel count come from one direct solve after the timed
loop (a replay runs the kernels of its capture).  ``e2e`` goes through ``hsc_solve`` with host
buffers.

Modes: ``fp64`` (plain FP64 Neumann order 2, the bar) and ``fp32`` (FP32
bulk SpMV/Neumann with FP64 coupled-node blocks, FP64 residual replacement
every 50 iterations, FP64-verified result); ``block64`` / ``block32`` (the
block-local Woodbury preconditioner: a polynomial in w Dd^-1 D over each CTA's
part of the mesh plus the exact low-rank correction Y K Y^T, pipelined PCG with
two split-phase grid barriers per iteration; FP64 or FP32 matrix values, FP64
vectors and arithmetic; the polynomial is chosen per system by
``autotune.tune_block`` before any timing, ``block_tuning`` lists the candidates).  ``value`` is the flagship mode
(the fastest one that met the FP64-verified residual); every mode's numbers
are in ``modes``.  ``other_workloads`` repeats fp64/fp32 on the structured
annulus tires (``make_vehicle_system``) and the reference's C1 cube case.  ``e2e_repattern`` is ``e2e`` with a
different sparsity pattern every step (two seeds alternate), so the pattern
analysis is inside the timed region.

Multi-GPU: replicas only (one independent system per rank, no data-path
collective); value = solves of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "HSC solves/s & PCG iters to rel-res 1e-6: learned/FP32 vs plain FP64, 1 B200"
UNIT = "solves/s"
TARGET = 1e-6
# DRAM bytes per PCG iteration on the vehicle workload, per mode, from ncu
# captures (dram__bytes_read.sum / dram__bytes_write.sum of pcg_kernel) of one
# order-2 solve on the default (shared-memory-resident) path: FP64 24.84 MB read + 1.11 MB written over
# 204 iterations, FP32 32.19 MB + 0.50 MB over 245.  The learned modes run
# the same kernel with eight Schur-basis terms and have no capture of their own.
NCU_TRAFFIC_PER_ITER = {"fp64": (24.84e6 + 1.11e6) / 204, "fp32": (32.19e6 + 0.50e6) / 245,
                        # block_pcg_kernel<float>, one solve (Chebyshev degree 6): 20.09 MB read + 0.17 MB
                        # written over 68 iterations
                        "block32": (20.09e6 + 0.167e6) / 68}
BLOCK_TERMS = 4  # the block modes' default polynomial (Neumann, 4 terms) before the per-system tuning


def parse():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--modes", default="fp64,fp32,block64,block32,learned64,learned32")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-other", action="store_true", help="skip the annulus-tire workload lines")
    ap.add_argument("--no-graph", action="store_true",
                    help="time each solve as direct launches (hsc_solve) instead of the replay of its captured "
                         "CUDA graph (hsc_solve_batch with use_graph)")
    ap.add_argument("--block-poly", default=None,
                    help="the block modes' polynomial by tuner candidate name (e.g. 'cheb6 a=0.5 b=3.9'), "
                         "skipping the per-system tuning (profiling runs)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(ms, dist, device):
    """The slowest rank's device time (every rank takes this same collective)."""
    import torch
    el = torch.tensor([ms], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(el, op=dist.ReduceOp.MAX)
    return float(el.item())


def replica_throughput(steps, ws, max_ms):
    """Whole-job solves/s: every rank solved `steps` systems within `max_ms`."""
    return ws * steps / (max_ms / 1000.0)


OMEGA = 0.5


def make_workload(seed):
    from hsc_reimpl_b200.systems import make_reference_vehicle_system
    return make_reference_vehicle_system(seed=seed)


def workload_config(s):
    m = s.meta
    return {"workload": "vehicle_tire_tet4_78k_tets", "mesh": "reproduction/vehicle_research/prepared/tire_tet4.npz "
            "x 7 (scene_manifest placements)", "tires": m["tires"], "tets": m["tets"], "nodes": m["nodes"],
            "fem_dofs": s.layout[3], "abd_dofs": s.layout[1], "nnzb_one_triangle": m["nnzb"],
            "neumann_order": 2, "omega": OMEGA, "schur_tol": 1e-6, "full_residual_target": TARGET,
            "abd_inverse": "exact FP64 Cholesky", "aca": "fixed rank cap 128, roundoff guard",
            "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas", "seed": m["seed"]}


# ----------------------------------------------------------------------------
# CPU side: the oracle port of the reference algorithm (reference arm and the
# cpu_baseline leg are the only users of oracle/ in this file)
# ----------------------------------------------------------------------------
def cpu_solve_once(s):
    """One FP64 solve with the oracle port, on one host thread: SciPy's CSR product is
    single-threaded, and the BLAS of the small dense parts is held to one thread too, so
    ``cores`` = 1 is the thread count that actually ran."""
    from threadpoolctl import threadpool_limits
    from oracle import hsc_oracle as O
    with threadpool_limits(limits=1):
        x, st, _ = O.hsc_solve(s.H, s.layout, s.b, order=2, omega=OMEGA, tol=1e-6, max_iter=20000,
                               abd_inverse="exact", max_rank=128)
    return x, st


def cpu_baseline(s, budget_s=12.0):
    t0 = time.perf_counter()
    times, iters = [], []
    cpu_solve_once(s)  # warm-up
    while time.perf_counter() - t0 < budget_s and len(times) < 8:
        t = time.perf_counter()
        _, st = cpu_solve_once(s)
        times.append(time.perf_counter() - t)
        iters.append(st["pcg_iterations"])
    med = statistics.median(times)
    return {"value": 1.0 / med, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{len(times)} full FP64 solves of the vehicle system (median {med:.3f} s, "
                      f"{iters[0]} PCG iterations) with the NumPy/SciPy oracle port on one host thread "
                      f"({os.cpu_count()} cores on the host), after 1 warm-up"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    s = make_workload(args.seed)
    for _ in range(args.warmup):
        cpu_solve_once(s)
    t = time.perf_counter()
    full = []
    for _ in range(args.steps):
        x, st = cpu_solve_once(s)
        full.append(st["full_relative_residual"])
    el = time.perf_counter() - t
    v = args.steps / el
    cores = 1
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(s),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} full FP64 solves of the vehicle system with the "
                                       "NumPy/SciPy restatement of the reference algorithm on one host thread "
                                       "(SciPy's CSR product is single-threaded)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "max_full_relative_residual": max(full)}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
# GPU side
# ----------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def survey_bytes_per_iteration(s, a, k, order, sb):
    """Algorithmic bytes of one Schur PCG iteration at Neumann order r, the formula the
    hot-path scope fixes: r SpMVs over the STORED (one-triangle) FEM blocks,
    nnzb (9 s + 4) + 4 (n + 1) + 2 N s each; the low-rank apply (2 a k + k^2) s; the
    vector passes: update 4N, Jacobi r (9n + 2N), axpby 6 (r - 1) N, three dots 2N each,
    all times s (s = 8 FP64, 4 FP32)."""
    qo, qm, fo, fn = s.layout
    n, N = fn // 3, fn
    fb0 = fo // 3
    nnzb = int(((s.rows >= fb0) & (s.cols >= fb0)).sum())
    spmv = nnzb * (9 * sb + 4) + 4 * (n + 1) + 2 * N * sb
    lowrank = (2 * a * k + k * k) * sb
    vec = (4 * N + order * (9 * n + 2 * N) + 6 * (order - 1) * N + 3 * 2 * N) * sb
    return order * spmv + lowrank + vec


def measure_l2_copy_gbs(dev):
    """Copy bandwidth with both buffers L2-resident (2 x 24 MiB), read + write bytes over the
    best of 5 bursts of 50 copies (CUDA events): the denominator of the L2 fraction."""
    import torch
    a = torch.empty(6 * 1024 * 1024, dtype=torch.float32, device=dev).normal_()
    b = torch.empty_like(a)
    for _ in range(20):
        b.copy_(a)
    best = 1e30
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(5):
        torch.cuda.synchronize()
        e0.record()
        for _ in range(50):
            b.copy_(a)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 50)
    return 2 * a.numel() * 4 / (best / 1000.0) / 1e9


def time_modes(args, s, ds, ctx_holder, mode_opts, flush, dist, dev, lib, sample_clocks=True, steps=None):
    import numpy as np
    import torch
    import scipy.sparse.linalg as spla
    ws = dist.get_world_size() if dist is not None else 1
    steps = steps or args.steps
    x_direct = spla.splu(s.H.tocsc()).solve(s.b)
    modes, clocks, launches = {}, None, None
    for mi, (mode, opt) in enumerate(mode_opts.items()):
        if ctx_holder[0] is None:
            from hsc_reimpl_b200.solver import HSCContext
            ctx_holder[0] = HSCContext(opt)
        ctx = ctx_holder[0]
        if ctx_holder[1] is not None:
            ctx.set_learned_model(ctx_holder[1])
        ctx.set_options(opt)
        x = torch.empty_like(ds.b)
        graph = not args.no_graph
        stream = torch.cuda.Stream()

        def one_solve():
            if graph:  # the captured graph of this pattern, replayed (captured in the first warm-up)
                xs_, sts = ctx.solve_batch([ds], xs=[x], use_graph=True, stream=stream, raise_on_error=False)
                return sts[0]
            return ctx.solve(ds, x=x, stream=stream, raise_on_error=False)[1]

        for _ in range(args.warmup):
            one_solve()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        sampler = ClockSampler(dev.index) if (mi == 0 and sample_clocks) else None
        if sampler:
            sampler.start()
        total_ms, stats_all = 0.0, []
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            ev0.record(stream)
            st = one_solve()
            ev1.record(stream)
            torch.cuda.synchronize()
            total_ms += ev0.elapsed_time(ev1)
            stats_all.append(st)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        if sampler:
            clocks = sampler.stop()
        # the per-stage device times and the kernel count of one solve come from a direct (uncaptured)
        # solve after the timed loop: a replay runs the same kernels as its capture
        l0 = lib.hsc_kernel_launches()
        st_plain = ctx.solve(ds, x=x, stream=stream, raise_on_error=False)[1]
        torch.cuda.synchronize()
        per_solve = lib.hsc_kernel_launches() - l0
        pcg_ms = st_plain["pcg_ms"] * steps
        if mi == 0:
            launches = per_solve * steps
        total_ms = max_over_ranks(total_ms, dist, dev)
        last = stats_all[-1]
        xs = x.cpu().numpy()
        ok = all(t["status"] == 0 and t["full_relative_residual"] <= TARGET for t in stats_all)
        iters = last["pcg_iterations"]
        sb = 8 if mode.endswith("64") else 4
        # the block modes apply the FEM blocks BLOCK_TERMS times per iteration (the operator and the
        # polynomial's local terms), counted as full SpMVs over the stored blocks
        bytes_iter = survey_bytes_per_iteration(s, last["active_fem_dofs"], last["rank"],
                                                len(opt.poly_weights) if mode.startswith("block") else 2, sb)
        pcg_launch_ms = pcg_ms / steps
        modes[mode] = {
            "solves_per_s": replica_throughput(steps, ws, total_ms),
            "ms_per_solve": total_ms / steps,
            "pcg_iterations": iters,
            "full_relative_residual": max(t["full_relative_residual"] for t in stats_all),
            "schur_relative_residual": last["schur_relative_residual"],
            "error_vs_direct": float(np.linalg.norm(xs - x_direct) / np.linalg.norm(x_direct)),
            "met_target": ok, "status": last["status_name"] if "status_name" in last else last["status"],
            "fallback": last.get("fallback", 0),
            "rank": last["rank"], "active_fem_dofs": last["active_fem_dofs"],
            "residual_replacements": last["residual_replacements"],
            "stage_ms": [round(v, 4) for v in st_plain["stage_ms"]],
            "setup_ms": st_plain["setup_ms"], "pcg_ms": pcg_launch_ms, "graph_replay": graph,
            "kernel_launches_per_solve": per_solve,
            "pcg_us_per_iteration": 1000.0 * pcg_launch_ms / max(1, iters),
            "pcg_bytes_per_iteration": bytes_iter,
        }
    return modes, clocks, launches


def timed_e2e(args, ctx, opt, systems_dev, flush, dist, dev, repattern):
    """Solves through the public API from pinned host buffers: H2D of the matrix values and b
    (and of rows/cols when ``repattern``: two systems of different sparsity alternate, so every
    step pays the pattern analysis), the solve, D2H of x."""
    import torch
    from dataclasses import replace
    from hsc_reimpl_b200.solver import DeviceSystem
    ws = dist.get_world_size() if dist is not None else 1
    # a fixed pattern replays hsc_solve's captured graph (graph_replay, on a non-default stream); an
    # alternating pattern is analysed again every step, so it launches directly
    graph = not repattern and not args.no_graph
    ctx.set_options(replace(opt, graph_replay=graph))
    stream = torch.cuda.Stream()
    host = []
    for ds in systems_dev:
        host.append(dict(rows=ds.rows.cpu().pin_memory(), cols=ds.cols.cpu().pin_memory(),
                         vals=ds.values.cpu().pin_memory(), b=ds.b.cpu().pin_memory()))
    nmax = max(h["rows"].numel() for h in host)
    Nmax = max(h["b"].numel() for h in host)
    # one index buffer pair per pattern: the solver keys its cached analysis on these pointers,
    # so alternating patterns re-run the analysis up front every step
    idx_d = [(torch.empty(nmax, dtype=torch.int32, device=dev), torch.empty(nmax, dtype=torch.int32, device=dev))
             for _ in host]
    vals_d = torch.empty((nmax, 9), dtype=torch.float64, device=dev)
    b_d = torch.empty(Nmax, dtype=torch.float64, device=dev)
    x_d = torch.empty(Nmax, dtype=torch.float64, device=dev)
    x_h = torch.empty(Nmax, dtype=torch.float64).pin_memory()
    h2d = d2h = 0
    fails = 0

    def step(i):
        with torch.cuda.stream(stream):  # the copies, the solve and the read-back in one stream's order
            step_on_stream(i)

    def step_on_stream(i):
        nonlocal h2d, d2h, fails
        h = host[i % len(host)]
        src = systems_dev[i % len(host)]
        nz, N = h["rows"].numel(), h["b"].numel()
        rows_d, cols_d = idx_d[i % len(host)]
        if repattern:
            rows_d[:nz].copy_(h["rows"], non_blocking=True)
            cols_d[:nz].copy_(h["cols"], non_blocking=True)
        vals_d[:nz].copy_(h["vals"], non_blocking=True)
        b_d[:N].copy_(h["b"], non_blocking=True)
        ds2 = DeviceSystem(rows_d[:nz] if repattern else src.rows, cols_d[:nz] if repattern else src.cols,
                           vals_d[:nz], src.nblock, src.layout, b_d[:N])
        _, st = ctx.solve(ds2, x=x_d[:N], stream=stream, raise_on_error=False)
        fails += st["status"] != 0
        x_h[:N].copy_(x_d[:N], non_blocking=True)
        h2d = (2 * nz * 4 if repattern else 0) + nz * 72 + N * 8
        d2h = N * 8

    for i in range(max(args.warmup, 2)):
        step(i)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    tot = 0.0
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    fails = 0
    for i in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ev0.record(stream)
        step(i)
        ev1.record(stream)
        torch.cuda.synchronize()
        tot += ev0.elapsed_time(ev1)
    tot = max_over_ranks(tot, dist, dev)
    return {"value": replica_throughput(args.steps, ws, tot), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "graph_replay": graph,
            "d2h_bytes_per_step": int(d2h), "failed_solves": int(fails)}


def run_gpu(args):
    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    from hsc_reimpl_b200 import _lib
    from hsc_reimpl_b200.solver import HSCOptions, DeviceSystem
    from hsc_reimpl_b200.systems import make_vehicle_system

    s = make_workload(args.seed + rank)
    dev = torch.device("cuda", local)
    ds = DeviceSystem.from_system(s, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2
    lib = _lib.load()
    base = dict(neumann_order=2, omega=OMEGA, tol=1e-6, abd_inverse="exact")
    mode_opts = {
        "fp64": HSCOptions(precision="fp64", **base),
        "fp32": HSCOptions(precision="fp32", residual_replacement=50, **base),
        "block64": HSCOptions(block=True, poly_weights=(1.0,) * BLOCK_TERMS, omega=OMEGA, tol=1e-6,
                              abd_inverse="exact", precision="fp64"),
        "block32": HSCOptions(block=True, poly_weights=(1.0,) * BLOCK_TERMS, omega=OMEGA, tol=1e-6,
                              abd_inverse="exact", precision="fp32"),
        "learned64": HSCOptions(learned=True, omega=OMEGA, tol=1e-6, abd_inverse="exact", precision="fp64"),
        "learned32": HSCOptions(learned=True, omega=OMEGA, tol=1e-6, abd_inverse="exact", precision="fp32",
                                residual_replacement=50),
    }
    # the block modes' polynomial: tuned once on this system, outside every timed region (a Newton
    # loop tunes once per system family and reuses the choice)
    tuning = None
    if args.block_poly is not None:
        from dataclasses import replace
        from hsc_reimpl_b200.autotune import block_candidates
        named = {c[0]: c for c in block_candidates()}
        if args.block_poly not in named:
            raise SystemExit(f"--block-poly: unknown candidate {args.block_poly!r}; one of {sorted(named)}")
        _, w, om = named[args.block_poly]
        mode_opts["block32"] = replace(mode_opts["block32"], poly_weights=tuple(w), omega=om)
        mode_opts["block64"] = replace(mode_opts["block64"], poly_weights=tuple(w), omega=om)
        tuning = {"chosen": args.block_poly, "weights": list(w), "omega": om, "candidates": None}
    elif any(m.startswith("block") for m in args.modes.split(",")):
        from dataclasses import replace
        from hsc_reimpl_b200.autotune import tune_block
        best, table = tune_block(ds, base=mode_opts["block32"], reps=3)
        if best is not None:
            mode_opts["block32"] = best
            mode_opts["block64"] = replace(best, precision="fp64")
            wb = [round(v, 6) for v in best.poly_weights]
            chosen = next(r for r in table if r["ok"] and r["omega"] == best.omega and r["weights"] == wb)
            tuning = {"chosen": chosen["name"], "weights": chosen["weights"], "omega": chosen["omega"],
                      "candidates": [{k: r[k] for k in ("name", "ms", "iterations", "ok")} for r in table]}
    from hsc_reimpl_b200 import learned as L
    model = L.load_model()[0] if L.MODEL_PATH.exists() else None
    want = {m: o for m, o in mode_opts.items() if m in args.modes.split(",") and (model is not None or "learned" not in m)}
    ctx_holder = [None, model]
    modes, clocks, launches = time_modes(args, s, ds, ctx_holder, want, flush, dist, dev, lib)
    ctx = ctx_holder[0]
    # flagship: fastest mode that met the FP64-verified target
    ok_modes = [m for m in modes if modes[m]["met_target"]]
    flag = max(ok_modes, key=lambda m: modes[m]["solves_per_s"]) if ok_modes else "fp64"
    F = modes[flag]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    alg_bytes = F["pcg_bytes_per_iteration"] * F["pcg_iterations"]
    achieved = alg_bytes / (F["pcg_ms"] / 1000.0) / 1e9
    l2_gbs = measure_l2_copy_gbs(dev)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (NCU_TRAFFIC_PER_ITER[flag] * F["pcg_iterations"]) if flag in NCU_TRAFFIC_PER_ITER else None,
                "kernel": ("hsc::block_pcg_kernel (persistent pipelined Schur PCG, one CTA per mesh part)"
                           if flag.startswith("block") else "hsc::pcg_kernel (persistent Schur PCG)")
                          + ", one launch per solve",
                "bytes": "per iteration: r SpMVs over the stored one-triangle FEM blocks "
                         "nnzb (9 s + 4) + 4 (n + 1) + 2 N s, low-rank (2 a k + k^2) s, vector passes "
                         "(4N + r (9n + 2N) + 6 (r - 1) N + 6N) s; times the launch's iterations; r = 2 for the "
                         "Neumann modes, r = the polynomial's terms for the block modes (the operator and terms - 1 "
                         "local products)",
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650 GB/s",
                "l2": {"achieved": achieved, "peak": l2_gbs, "unit": "GB/s", "frac": achieved / l2_gbs,
                       "peak_source": "measured in this run: torch copy between two L2-resident 24 MiB buffers"},
                "note": "the vehicle matrix stays in L2 and the CTAs' shared memory across iterations, so "
                        "HBM is not the binding resource; the l2 entry puts the same bytes against L2"}
    e2e = e2e_rep = None
    if not args.no_e2e:
        e2e = timed_e2e(args, ctx, want[flag], [ds], flush, dist, dev, repattern=False)
        e2e["mode"] = flag
        s_alt = make_workload(args.seed + rank + 1000)
        ds_alt = DeviceSystem.from_system(s_alt, device=dev)
        e2e_rep = timed_e2e(args, ctx, want[flag], [ds, ds_alt], flush, dist, dev, repattern=True)
        e2e_rep["mode"] = flag
        e2e_rep["note"] = "two seeds with different contact sets alternate; rows/cols copied every step"
    other = None
    if not args.no_other:
        sa = make_vehicle_system(seed=args.seed + rank)
        dsa = DeviceSystem.from_system(sa, device=dev)
        oo = {"fp64": HSCOptions(precision="fp64", neumann_order=2, omega=0.7, tol=1e-6, abd_inverse="exact"),
              "fp32": HSCOptions(precision="fp32", neumann_order=2, omega=0.7, tol=1e-6, abd_inverse="exact",
                                 residual_replacement=50)}
        om, _, _ = time_modes(args, sa, dsa, ctx_holder, oo, flush, dist, dev, lib, sample_clocks=False,
                              steps=min(args.steps, 10))
        other = {"vehicle_annulus_78k_tets": {"nodes": sa.meta["nodes"], "fem_dofs": sa.layout[3], "omega": 0.7,
                                              "modes": om}}
        # C1, the reference's cube case (1,331 nodes, FP64 Neumann order 2): 20 timed solves, the error
        # against the FP64 direct solve
        from hsc_reimpl_b200 import bench_configs
        other["cube_c1"] = bench_configs.c1(flush)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(s)
    if rank == 0:
        line = {"metric": METRIC, "value": F["solves_per_s"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": F["ms_per_solve"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                # arithmetic type: the block modes compute in FP64 over FP32 or FP64 matrix planes
                "dtype": "f64" if flag in ("fp64", "block64", "block32") else "f32",
                "matrix_storage": "f32" if flag.endswith("32") else "f64",
                "data": "synthetic (seeded Newton system on the vehicle scene's tire mesh; no public dataset)",
                "config": workload_config(s), "mode": flag, "pcg_iterations": F["pcg_iterations"],
                "full_relative_residual": F["full_relative_residual"], "error_vs_direct": F["error_vs_direct"],
                "modes": modes, "clocks": clocks, "e2e": e2e, "e2e_repattern": e2e_rep, "gpu_launches": launches,
                "roofline": roofline, "cpu_baseline": cpu, "other_workloads": other, "block_tuning": tuning}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    main()
