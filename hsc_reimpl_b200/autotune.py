"""Autotuner of the batched HSC solve: SpMV tile width and ACA rank cap.

For a list of systems solved together in one persistent launch
(``hsc_solve_batch``, optionally replayed as a CUDA graph) it times every
candidate (``threads_per_row`` -> slices of 32 blocks a warp loads per round
trip, ``max_rank`` -> ACA rank cap) with CUDA events and keeps the fastest one
whose every system still meets the FP64-verified full-system residual target.
A rank cap below what the coupling needs leaves an ACA error that no PCG
tolerance can remove -- and can make the approximate Schur complement
indefinite, which PCG reports as a breakdown -- so the status and residual
tests are what bound the rank from below; with 12 bodies the coupling rank
reaches 139, so the sweep ends at a cap (256) at or above every coupling rank.  The default relaxation is
omega = 0.6: block-Jacobi-scaled cube and torus operators reach
lambda_max(Dd^-1 D) = 2.9, where the order-2 series needs omega < 2 / 2.9.
"""
from __future__ import annotations

import itertools
import json
from dataclasses import replace

import numpy as np

from .solver import DeviceSystem, HSCContext, HSCOptions

TILES = (2, 4, 8)
RANKS = (4, 8, 16, 32, 64, 128, 256)


def time_batch(ctx, systems, xs, reps=3, warmup=1, use_graph=True):
    """Median milliseconds of one batched solve and the per-system stats of the last one."""
    import torch
    stream = torch.cuda.Stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        stats = None
        for _ in range(warmup):
            _, stats = ctx.solve_batch(systems, xs=xs, use_graph=use_graph, stream=stream, raise_on_error=False)
        times = []
        for _ in range(reps):
            ev0.record(stream)
            _, stats = ctx.solve_batch(systems, xs=xs, use_graph=use_graph, stream=stream, raise_on_error=False)
            ev1.record(stream)
            ev1.synchronize()
            times.append(ev0.elapsed_time(ev1))
    return float(np.median(times)), stats


def autotune(systems, base: HSCOptions | None = None, tiles=TILES, ranks=RANKS, target=1e-6, reps=3,
             use_graph=True, log=None):
    """Returns (best options, table of every candidate)."""
    import torch
    base = base or HSCOptions(precision="fp32", residual_replacement=50, omega=0.6)
    devs = [s if isinstance(s, DeviceSystem) else DeviceSystem.from_system(s) for s in systems]
    xs = [torch.empty_like(d.b) for d in devs]
    table = []
    best = None
    for tpr, rank in itertools.product(tiles, ranks):
        opt = replace(base, threads_per_row=tpr, max_rank=rank)
        ctx = HSCContext(opt)
        ms, stats = time_batch(ctx, devs, xs, reps=reps, use_graph=use_graph)
        full = max(s["full_relative_residual"] for s in stats)
        ok = all(s["status"] == 0 for s in stats) and full <= target
        rec = dict(threads_per_row=tpr, max_rank=rank, ms=ms, ok=bool(ok), max_full_relative_residual=full,
                   max_iterations=max(s["pcg_iterations"] for s in stats),
                   mean_iterations=float(np.mean([s["pcg_iterations"] for s in stats])))
        table.append(rec)
        if log:
            log(json.dumps(rec))
        if ok and (best is None or ms < best[1]):
            best = (opt, ms)
        ctx.close()
    return (best[0] if best else None), table
