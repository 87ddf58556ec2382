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


# ---------------------------------------------------------------------------
# Per-system polynomial of the block preconditioner (HSC_PRECOND_BLOCK)
# ---------------------------------------------------------------------------
def chebyshev_weights(n, a, b, omega):
    """Weights w_0..w_{n-1} of the block polynomial L = sum_k w_k (I - omega B)^k omega Dd^-1,
    B = Dd^-1 D_loc, whose residual polynomial 1 - lambda p(lambda) is the degree-n Chebyshev
    polynomial of [a, b] normalised to 1 at lambda = 0: r(lambda) = T_n((b + a - 2 lambda) / (b - a))
    / T_n((b + a) / (b - a)).  With mu = 1 - omega lambda, sum_k w_k mu^k = (1 - R(mu)) / (1 - mu) for
    R(mu) = r((1 - mu) / omega), a polynomial of degree n - 1 since R(1) = r(0) = 1.  All-ones weights
    are the Neumann series, R(mu) = mu^n."""
    from numpy.polynomial import chebyshev as Ch, polynomial as Po
    tn = Ch.cheb2poly([0] * n + [1])
    beta = 2.0 / (omega * (b - a))
    alpha = (b + a - 2.0 / omega) / (b - a)
    R, xp = np.zeros(1), np.array([1.0])
    for c in tn:                      # T_n(alpha + beta mu) in powers of mu
        R = Po.polyadd(R, c * xp)
        xp = Po.polymul(xp, [alpha, beta])
    R = R / Ch.chebval((b + a) / (b - a), [0] * n + [1])
    q, rem = Po.polydiv(Po.polysub([1.0], R), [1.0, -1.0])
    if np.max(np.abs(rem)) > 1e-8 * max(1.0, float(np.max(np.abs(R)))):
        raise ValueError("residual polynomial is not 1 at the origin")
    q = np.concatenate([q, np.zeros(max(0, n - len(q)))])[:n]
    return [float(v) for v in q]


def block_candidates(lam_max=3.9):
    """(name, weights, omega) of the polynomials the block tuner times: Neumann series of degree 3-8
    (odd degrees also at a larger omega: their residual polynomial (1 - omega lambda)^n stays below 1
    for any omega lambda > 0, so the preconditioner stays SPD) and Chebyshev weights of degree 5-6
    on [a, lam_max]."""
    out = [(f"neumann{n} omega=0.5", [1.0] * n, 0.5) for n in (3, 4, 5, 6, 8)]
    out += [(f"neumann{n} omega={om}", [1.0] * n, om) for n in (3, 5) for om in (0.6, 0.7)]
    out += [(f"cheb{n} a={a} b={lam_max}", chebyshev_weights(n, a, lam_max, 0.5), 0.5)
            for n in (5, 6) for a in (0.4, 0.5)]
    return out


def time_solve(ctx, ds, reps=3, warmup=1):
    """Median milliseconds of one solve (CUDA events) and the stats of the last one."""
    import torch
    x = torch.empty_like(ds.b)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st = None
    for _ in range(warmup):
        _, st = ctx.solve(ds, x=x, raise_on_error=False)
    times = []
    for _ in range(reps):
        ev0.record()
        _, st = ctx.solve(ds, x=x, raise_on_error=False)
        ev1.record()
        ev1.synchronize()
        times.append(ev0.elapsed_time(ev1))
    return float(np.median(times)), st


def tune_block(system, base: HSCOptions | None = None, candidates=None, target=1e-6, reps=3, log=None, tie=0.01):
    """Times every candidate polynomial of the block preconditioner on this system and returns
    (options of the fastest one whose solve met ``target`` on the FP64-verified full residual,
    table of every candidate).  Candidates within ``tie`` (relative) of the fastest time count as
    tied and the one with the fewest PCG iterations wins, so timing noise does not flip the choice
    between near-equal polynomials.  A tuned polynomial is a property of the system family (mesh,
    materials, coupling), so a Newton loop tunes once and reuses it."""
    base = base or HSCOptions(block=True, precision="fp32", tol=1e-6, abd_inverse="exact")
    ds = system if isinstance(system, DeviceSystem) else DeviceSystem.from_system(system)
    cands = candidates if candidates is not None else block_candidates()
    table, passed = [], []
    for name, w, om in cands:
        opt = replace(base, block=True, poly_weights=tuple(w), omega=om, fallback_on_stall=False)
        ctx = HSCContext(opt)
        ms, st = time_solve(ctx, ds, reps=reps)
        ok = st["status"] == 0 and st["full_relative_residual"] <= target
        rec = dict(name=name, omega=om, weights=[round(v, 6) for v in w], ms=ms, ok=bool(ok),
                   iterations=st["pcg_iterations"], full_relative_residual=st["full_relative_residual"])
        table.append(rec)
        if log:
            log(json.dumps(rec))
        if ok:
            passed.append((ms, st["pcg_iterations"], len(passed), opt))
        ctx.close()
    if not passed:
        return None, table
    fastest = min(p[0] for p in passed)
    tied = [p for p in passed if p[0] <= fastest * (1.0 + tie)]
    return min(tied, key=lambda p: (p[1], p[0], p[2]))[3], table
