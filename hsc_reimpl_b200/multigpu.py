"""Batched solves across the GPUs of one node: independent systems, no data-path collective.

One HSC solve does not shard (every SpMV would need a halo exchange and every
dot an all-reduce, several per iteration of a few microseconds of work), but a
batch of independent Newton systems does.  ``partition_systems`` assigns the
systems to ranks by greedy bin-packing on an estimate of their PCG work
(largest first onto the least-loaded rank; ties to the lower rank, so every
rank computes the same assignment); each rank then solves its share in one
persistent launch (``HSCContext.solve_batch``), and ``solve_batch_distributed``
gathers the per-system stats to rank 0 on the host -- the only communication.

    python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 \\
        -m hsc_reimpl_b200.multigpu --count 64
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np


def system_work(s) -> float:
    """Estimated PCG work of one system: its stored blocks (each read twice per SpMV: both
    triangles), its rows, and the low-rank rows of its coupled FEM nodes."""
    rows = np.asarray(s.rows)
    cols = np.asarray(s.cols)
    qo, qm, fo, fn = (int(v) for v in s.layout)
    coupled = 0
    if qm:
        qb0, qb1, fb0, fb1 = qo // 3, (qo + qm) // 3, fo // 3, (fo + fn) // 3
        in_q = lambda b: (b >= qb0) & (b < qb1)
        in_f = lambda b: (b >= fb0) & (b < fb1)
        cross = (in_q(rows) & in_f(cols)) | (in_f(rows) & in_q(cols))
        coupled = int(np.unique(np.where(in_f(rows[cross]), rows[cross], cols[cross])).size)
    return 2.0 * rows.size + float(s.nblock) + 10.0 * coupled


def partition_systems(works, world_size):
    """Rank of each system: greedy bin-packing, heaviest first onto the least-loaded rank."""
    works = [float(w) for w in works]
    order = sorted(range(len(works)), key=lambda i: (-works[i], i))
    load = [0.0] * world_size
    owner = [0] * len(works)
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += works[i]
    return owner, load


def solve_batch_distributed(systems, options=None, dist=None, use_graph=False, solve=None):
    """Solve this rank's share of `systems`; rank 0 returns every system's stats in input order
    (other ranks return None).  `solve(share) -> list of stats dicts` replaces the GPU solve
    (tests run the host logic on CPU ranks).  A share that raises is reported per system as
    {"status": the HSCError code or -1, "error": ...}; a rank that leaves without joining the
    gather makes the process group's timeout end rank 0's gather with an error."""
    ws = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    owner, _ = partition_systems([system_work(s) for s in systems], ws)
    mine = [i for i, o in enumerate(owner) if o == rank]
    try:
        if solve is None:
            stats = _solve_share([systems[i] for i in mine], options, use_graph)
        else:
            stats = solve([systems[i] for i in mine]) if mine else []
        if len(stats) != len(mine):
            raise RuntimeError(f"{len(stats)} stats for {len(mine)} systems")
    except Exception as e:
        # A rank whose share failed on the host (bad input, a CUDA error raised by the runtime)
        # still takes the gather below, so the other ranks never wait on it; its systems come
        # back to rank 0 marked with the error.
        code = getattr(e, "code", None)
        stats = [{"status": code if isinstance(code, int) and code > 0 else -1,
                  "error": f"{type(e).__name__}: {e}", "solved_on_rank": rank} for _ in mine]
    local = list(zip(mine, stats))
    if dist is None or ws == 1:
        gathered = [local]
    else:
        gathered = [None] * ws if rank == 0 else None
        dist.gather_object(local, gathered, dst=0)
    if rank != 0:
        return None
    out = [None] * len(systems)
    for part in gathered:
        for i, st in part:
            out[i] = st
    return out


def _solve_share(share, options, use_graph):
    """One launch for this rank's systems on its own stream."""
    if not share:
        return []
    from .solver import DeviceSystem, HSCContext
    import torch
    devs = [DeviceSystem.from_system(s) for s in share]
    ctx = HSCContext(options)
    try:
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            _, stats = ctx.solve_batch(devs, use_graph=use_graph, stream=stream, raise_on_error=False)
        stream.synchronize()
    finally:
        ctx.close()
    return stats


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    import torch
    import torch.distributed as dist
    from .solver import HSCOptions
    from .systems import make_batch_systems
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1:
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    systems = make_batch_systems(seed=args.seed, count=args.count)
    opts = HSCOptions(precision="fp32", residual_replacement=50, omega=0.6, max_rank=256)
    stats = solve_batch_distributed(systems, opts, dist if ws > 1 else None)
    if stats is not None:
        ok = [s for s in stats if s["status"] == 0]
        print(json.dumps({"systems": len(stats), "ranks": ws, "ok": len(ok),
                          "errors": sorted({s["error"] for s in stats if "error" in s}),
                          "max_full_relative_residual": max((s["full_relative_residual"] for s in ok),
                                                            default=None)}))
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
