"""Batches across GPUs (hsc_reimpl_b200/multigpu.py): greedy bin-packing of
independent systems by estimated work, one launch per rank, stats gathered to
rank 0 on the host.  The host logic runs here as world_size-2 gloo ranks."""
import os
import socket

import numpy as np
import pytest

from hsc_reimpl_b200 import multigpu as MG


def test_partition_is_balanced_deterministic_and_complete():
    rng = np.random.default_rng(0)
    works = rng.lognormal(10, 1, 64)
    owner, load = MG.partition_systems(works, 4)
    assert sorted(set(owner)) == [0, 1, 2, 3]
    assert np.isclose(sum(load), works.sum())
    # greedy bound: no rank exceeds the mean by more than the largest item
    assert max(load) <= works.sum() / 4 + works.max()
    assert MG.partition_systems(works, 4)[0] == owner             # every rank computes the same
    assert MG.partition_systems(works, 1)[0] == [0] * 64


def test_system_work_counts_blocks_rows_and_coupled_nodes(cube_system):
    s = cube_system
    w = MG.system_work(s)
    assert w > 2 * s.rows.size + s.nblock                           # the coupled bottom nodes add work


def gather_rank(rank, ws, port, q):
    import torch.distributed as dist
    from hsc_reimpl_b200 import multigpu as MG2
    from hsc_reimpl_b200.systems import make_cube_system
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        systems = [make_cube_system(seed=i, n=3 + i % 3) for i in range(5)]
        tag = lambda share: [{"status": 0, "rank": rank, "n": s.N} for s in share]
        out = MG2.solve_batch_distributed(systems, dist=dist, solve=tag)
        q.put((rank, out))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_every_system_in_order():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=gather_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs)
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res[1] is None
    out = res[0]
    from hsc_reimpl_b200.systems import make_cube_system
    Ns = [make_cube_system(seed=i, n=3 + i % 3).N for i in range(5)]
    assert [o["n"] for o in out] == Ns                               # input order restored
    assert {o["rank"] for o in out} == {0, 1}                        # both ranks solved a share


def failure_rank(rank, ws, port, q, mode):
    import datetime
    import torch.distributed as dist
    from hsc_reimpl_b200 import multigpu as MG2
    from hsc_reimpl_b200._lib import HSCError, HSC_ERR_NONSPD
    from hsc_reimpl_b200.systems import make_cube_system
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=10))
    systems = [make_cube_system(seed=i, n=3 + i % 3) for i in range(2)]

    def solve(share):
        if mode == "raise" and rank == 1:
            raise HSCError(HSC_ERR_NONSPD, "planted on rank 1")
        return [{"status": 0, "solved_on_rank": rank} for _ in share]

    try:
        if mode == "leave" and rank == 1:
            q.put((rank, "left"))
            q.close()
            q.join_thread()                                      # flushed before the hard exit
            os._exit(0)                                          # leaves before the gather
        try:
            out = MG2.solve_batch_distributed(systems, dist=dist, solve=solve)
        except RuntimeError as e:                                # the peer is gone: the gather ends
            out = ("gather failed", str(e)[:200])
        q.put((rank, out))
    finally:
        if mode != "leave":
            dist.destroy_process_group()


def run_ranks(ws, mode):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=failure_rank, args=(r, ws, port, q, mode)) for r in range(ws)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=240) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
    return res, [p.exitcode for p in procs]


def test_more_ranks_than_systems():
    res, codes = run_ranks(3, "ok")
    assert codes == [0, 0, 0]
    assert [o["status"] for o in res[0]] == [0, 0] and res[1] is None and res[2] is None
    assert len({o["solved_on_rank"] for o in res[0]}) == 2        # the third rank had nothing to do


def test_a_share_that_raises_is_reported_and_no_rank_waits():
    from hsc_reimpl_b200._lib import HSC_ERR_NONSPD
    res, codes = run_ranks(2, "raise")
    assert codes == [0, 0]
    out = res[0]
    bad = [o for o in out if "error" in o]
    assert len(bad) == 1 and bad[0]["status"] == HSC_ERR_NONSPD and bad[0]["solved_on_rank"] == 1
    assert "planted on rank 1" in bad[0]["error"]
    assert [o["status"] for o in out if "error" not in o] == [0]


def test_a_rank_that_leaves_ends_the_gather_with_an_error():
    res, codes = run_ranks(2, "leave")
    assert res[1] == "left"
    assert isinstance(res[0], tuple) and res[0][0] == "gather failed", res[0]
    assert codes[0] == 0


@pytest.mark.gpu
def test_single_rank_batch_on_the_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hsc_reimpl_b200.solver import HSCOptions
    from hsc_reimpl_b200.systems import make_cube_system
    systems = [make_cube_system(seed=i, n=4 + i) for i in range(3)]
    stats = MG.solve_batch_distributed(systems, HSCOptions(omega=2 / 3))
    assert len(stats) == 3 and all(s["status"] == 0 and s["full_relative_residual"] <= 1e-6 for s in stats), stats
