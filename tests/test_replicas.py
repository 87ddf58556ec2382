"""Multi-GPU replicas (bench.py --gpus N): one independent system per rank,
no data-path collective, whole-job throughput over the slowest rank's time.
Run here as world_size-2 gloo ranks on CPU."""
import os
import socket

import pytest


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def replica_rank(rank, ws, port, q):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        local_ms = 100.0 * (rank + 1)               # rank 1 is the slower replica
        mx = bench.max_over_ranks(local_ms, dist, "cpu")
        from hsc_reimpl_b200.systems import make_cube_system
        s = make_cube_system(seed=rank)             # each rank its own system
        q.put((rank, mx, bench.replica_throughput(5, ws, mx), float(s.b[:8].sum())))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_max_over_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=replica_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs)
    out = sorted(q.get(timeout=5) for _ in range(2))
    assert [o[1] for o in out] == [200.0, 200.0]     # both ranks see the slowest time
    assert out[0][2] == pytest.approx(2 * 5 / 0.2)   # 10 solves in 0.2 s
    assert out[0][3] != out[1][3]                    # distinct systems per rank


def test_reference_arm_only_on_rank0(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        seed, warmup, steps = 0, 0, 1
    assert bench.run_reference(A()) is None
    assert capsys.readouterr().out == ""
