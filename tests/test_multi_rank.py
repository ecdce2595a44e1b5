"""The multi-process pieces of bench.py on CPU: two gloo ranks (world size
2) reduce their step times to the max over ranks, and only rank 0 of the
reference arm does work."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as tdist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    tdist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    vals = bench.max_over_ranks([1.0 + rank, 10.0 - rank])
    r, w, local = bench.dist_env()
    out.put((rank, vals, (r, w, local)))
    tdist.barrier()
    tdist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, vals, env in got:
        assert vals == [2.0, 10.0]
        assert env == (rank, 2, rank)


def test_reference_arm_rank_nonzero_does_nothing(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    class A:
        workload = "wind64"; steps = 1; warmup = 0; cpu_sample_s = 1.0
    bench.run_reference(A())
    assert capsys.readouterr().out == ""
