"""The replicated multi-GPU path of bench.py on CPU: two gloo ranks agree on
the slowest rank's time (the job time), seed their replicas differently, and
the reference arm runs on rank 0 only."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ws, r, local = bench.dist_setup()
    job = bench.max_over_ranks(10.0 + 5.0 * rank, dist)  # rank 1 is the slow one
    seed = bench.rank_seed(2, rank)
    seeds = [None] * world
    dist.all_gather_object(seeds, seed)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ws, r, local, job, seeds))


def test_two_gloo_ranks_take_the_max_and_distinct_seeds():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, (r, ws, r2, local, job, seeds) in enumerate(res):
        assert (r, ws, r2, local) == (rank, 2, rank, rank)
        assert job == 15.0
        assert len(set(seeds)) == 2


def test_reference_arm_is_rank0_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        cpu_sample_draws = 1000
        steps = 1
        warmup = 1

    assert bench.run_reference(A()) == 0
    assert capsys.readouterr().out == ""
