"""Sharding logic of alto_b200.shard on CPU: two gloo ranks each take their
contiguous equal-nnz range of the ALTO stream (shard_bounds), compute the
partial MTTKRP of that range (the oracle stands in for the GPU kernel here),
and the host all-reduce callback (the one the sharded CP-ALS calls) sums the
partial rows; the result equals the whole tensor's MTTKRP.  The callback's
max reduction and its error status are checked too."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_shard_bounds_follow_the_partition_rule():
    sys.path.insert(0, ROOT)
    from alto_b200.shard import shard_bounds
    assert shard_bounds(10, 3) == [(0, 4), (4, 8), (8, 10)]
    assert shard_bounds(2, 4) == [(0, 1), (1, 2), (2, 2), (2, 2)]
    assert shard_bounds(0, 2) == [(0, 0), (0, 0)]
    b = shard_bounds(1_000_003, 8)
    assert b[0][0] == 0 and b[-1][1] == 1_000_003
    assert all(b[k][1] == b[k + 1][0] for k in range(7))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _pext(words, mask):
    """Mode index of every key: the key bits under `mask` (lo, hi words),
    packed from the lowest (alto.hpp's pext)."""
    out = np.zeros(words.shape[0], np.uint64)
    k = 0
    for w in range(2):
        m = int(mask[w])
        for b in range(64):
            if m >> b & 1:
                out |= ((words[:, w] >> np.uint64(b)) & np.uint64(1)) << np.uint64(k)
                k += 1
    return out


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    from alto_b200 import F64, synth
    from alto_b200.shard import REDUCE_MAX, REDUCE_SUM, host_allreduce, shard_bounds
    from oracle.orc import Oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        o = Oracle()
        dims, cidx, vals = synth.uniform_distinct((300, 200, 150), 40_000, seed=9)
        ot = o.create(dims, cidx, vals, 8, 64)
        d = ot.dump()
        # the ALTO stream's nonzeros in order, with their coordinates
        scidx = np.stack([_pext(d["idx"], d["masks"][m]) for m in range(3)])
        svals = d["vals"]
        b, e = shard_bounds(svals.shape[0], world)[rank]
        red = host_allreduce()
        rank_r = 12
        errs = []
        for mode in range(3):
            U = synth.random_factors(dims, rank_r, seed=mode)
            want = [u.copy() for u in U]
            want[mode][:] = 0
            ot.mttkrp(mode, want, rank_r)
            part = [u.copy() for u in U]
            part[mode] = np.zeros_like(U[mode])
            o.mttkrp_coo(dims, scidx[:, b:e], svals[b:e], mode, part, rank_r)
            # the rows this shard touched lie inside its mode interval
            touched = np.nonzero(np.any(part[mode] != 0, axis=1))[0]
            if touched.size:
                lo, hi = scidx[mode, b:e].min(), scidx[mode, b:e].max()
                assert touched.min() >= lo and touched.max() <= hi
            rc = red(part[mode].ctypes.data, part[mode].size, F64, REDUCE_SUM, None, None)
            assert rc == 0
            errs.append(float(np.linalg.norm(part[mode] - want[mode]) / np.linalg.norm(want[mode])))
        # max reduction (the fit's) and float32 buffers
        x = np.array([1.0 + rank], np.float32)
        assert red(x.ctypes.data, 1, 1, REDUCE_MAX, None, None) == 0  # 1 = F32
        out.put((rank, errs, float(x[0]), (b, e)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_mttkrp_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, e0, m0, b0), (_, e1, m1, b1) = res
    assert b0[0] == 0 and b0[1] == b1[0] and b1[1] == 40_000
    for errs in (e0, e1):
        assert max(errs) < 1e-12, errs
    assert m0 == m1 == 2.0


def test_host_allreduce_reports_failure_without_a_group():
    """Outside an initialised process group the callback returns an error
    status instead of raising into the library."""
    sys.path.insert(0, ROOT)
    from alto_b200 import F64
    from alto_b200.shard import REDUCE_SUM, host_allreduce
    if dist.is_initialized():
        pytest.skip("a process group is already initialised")
    x = np.ones(4)
    assert host_allreduce()(x.ctypes.data, 4, F64, REDUCE_SUM, None, None) != 0
