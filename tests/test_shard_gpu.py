"""Sharded MTTKRP and CP-ALS (altob_slice, altob_cpd_als_sharded) on one GPU,
with two host threads standing in for two GPUs: each thread owns one slice
of the tensor and its own stream, and the all-reduce callback exchanges the
partial results on the host side (a thread waits for the other's buffer,
then thread 0 reduces both).  No kernel waits for another.  The sharded
results must equal the single-tensor ones: MTTKRP FP64 within 1e-12; CP-ALS
fits within 1e-9 (FP64) and 1e-4 (FP32), factors within 1e-7 (FP64)."""
import threading

import numpy as np
import pytest

import alto_b200 as ab
from alto_b200 import synth
from alto_b200.shard import ALLREDUCE_FN, REDUCE_MAX, ShardedTensor, _DeviceView, _TYPESTR
from conftest import rel_fro

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


class ThreadReducer:
    def __init__(self, world):
        self.bar = threading.Barrier(world)
        self.bufs = [None] * world
        self.fns = [ALLREDUCE_FN(self._make(r)) for r in range(world)]

    def _make(self, rank):
        def fn(buf, count, dtype, op, stream, user):
            try:
                t = torch.as_tensor(_DeviceView(buf, count, _TYPESTR[dtype]), device="cuda")
                (torch.cuda.ExternalStream(int(stream)) if stream else torch.cuda.default_stream()).synchronize()
                self.bufs[rank] = t
                self.bar.wait(timeout=120)
                if rank == 0:
                    acc = self.bufs[0].clone()
                    for b in self.bufs[1:]:
                        acc = torch.maximum(acc, b) if op == REDUCE_MAX else acc + b
                    for b in self.bufs:
                        b.copy_(acc)
                    torch.cuda.synchronize()
                self.bar.wait(timeout=120)
                return 0
            except Exception:  # noqa: BLE001
                self.bar.abort()
                return 3
        return fn


def _run_threads(fn, world):
    out = [None] * world
    err = []

    def body(r):
        try:
            out[r] = fn(r)
        except Exception as e:  # noqa: BLE001
            err.append(e)

    th = [threading.Thread(target=body, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    if err:
        raise err[0]
    return out


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_mttkrp_equals_whole(world):
    dims, cidx, vals = synth.zipf_tensor((3000, 2000, 1000), 400_000, 5, s=1.1)
    full = ab.create_alto(ab.SparseTensor.from_arrays(dims, cidx, vals), 16, 0)
    shards = [ShardedTensor(full, r, world, nprtn=8) for r in range(world)]
    assert sum(s.local.info()["nnz"] for s in shards) == full.info()["nnz"]
    rank = 16
    red = ThreadReducer(world)
    streams = [torch.cuda.Stream() for _ in range(world)]
    for mode in range(3):
        U = synth.random_factors(dims, rank, seed=mode)
        d = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, d, rank, full, accumulate=False)
        want = d[mode].cpu().numpy()
        per = [[torch.from_numpy(u).cuda() for u in U] for _ in range(world)]
        torch.cuda.synchronize()
        _run_threads(lambda r: shards[r].mttkrp(mode, per[r], rank, red.fns[r], stream=streams[r]), world)
        torch.cuda.synchronize()
        for r in range(world):
            assert rel_fro(per[r][mode].cpu().numpy(), want) < 1e-12, (mode, r)


def test_sharded_slices_low_reuse_and_long_keys():
    """Slices of a 5-mode tensor with 80-bit keys (a high-word run table) and
    low fiber reuse (oidx rebuilt per slice): each slice's MTTKRP alone equals
    the whole tensor's restricted to the slice's nonzeros."""
    dims, cidx, vals = synth.uniform_distinct((50_000, 45_000, 40_000, 35_000, 60_000), 60_000, seed=4)
    full = ab.create_alto(ab.SparseTensor.from_arrays(dims, cidx, vals), 8, 0)
    assert full.info()["alto_bits"] == 80
    rank = 8
    U = synth.random_factors(dims, rank, seed=1)
    for mode in (0, 3):
        d = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, d, rank, full, accumulate=False)
        want = d[mode].cpu().numpy()
        total = np.zeros_like(want)
        for r in range(2):
            s = ShardedTensor(full, r, 2, nprtn=4)
            assert s.local.info()["is_oidx"]
            dd = [torch.from_numpy(u).cuda() for u in U]
            ab.mttkrp_alto_par(mode, dd, rank, s.local, accumulate=False)
            total += dd[mode].cpu().numpy()
        assert rel_fro(total, want) < 1e-12


def _sparse_low_rank(dims, rank, support, seed):
    """A sparse tensor that is exactly of rank `rank`: component r has
    positive factor columns supported on `support[n]` random rows of each
    mode, and the tensor holds every entry of the sum of the components (the
    union of their supports).  CP-ALS converges on it along a stable
    trajectory; on structureless data its fit stays near 0 and rounding
    differences grow from iteration to iteration."""
    rng = np.random.default_rng(seed)
    N = len(dims)
    A = [np.zeros((d, rank)) for d in dims]
    for r in range(rank):
        for n in range(N):
            rows = rng.choice(dims[n], support[n], replace=False)
            A[n][rows, r] = rng.random(support[n]) + 0.5
    coords = set()
    for r in range(rank):
        sup = [np.nonzero(A[n][:, r])[0] for n in range(N)]
        grid = np.stack(np.meshgrid(*sup, indexing="ij"), axis=0).reshape(N, -1)
        coords.update(map(tuple, grid.T))
    cidx = np.array(sorted(coords), dtype=np.uint64).T
    vals = np.ones((cidx.shape[1], rank))
    for n in range(N):
        vals *= A[n][cidx[n].astype(np.int64)]
    # 10% multiplicative noise: the fit converges near 0.9, away from the
    # cancellation of an exact fit (residual ~ rounding of the model)
    noise = 1.0 + 0.2 * (rng.random(cidx.shape[1]) - 0.5)
    return np.array(dims, np.uint64), cidx, vals.sum(axis=1) * noise


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_sharded_cpd_als_equals_whole(prec):
    world = 2
    vd = "f64" if prec == "f64" else "f32"
    dt = np.float64 if prec == "f64" else np.float32
    dims, cidx, vals = _sparse_low_rank((400, 300, 200), 4, (60, 40, 30), seed=2)
    full = ab.create_alto(ab.SparseTensor.from_arrays(dims, cidx, vals), 16, 0, val_dtype=vd)
    rank, iters = 4, 10

    def model():
        M = ab.random_init_factors(dims, rank, 3, dtype=dt)
        return ab.KruskalModel([int(x) for x in dims], rank, [torch.from_numpy(u.copy()).cuda() for u in M.U],
                               torch.from_numpy(M.lam.copy()).cuda())

    Mw = model()
    want = ab.cpd_alto(full, Mw, iters, 1e-30)
    shards = [ShardedTensor(full, r, world, nprtn=8) for r in range(world)]
    models = [model() for _ in range(world)]
    red = ThreadReducer(world)
    streams = [torch.cuda.Stream() for _ in range(world)]
    torch.cuda.synchronize()
    fits = _run_threads(lambda r: shards[r].cpd_als(models[r], iters, 1e-30, red.fns[r], stream=streams[r]), world)
    torch.cuda.synchronize()
    tol = 1e-9 if prec == "f64" else 1e-4
    for r in range(world):
        assert len(fits[r]) == len(want) == iters
        assert np.max(np.abs(fits[r] - want)) < tol, (r, fits[r], want)
        if prec == "f64":
            for n in range(3):
                assert rel_fro(models[r].U[n].cpu().numpy(), Mw.U[n].cpu().numpy()) < 1e-7, (r, n)
    assert np.array_equal(fits[0], fits[1])  # one stopping decision for every GPU
