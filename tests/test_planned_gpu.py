"""MTTKRP through the per-mode tile plan (k_tile_plan + k_planned) against
the oracle and against the plan-free grouped kernel, and a handle shared by
two streams.  FP64: relative Frobenius error <= 1e-12; FP32: <= 1e-5."""
import os

import numpy as np
import pytest

import alto_b200 as ab
from alto_b200 import synth
from conftest import rel_fro

pytestmark = pytest.mark.gpu
TOL64, TOL32 = 1e-12, 1e-5

CASES = [
    # dims, nnz, rank: tail tiles, one partial tile, orders 3-5, every lane count
    ((1000, 800, 600), 300_001, 32),
    ((1000, 800, 600), 700, 16),
    ((1000, 800, 600), 1024, 8),
    ((300, 5_000, 40, 9), 80_000, 64),
    ((300, 5_000, 40, 9), 80_000, 4),
    ((64, 64, 64, 64, 64), 50_000, 16),
    ((200, 300, 400), 50_000, 2),
    ((200, 300, 400), 50_000, 24),   # lanes past the rank
    ((1000, 800, 600), 200_000, 64),  # order 3, 16 lanes per nonzero (5 blocks per SM in FP32)
    ((1000, 800, 600), 100_000, 48),  # 16 lanes, four past the rank
    ((500, 400, 300), 60_000, 100),   # 32 lanes (4 blocks per SM in FP32), seven past the rank
]


def _plan_env(value):
    old = os.environ.get("ALTOB_PLAN")
    os.environ["ALTOB_PLAN"] = value
    return old


def _restore(old):
    if old is None:
        os.environ.pop("ALTOB_PLAN", None)
    else:
        os.environ["ALTOB_PLAN"] = old


# FP64 ranks above 64 need two vector chunks per lane: the grouped kernel
@pytest.mark.parametrize("case", [c for c in CASES if c[2] <= 64])
def test_planned_fp64_matches_oracle(oracle, case):
    torch = pytest.importorskip("torch")
    dims, nnz, rank = case
    dims_a, cidx, vals = synth.uniform_distinct(dims, nnz, seed=nnz % 89 + rank)
    at = ab.create_alto(ab.SparseTensor.from_arrays(dims_a, cidx, vals), 16, 0)
    ot = oracle.create(dims_a, cidx, vals, 16, at.info()["lit_bits"])
    for mode in range(len(dims)):
        if nnz // dims[mode] <= 4:
            continue  # low fiber reuse: op_sched, not the planned kernel
        U = synth.random_factors(dims_a, rank, seed=mode + 3)
        want = [u.copy() for u in U]
        ot.mttkrp(mode, want, rank)
        dU = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, dU, rank, at)
        assert rel_fro(dU[mode].cpu().numpy(), want[mode]) < TOL64, (case, mode)
        assert at.info()["plan_modes"] >> mode & 1, "the tile plan was not used"


@pytest.mark.parametrize("case", CASES[:4] + CASES[5:6] + CASES[8:])
def test_planned_fp32_matches_grouped_and_fp64(case):
    torch = pytest.importorskip("torch")
    dims, nnz, rank = case
    dims_a, cidx, vals = synth.uniform_distinct(dims, nnz, seed=7 + rank)
    at32 = ab.create_alto(ab.SparseTensor.from_arrays(dims_a, cidx, vals), 16, 0, val_dtype="f32")
    at64 = ab.create_alto(ab.SparseTensor.from_arrays(dims_a, cidx, vals), 16, 0)
    for mode in range(len(dims)):
        if nnz // dims[mode] <= 4:
            continue
        U = synth.random_factors(dims_a, rank, seed=mode)
        d64 = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, d64, rank, at64, accumulate=False)
        want = d64[mode].cpu().numpy()
        outs = []
        for plan in ("1", "0"):
            old = _plan_env(plan)
            try:
                d32 = [torch.from_numpy(u).float().cuda() for u in U]
                ab.mttkrp_alto_par(mode, d32, rank, at32, accumulate=False)
                outs.append(d32[mode].double().cpu().numpy())
            finally:
                _restore(old)
        assert rel_fro(outs[0], want) < TOL32, (case, mode, "planned")
        assert rel_fro(outs[1], want) < TOL32, (case, mode, "grouped")


def test_planned_high_key_word_runs(oracle):
    """66-bit keys with few nonzeros: the high key bits change every few
    hundred nonzeros, so tiles span two or more runs of the high-word table."""
    torch = pytest.importorskip("torch")
    dims = (1 << 22, 1 << 22, 1 << 22)
    dims_a, cidx, vals = synth.uniform_distinct(dims, 3000, seed=5)
    at = ab.create_alto(ab.SparseTensor.from_arrays(dims_a, cidx, vals), 4, 0)
    info = at.info()
    assert info["alto_bits"] == 66
    ot = oracle.create(dims_a, cidx, vals, 4, info["lit_bits"])
    # reuse nnz / I_n is 0 for every mode here, so the default dispatch picks
    # op_sched; the ALTO-order algorithm is asked for explicitly
    for mode in range(3):
        U = synth.random_factors(dims_a, 8, seed=mode)
        want = [u.copy() for u in U]
        ot.mttkrp(mode, want, 8)
        dU = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, dU, 8, at, algo="tiled")
        assert rel_fro(dU[mode].cpu().numpy(), want[mode]) < TOL64, mode
        assert info["nruns"] == 0 or at.info()["plan_modes"] >> mode & 1


def test_one_handle_two_streams():
    """Calls on one handle from two streams, without host synchronisation
    between them, give the results of the same calls on one stream (the
    handle's hot-row buffers and plans are shared: the second stream waits
    for the first)."""
    torch = pytest.importorskip("torch")
    dims = (4000, 3000, 2000)
    dims_a, cidx, vals = synth.zipf_tensor(dims, 600_000, 3, s=1.1)
    rank = 32
    at = ab.create_alto(ab.SparseTensor.from_arrays(dims_a, cidx, vals), 16, 0, val_dtype="f32")
    U = [torch.from_numpy(u).float().cuda() for u in synth.random_factors(dims_a, rank, seed=1)]
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def run(streams):
        outs = []
        for k in range(6):
            mode = k % 3
            st = streams[k % len(streams)]
            o = torch.zeros(dims[mode], rank, device="cuda")
            st.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(st):
                ab.mttkrp_alto_par(mode, [o if m == mode else U[m] for m in range(3)], rank, at, accumulate=True,
                                   stream=st)
            outs.append((o, st))
        torch.cuda.synchronize()
        return [o.double().cpu().numpy() for o, _ in outs]

    one = run([s1])
    two = run([s1, s2])
    for a, b in zip(one, two):
        assert rel_fro(b, a) < 1e-6


TMA_CASES = [
    # dims, nnz, rank: tail tile, ranks 16/32/64, 65-bit keys (run table), skew (hot rows)
    ((1000, 800, 600), 300_001, 32, "uniform"),
    ((1000, 800, 600), 1500, 16, "uniform"),
    ((200, 300, 400), 60_000, 64, "uniform"),
    ((1 << 22, 1 << 21, 1 << 22), 2_000_000, 32, "zipf"),
]


@pytest.mark.parametrize("stages", ["2", "4"])
@pytest.mark.parametrize("case", TMA_CASES)
def test_tma_staged_kernel_matches_planned_and_fp64(case, stages, monkeypatch):
    """The TMA-staged kernel (factor rows gathered into shared memory by
    cp.async.bulk.tensor tile::gather4) against the planned kernel and the
    FP64 result, FP32 within 1e-5; its wait-limit flag stays clear."""
    torch = pytest.importorskip("torch")
    dims, nnz, rank, kind = case
    if kind == "zipf":
        d, cidx, vals = synth.zipf_tensor(dims, nnz, 7, s=1.1)
    else:
        d, cidx, vals = synth.uniform_distinct(dims, nnz, seed=rank)
    at32 = ab.create_alto(ab.SparseTensor.from_arrays(d, cidx, vals), 16, 0, val_dtype="f32")
    at64 = ab.create_alto(ab.SparseTensor.from_arrays(d, cidx, vals), 16, 0)
    for mode in range(3):
        U = synth.random_factors(d, rank, seed=mode)
        d64 = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, d64, rank, at64, accumulate=False)
        want = d64[mode].cpu().numpy()
        got = {}
        for tma in ("0", "1"):
            monkeypatch.setenv("ALTOB_TMA", tma)
            monkeypatch.setenv("ALTOB_TMA_STAGES", stages)
            d32 = [torch.from_numpy(u).float().cuda() for u in U]
            ab.mttkrp_alto_par(mode, d32, rank, at32, accumulate=False)
            torch.cuda.synchronize()
            got[tma] = d32[mode].double().cpu().numpy()
        assert at32.info()["tma_err"] == 0
        assert rel_fro(got["1"], want) < TOL32, (case, mode)
        assert rel_fro(got["1"], got["0"]) < TOL32, (case, mode)
