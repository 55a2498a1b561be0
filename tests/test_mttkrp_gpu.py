"""MTTKRP on the GPU against the reference (fixtures) and the oracle.
FP64: relative Frobenius error <= 1e-12.  FP32: <= 1e-5 against FP64."""
import numpy as np
import pytest

import alto_b200 as ab
from alto_b200 import synth
from conftest import golden_cases, load_golden, rel_fro
from helpers import mttkrp_from_golden

pytestmark = pytest.mark.gpu
TOL64, TOL32 = 1e-12, 1e-5


def _coo(dims, cidx, vals):
    return ab.SparseTensor.from_arrays(dims, cidx, vals)


@pytest.mark.parametrize("name", [n for n in golden_cases("enc_") if "mttkrp0_rows" in load_golden(n)])
def test_gpu_mttkrp_matches_reference_fixture(name):
    g = load_golden(name)
    rank = int(g["rank"])
    at = ab.create_alto(_coo(g["dims"], g["cidx"], g["vals"]), int(g["nprtn"]), int(g["lit_bits"]))
    for mode in range(len(g["dims"])):
        U, want = mttkrp_from_golden(g, mode, synth)
        ab.mttkrp_alto_par(mode, U, rank, at)  # host factors, += semantics
        assert rel_fro(U[mode], want) < TOL64, (name, mode)


ALGO_CASES = [
    # dims, nnz, nprtn, rank, algos
    ((1000, 800, 600), 300_000, 64, 16, ["auto", "tiled", "atomic"]),
    ((1000, 800, 600), 100_000, 8, 32, ["tiled"]),
    ((40_000, 30_000, 20_000), 60_000, 16, 8, ["auto", "tiled", "atomic", "atomic_cr", "op_sched"]),
    ((300, 5_000, 40, 9), 80_000, 12, 64, ["auto", "tiled", "atomic"]),
    ((512, 512, 512, 512, 512), 50_000, 10, 16, ["auto", "tiled", "atomic", "op_sched", "atomic_cr"]),
    ((200, 300, 400), 50_000, 4, 5, ["tiled", "atomic"]),      # odd rank: scalar lanes
    ((200, 300, 400), 50_000, 4, 100, ["tiled"]),              # rank 100 (reference specialisation)
]


@pytest.mark.parametrize("case", ALGO_CASES)
def test_gpu_mttkrp_fp64_all_algorithms(oracle, case):
    torch = pytest.importorskip("torch")
    dims, nnz, nprtn, rank, algos = case
    dims_a, cidx, vals = synth.uniform_distinct(dims, nnz, seed=nnz % 97)
    at = ab.create_alto(_coo(dims_a, cidx, vals), nprtn, 0)
    ot = oracle.create(dims_a, cidx, vals, nprtn, at.info()["lit_bits"])
    for mode in range(len(dims)):
        U = synth.random_factors(dims_a, rank, seed=mode)
        want = [u.copy() for u in U]
        ot.mttkrp(mode, want, rank)
        for algo in algos:
            if algo == "atomic_cr" and not at.info()["cr_masks"][mode].any():
                continue
            if algo == "op_sched" and nnz // dims[mode] > 4:
                continue
            dU = [torch.from_numpy(u).cuda() for u in U]
            ab.mttkrp_alto_par(mode, dU, rank, at, algo=algo)
            got = dU[mode].cpu().numpy()
            assert rel_fro(got, want[mode]) < TOL64, (case, mode, algo)


@pytest.mark.parametrize("case", ALGO_CASES[:4])
def test_gpu_mttkrp_fp32_against_fp64(oracle, case):
    torch = pytest.importorskip("torch")
    dims, nnz, nprtn, rank, _ = case
    dims_a, cidx, vals = synth.uniform_distinct(dims, nnz, seed=nnz % 89)
    at = ab.create_alto(_coo(dims_a, cidx, vals), nprtn, 0, val_dtype="f32")
    ot = oracle.create(dims_a, cidx, vals.astype(np.float32).astype(np.float64), nprtn, at.info()["lit_bits"])
    for mode in range(len(dims)):
        U = [u.astype(np.float32) for u in synth.random_factors(dims_a, rank, seed=mode)]
        want = [u.astype(np.float64) for u in U]
        ot.mttkrp(mode, want, rank)
        dU = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, dU, rank, at, accumulate=False)
        want_mode = want[mode] - U[mode].astype(np.float64)  # accumulate=False: output only
        assert rel_fro(dU[mode].cpu().numpy(), want_mode) < TOL32


@pytest.mark.parametrize("rank", [12, 24])
def test_gpu_mttkrp_lanes_past_rank(oracle, rank):
    """Ranks that leave lanes of a nonzero's lane group past the rank (12 and
    24: 4 or 8 lanes of 4 FP32 values, 8 or 16 lanes of 2 FP64 values, the
    last ones beyond R); their loads stay in the row and nothing they hold is
    written, in FP64 (+= semantics) and FP32 (overwrite)."""
    torch = pytest.importorskip("torch")
    dims, nnz, nprtn = (300, 200, 100), 40_000, 8
    dims_a, cidx, vals = synth.uniform_distinct(dims, nnz, seed=rank)
    at = ab.create_alto(_coo(dims_a, cidx, vals), nprtn, 0)
    ot = oracle.create(dims_a, cidx, vals, nprtn, at.info()["lit_bits"])
    at32 = ab.create_alto(_coo(dims_a, cidx, vals), nprtn, 0, val_dtype="f32")
    ot32 = oracle.create(dims_a, cidx, vals.astype(np.float32).astype(np.float64), nprtn, at32.info()["lit_bits"])
    for mode in range(len(dims)):
        U = synth.random_factors(dims_a, rank, seed=mode)
        want = [u.copy() for u in U]
        ot.mttkrp(mode, want, rank)
        dU = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, dU, rank, at)
        assert rel_fro(dU[mode].cpu().numpy(), want[mode]) < TOL64, (rank, mode)
        U32 = [u.astype(np.float32) for u in U]
        want32 = [u.astype(np.float64) for u in U32]
        ot32.mttkrp(mode, want32, rank)
        d32 = [torch.from_numpy(u).cuda() for u in U32]
        ab.mttkrp_alto_par(mode, d32, rank, at32, accumulate=False)
        got32 = d32[mode].cpu().numpy()
        assert rel_fro(got32, want32[mode] - U32[mode].astype(np.float64)) < TOL32, (rank, mode)


def test_gpu_mttkrp_zipf_skew_fp64_and_fp32(oracle):
    """Config-2 shape (Zipf 1.1 skew, 65-bit keys) at reduced size."""
    torch = pytest.importorskip("torch")
    dims, cidx, vals = synth.zipf_tensor((4_800_000, 1_800_000, 1_800_000), 300_000, seed=2)
    rank = 32
    at64 = ab.create_alto(_coo(dims, cidx, vals), 32, 0)
    at32 = ab.create_alto(_coo(dims, cidx, vals), 32, 0, val_dtype="f32")
    ot = oracle.create(dims, cidx, vals, 32, 128)
    rng = np.random.default_rng(0)
    for mode in range(3):
        U = [rng.random((int(d), rank)) for d in dims]
        want = [u.copy() for u in U]
        want[mode][:] = 0
        ot.mttkrp(mode, want, rank)
        d64 = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, d64, rank, at64, accumulate=False)
        assert rel_fro(d64[mode].cpu().numpy(), want[mode]) < TOL64
        d32 = [torch.from_numpy(u.astype(np.float32)).cuda() for u in U]
        ab.mttkrp_alto_par(mode, d32, rank, at32, accumulate=False)
        assert rel_fro(d32[mode].cpu().numpy(), want[mode]) < TOL32


def test_gpu_mttkrp_u32_counts(oracle):
    torch = pytest.importorskip("torch")
    dims, cidx, vals = synth.poisson_kruskal((300, 200, 100, 20), 5, 100_000, seed=3)
    at = ab.create_alto(_coo(dims, cidx, vals), 8, 0, val_dtype="u32")
    ot = oracle.create(dims, cidx, vals, 8, 64)
    for mode in range(4):
        U = synth.random_factors(dims, 16, seed=mode)
        want = [u.copy() for u in U]
        ot.mttkrp(mode, want, 16)
        dU = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, dU, 16, at)
        assert rel_fro(dU[mode].cpu().numpy(), want[mode]) < TOL64


@pytest.mark.parametrize("iters", [0, 1, 2])
@pytest.mark.parametrize("shape", [(500, 400, 300), (60, 50, 40, 30)])
def test_gpu_mttkrp_sweep_host_matches_sequential_calls(oracle, iters, shape):
    """The sweep copies each factor back as soon as its mode is final (on a
    second stream); the result equals mode-by-mode calls."""
    dims, cidx, vals = synth.uniform_distinct(shape, 100_000, seed=4)
    at = ab.create_alto(_coo(dims, cidx, vals), 16, 0)
    ot = oracle.create(dims, cidx, vals, 16, 64)
    U = synth.random_factors(dims, 16, seed=1)
    want = [u.copy() for u in U]
    for _ in range(iters):
        for m in range(len(shape)):
            ot.mttkrp(m, want, 16)
    ab.mttkrp_sweep_host(at, U, 16, iters=iters)
    for m in range(len(shape)):
        s = np.abs(want[m]).max()  # += sweeps grow the values fast (1e238 for 4 modes): compare scaled
        assert rel_fro(U[m] / s, want[m] / s) < TOL64


def test_gpu_mttkrp_empty_and_errors():
    torch = pytest.importorskip("torch")
    dims = np.array([10, 20, 30], np.uint64)
    at = ab.create_alto(_coo(dims, np.zeros((3, 0), np.uint64), np.zeros(0)), 4, 64)
    U = [torch.ones(int(d), 8, dtype=torch.float64, device="cuda") for d in dims]
    ab.mttkrp_alto_par(1, U, 8, at)
    assert float(U[1].sum()) == 20 * 8  # += nothing
    ab.mttkrp_alto_par(1, U, 8, at, accumulate=False)
    assert float(U[1].abs().sum()) == 0.0
    with pytest.raises(ab.AltobError):
        ab.mttkrp_alto_par(3, U, 8, at)


def test_gpu_mttkrp_fp32_skewed_large_within_1e5():
    """FP32 MTTKRP on a large Zipf(1.1)-skewed tensor (the head rows collect
    contributions from almost every 1024-nonzero tile) against FP64 on the
    same values: relative Frobenius error below 1e-5 in every mode."""
    torch = pytest.importorskip("torch")
    dims = (4_800_000, 1_800_000, 1_800_000)
    cidx, vals, nnz = synth.zipf_tensor_torch(dims, 140_000_000, 1.1, 5, "cuda")
    d = np.array(dims, np.uint64)
    at32 = ab.create_alto_device(3, d, nnz, cidx, vals, nprtn=1024, lit_bits=128, val_dtype="f32")
    at64 = ab.create_alto_device(3, d, nnz, cidx, vals.double(), nprtn=1024, lit_bits=128, val_dtype="f64")
    del cidx, vals
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    U = [torch.rand(x, 32, dtype=torch.float64, device="cuda", generator=g) for x in dims]
    for mode in range(3):
        U32 = [u.float() for u in U]
        U64 = [u.clone() for u in U]
        ab.mttkrp_alto_par(mode, U32, 32, at32, accumulate=False)
        ab.mttkrp_alto_par(mode, U64, 32, at64, accumulate=False)
        err = float((U32[mode].double() - U64[mode]).norm() / U64[mode].norm())
        assert err < 1e-5, (mode, err)
