"""Parity against the reference itself (oracle/_ref, the reference compiled
from its sources) at the sizes of the benchmark workloads:

* the large skewed tensor (4.8M x 1.8M x 1.8M, 140M Zipf(1.1) draws per mode
  merged to 100.85M nonzeros, 65-bit keys): the encoding bit for bit
  (index words, partitions, intervals, masks), FP64 MTTKRP of every mode
  within 1e-12 and FP32 within 1e-5 of the reference's FP64 mttkrp_alto_par
  (relative Frobenius error);
* CP-APR on a 4-mode count tensor of the benchmark's family (2M Poisson
  draws from a rank-10 Gamma(0.3, 1) model) with the full 50 outer x 10
  inner schedule: log-likelihood within 1e-4 (relative) of the reference's
  cp_apr_alto and the same iteration counts, FP64 and FP32 models.

The reference runs on the host cores; these tests need a few GB of host
memory and take about a minute."""
import numpy as np
import pytest

import alto_b200 as ab
from alto_b200 import synth
from conftest import rel_fro

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
orc = pytest.importorskip("oracle.orc")

DIMS = (4_800_000, 1_800_000, 1_800_000)
NPRTN = 64


@pytest.fixture(scope="module")
def ref():
    if not orc.ref_available():
        pytest.skip("reference library oracle/_ref not built")
    return orc.RefLib()


@pytest.fixture(scope="module")
def zipf_full():
    cidx, vals, nnz = synth.zipf_tensor_torch(DIMS, 140_000_000, 1.1, 2, "cuda")
    hc = cidx.cpu().numpy().astype(np.uint64)
    hv = vals.double().cpu().numpy()
    del cidx, vals
    torch.cuda.empty_cache()
    return np.array(DIMS, np.uint64), hc, hv, nnz


def test_fullsize_zipf_encoding_bit_exact(ref, zipf_full):
    dims, cidx, vals, nnz = zipf_full
    assert nnz > 100_000_000
    want = ref.create_dump(dims, cidx, vals, NPRTN, 128)
    at = ab.create_alto(ab.SparseTensor.from_arrays(dims, cidx, vals), NPRTN, 128)
    got = at.dump()
    assert want["alto_bits"] == at.info()["alto_bits"] == 65
    for key in ("idx", "prtn_ptr", "intervals"):
        assert np.array_equal(got[key].reshape(want[key].shape), want[key]), key
    assert np.array_equal(got["vals"], want["vals"])
    info = at.info()
    assert np.array_equal(info["masks"], want["masks"])
    assert np.array_equal(info["cr_masks"], want["cr_masks"])


def test_fullsize_zipf_mttkrp_fp64_and_fp32_vs_reference(ref, zipf_full):
    dims, cidx, vals, nnz = zipf_full
    rank = 32
    X = ab.SparseTensor.from_arrays(dims, cidx, vals)
    at64 = ab.create_alto(X, NPRTN, 128)
    at32 = ab.create_alto(X, NPRTN, 128, val_dtype="f32")
    rng = np.random.default_rng(11)
    U = [rng.random((int(d), rank)) for d in dims]
    for mode in range(3):
        want = [u if m != mode else np.zeros_like(u) for m, u in enumerate(U)]
        ref.mttkrp(dims, cidx, vals, NPRTN, 128, mode, want, rank)
        d64 = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, d64, rank, at64, accumulate=False)
        e64 = rel_fro(d64[mode].cpu().numpy(), want[mode])
        del d64
        d32 = [torch.from_numpy(u).float().cuda() for u in U]
        ab.mttkrp_alto_par(mode, d32, rank, at32, accumulate=False)
        e32 = rel_fro(d32[mode].double().cpu().numpy(), want[mode])
        del d32
        torch.cuda.empty_cache()
        assert e64 < 1e-12, (mode, e64)
        assert e32 < 1e-5, (mode, e32)


def test_fullsize_cp_apr_50x10_vs_reference(ref):
    dims = synth.CONFIG3_DIMS
    c, v = synth.poisson_kruskal_torch(dims, 10, 2_000_000, 303, "cuda", shape=0.3)
    cidx, vals = c.cpu().numpy().astype(np.uint64), v.cpu().numpy().astype(np.float64)
    nnz = vals.shape[0]
    assert nnz > 1_000_000
    rank, outer, inner, seed = 16, 50, 10, 5
    d = np.array(dims, np.uint64)
    _, _, want = ref.apr(d, cidx, vals, NPRTN, 64, rank, outer, inner, 0.0, 1e-10, 1e-10, 1e-2, True, seed)
    at = ab.create_alto(ab.SparseTensor.from_arrays(d, cidx, vals), NPRTN, 64, val_dtype="u32")
    for dtype in (np.float64, np.float32):
        M = ab.random_init_factors(d, rank, seed, dtype=dtype)
        got = ab.cp_apr_alto(at, M, outer, inner, 0.0, 1e-10, 1e-10, 1e-2, True)
        assert got["outer"] == want["outer"] and got["inner"] == want["inner"], (dtype, got, want)
        rel = abs(got["loglik"] - want["loglik"]) / abs(want["loglik"])
        assert rel < 1e-4, (dtype, got["loglik"], want["loglik"])
