"""CP-ALS and CP-APR on the GPU against fixtures written by the reference
and against the oracle.  Fit and log-likelihood tolerance: 1e-4 (FP32
model against the FP64 reference); FP64 runs are held much tighter."""
import time

import numpy as np
import pytest

import alto_b200 as ab
from alto_b200 import synth
from conftest import load_golden, rel_fro

pytestmark = pytest.mark.gpu


def _coo(dims, cidx, vals):
    return ab.SparseTensor.from_arrays(dims, cidx, vals)


def test_gpu_cpd_fp64_matches_reference_fixture():
    g = load_golden("cpd_u3")
    rank = int(g["rank"])
    at = ab.create_alto(_coo(g["dims"], g["cidx"], g["vals"]), int(g["nprtn"]), 64)
    M = ab.random_init_factors(g["dims"], rank, int(g["seed"]))
    fits = ab.cpd_alto(at, M, int(g["max_iters"]), 1e-30)
    assert len(fits) == len(g["fits"])
    np.testing.assert_allclose(fits, g["fits"], rtol=2e-6)  # printed with %g
    for n in range(3):
        assert rel_fro(M.U[n], g[f"U{n}"]) < 1e-8
    np.testing.assert_allclose(M.lam, g["lam"], rtol=1e-8)


def test_gpu_cpd_fp64_stopping_rule_matches_reference():
    g = load_golden("cpd_conv4")
    rank = int(g["rank"])
    at = ab.create_alto(_coo(g["dims"], g["cidx"], g["vals"]), int(g["nprtn"]), 64)
    M = ab.random_init_factors(g["dims"], rank, int(g["seed"]))
    fits = ab.cpd_alto(at, M, int(g["max_iters"]), float(g["eps"]))
    assert len(fits) == len(g["fits"])
    np.testing.assert_allclose(fits, g["fits"], rtol=2e-6)


def test_gpu_cpd_config1_fp64_and_fp32_fit_trajectory():
    """Config 1 (1000x800x600, 1M nonzeros, rank 16, 20 iterations): FP64
    and FP32 fits against the reference's printed trajectory."""
    ref = load_golden("cpd_config1_fits")
    dims, cidx, vals = synth.uniform_distinct((1000, 800, 600), 1_000_000, seed=int(ref["data_seed"]))
    at = ab.create_alto(_coo(dims, cidx, vals), int(ref["nprtn"]), 64)
    M = ab.random_init_factors(dims, 16, int(ref["seed"]))
    fits = ab.cpd_alto(at, M, 20, 1e-30)
    assert len(fits) == 20
    assert np.max(np.abs(fits - ref["fits"])) < 1e-7
    at32 = ab.create_alto(_coo(dims, cidx, vals), int(ref["nprtn"]), 64, val_dtype="f32")
    M32 = ab.random_init_factors(dims, 16, int(ref["seed"]), dtype=np.float32)
    fits32 = ab.cpd_alto(at32, M32, 20, 1e-30)
    assert np.max(np.abs(fits32 - ref["fits"])) < 1e-4


def test_gpu_cpd_device_model_matches_oracle(oracle):
    torch = pytest.importorskip("torch")
    dims, cidx, vals = synth.uniform_distinct((300, 200, 100, 50), 100_000, seed=5)
    rank = 24
    at = ab.create_alto(_coo(dims, cidx, vals), 16, 0)
    U, lam = oracle.random_init(dims, rank, 3)
    ot = oracle.create(dims, cidx, vals, 16, 64)
    dU = [torch.from_numpy(u.copy()).cuda() for u in U]
    dl = torch.from_numpy(lam.copy()).cuda()
    M = ab.KruskalModel([int(d) for d in dims], rank, dU, dl)
    fits = ab.cpd_alto(at, M, 8, 1e-30)
    ofits = ot.cpd_als(U, lam, rank, 8, 1e-30)
    np.testing.assert_allclose(fits, ofits, rtol=1e-9)
    for n in range(4):
        assert rel_fro(dU[n].cpu().numpy(), U[n]) < 1e-8


@pytest.mark.parametrize("phi", ["rows", "pre", "otf"])
@pytest.mark.parametrize("name", ["apr_bench", "apr_eps"])
def test_gpu_cp_apr_fp64_matches_reference_fixture(name, phi, monkeypatch):
    """Every Phi path (precomputed Khatri-Rao rows in the row-ordered stream
    or in ALTO order, on the fly) against the reference's own output."""
    monkeypatch.setenv("ALTOB_APR_PHI", phi)
    g = load_golden(name)
    rank = int(g["rank"])
    at = ab.create_alto(_coo(g["dims"], g["cidx"], g["vals"]), int(g["nprtn"]), 64, val_dtype="u32")
    M = ab.random_init_factors(g["dims"], rank, int(g["seed"]))
    r = ab.cp_apr_alto(at, M, int(g["max_iters"]), int(g["max_inner"]), float(g["eps"]), 1e-10, 1e-10, 1e-2,
                       bool(g["dobench"]))
    assert r["outer"] == int(g["outer"]) and r["inner"] == int(g["inner"])
    np.testing.assert_allclose(r["loglik"], g["loglik"], rtol=1e-6)
    np.testing.assert_allclose(r["fit"], g["fit"], rtol=1e-6)
    np.testing.assert_allclose(r["kkt"], g["kkt"], rtol=1e-6)
    for n in range(3):
        assert rel_fro(M.U[n], g[f"U{n}"]) < 1e-8


@pytest.mark.parametrize("phi", ["rows", "pre", "otf"])
def test_gpu_cp_apr_early_exit_and_fp32(oracle, phi, monkeypatch):
    monkeypatch.setenv("ALTOB_APR_PHI", phi)
    dims, cidx, vals = synth.poisson_kruskal((200, 150, 100, 20), 6, 200_000, seed=6)
    rank = 8
    U, lam = oracle.random_init(dims, rank, 4)
    ot = oracle.create(dims, cidx, vals, 8, 64)
    oU = [u.copy() for u in U]
    olam = lam.copy()
    want = ot.cp_apr(oU, olam, rank, 12, 10, eps=1e-2)
    at = ab.create_alto(_coo(dims, cidx, vals), 8, 0, val_dtype="u32")
    M = ab.KruskalModel([int(d) for d in dims], rank, [u.copy() for u in U], lam.copy())
    got = ab.cp_apr_alto(at, M, 12, 10, epsilon=1e-2)
    assert got["outer"] == want["outer"] and got["inner"] == want["inner"]
    np.testing.assert_allclose(got["loglik"], want["loglik"], rtol=1e-9)
    np.testing.assert_allclose(got["fit"], want["fit"], rtol=1e-8, atol=1e-10)
    # FP32 model, bench mode (fixed inner counts), against the FP64 oracle
    oU = [u.copy() for u in U]
    olam = lam.copy()
    want = ot.cp_apr(oU, olam, rank, 6, 5, eps=0.0, dobench=True)
    M32 = ab.KruskalModel([int(d) for d in dims], rank, [u.astype(np.float32) for u in U], lam.astype(np.float32))
    got = ab.cp_apr_alto(at, M32, 6, 5, epsilon=0.0, dobench=True)
    assert abs(got["loglik"] - want["loglik"]) <= 1e-4 * abs(want["loglik"])
    assert abs(got["fit"] - want["fit"]) <= 1e-4


@pytest.mark.parametrize("rank", [3, 16, 40, 100])
def test_gpu_cp_apr_row_stream_matches_on_the_fly(rank, monkeypatch):
    """The row-ordered Phi for every lane layout (ranks below, at and above
    one vector per lane group; 2 and 4 chunks per lane) against the
    on-the-fly Phi, FP64 and FP32, fixed inner counts."""
    dims, cidx, vals = synth.poisson_kruskal((300, 120, 80, 15), 5, 150_000, seed=21)
    at = ab.create_alto(_coo(dims, cidx, vals), 8, 0, val_dtype="u32")
    for dtype, tol in ((np.float64, 1e-10), (np.float32, 1e-4)):
        res = {}
        for phi in ("rows", "otf"):
            monkeypatch.setenv("ALTOB_APR_PHI", phi)
            M = ab.random_init_factors(dims, rank, 3, dtype=dtype)
            res[phi] = (ab.cp_apr_alto(at, M, 4, 5, epsilon=0.0, dobench=True), M)
        (ra, Ma), (rb, Mb) = res["rows"], res["otf"]
        assert abs(ra["loglik"] - rb["loglik"]) <= tol * abs(rb["loglik"])
        for n in range(4):
            assert rel_fro(Ma.U[n], Mb.U[n]) < (1e-9 if dtype == np.float64 else 1e-3), n


@pytest.mark.parametrize("rank", [4, 16, 24, 64])
def test_gpu_cp_apr_bulk_copy_phi_matches_register_staged(rank, monkeypatch):
    """The row-ordered Phi staged in shared memory by bulk copies
    (ALTOB_PHI_TMA=1) against the register-staged one, FP64 and FP32, fixed
    inner counts; a nonzero count that is not a multiple of 4 exercises the
    padded tail of the stream arrays."""
    dims, cidx, vals = synth.poisson_kruskal((300, 120, 80, 15), 5, 150_003, seed=22)
    at = ab.create_alto(_coo(dims, cidx, vals), 8, 0, val_dtype="u32")
    monkeypatch.setenv("ALTOB_APR_PHI", "rows")
    for dtype, tol in ((np.float64, 1e-10), (np.float32, 1e-4)):
        res = {}
        for tma in ("1", "0"):
            monkeypatch.setenv("ALTOB_PHI_TMA", tma)
            M = ab.random_init_factors(dims, rank, 3, dtype=dtype)
            res[tma] = (ab.cp_apr_alto(at, M, 4, 5, epsilon=0.0, dobench=True), M)
        (ra, Ma), (rb, Mb) = res["1"], res["0"]
        assert abs(ra["loglik"] - rb["loglik"]) <= tol * abs(rb["loglik"])
        for n in range(4):
            assert rel_fro(Ma.U[n], Mb.U[n]) < (1e-9 if dtype == np.float64 else 1e-3), n


def test_gpu_bulk_copy_phi_wait_runs_out_and_reports(monkeypatch):
    """Failure detection without a GPU fault: the bulk-copy-staged Phi's
    producer warp is told to issue nothing (ALTOB_TEST_STALL_PHI=1), so every
    consumer wait on a stage's mbarrier runs out after a short limit; the
    kernel returns normally, records the failure in the handle's error word,
    and the solve reports ALTOB_ERR_CUDA.  The GPU stays usable: a fresh
    handle then solves normally and equals the register-staged solve."""
    dims, cidx, vals = synth.poisson_kruskal((300, 120, 80, 15), 5, 60_000, seed=23)
    rank = 16
    monkeypatch.setenv("ALTOB_APR_PHI", "rows")
    monkeypatch.setenv("ALTOB_PHI_TMA", "1")
    monkeypatch.setenv("ALTOB_TEST_STALL_PHI", "1")
    at = ab.create_alto(_coo(dims, cidx, vals), 8, 0, val_dtype="u32")
    M = ab.random_init_factors(dims, rank, 3, dtype=np.float32)
    with pytest.raises(ab.AltobError, match="wait limit"):
        ab.cp_apr_alto(at, M, 2, 3, epsilon=0.0, dobench=True)
    monkeypatch.delenv("ALTOB_TEST_STALL_PHI")
    res = {}
    for tma in ("1", "0"):
        monkeypatch.setenv("ALTOB_PHI_TMA", tma)
        fresh = ab.create_alto(_coo(dims, cidx, vals), 8, 0, val_dtype="u32")
        M = ab.random_init_factors(dims, rank, 3, dtype=np.float32)
        res[tma] = ab.cp_apr_alto(fresh, M, 2, 3, epsilon=0.0, dobench=True)
    assert abs(res["1"]["loglik"] - res["0"]["loglik"]) <= 1e-4 * abs(res["0"]["loglik"])


def test_gpu_phi_and_loglik_match_oracle(oracle):
    torch = pytest.importorskip("torch")
    dims, cidx, vals = synth.poisson_kruskal((120, 90, 60), 5, 50_000, seed=8)
    rank = 12
    at = ab.create_alto(_coo(dims, cidx, vals), 4, 0, val_dtype="u32")
    ot = oracle.create(dims, cidx, vals, 4, 64)
    U = synth.random_factors(dims, rank, seed=9)
    dU = [torch.from_numpy(u).cuda() for u in U]
    for mode in range(3):
        want = ot.phi(mode, U, rank)
        phi = torch.empty(int(dims[mode]), rank, dtype=torch.float64, device="cuda")
        ab.calculate_phi(at, mode, dU, rank, phi)
        assert rel_fro(phi.cpu().numpy(), want) < 1e-12
    lam = np.linspace(0.5, 2.0, rank)
    oU = [u.copy() for u in U]
    olam = lam.copy()
    want = ot.loglik(oU, olam, rank)
    dl = torch.from_numpy(lam.copy()).cuda()
    M = ab.KruskalModel([int(d) for d in dims], rank, dU, dl)
    got = ab.tt_logLikelihood(at, M)
    np.testing.assert_allclose(got, want, rtol=1e-12)
    assert rel_fro(dU[0].cpu().numpy(), oU[0]) < 1e-13
    np.testing.assert_allclose(dl.cpu().numpy(), olam, rtol=1e-12)


def _grams(Us):
    return np.stack([u.T @ u for u in Us])


@pytest.mark.parametrize("R", [8, 37, 64])
def test_gpu_pseudo_inverse_cholesky_matches_oracle(oracle, R):
    """pseudo_inverse (cpd.hpp:546-646) with a positive definite V."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(R)
    Us = [rng.random((d, R)) for d in (300, 200, 150)]
    G = _grams(Us)
    U = rng.random((500, R))
    want, used_o = oracle.pseudo_inverse(G, 1, U)
    dU = torch.from_numpy(U.copy()).cuda()
    used = ab.pseudo_inverse(torch.from_numpy(G).cuda(), 1, dU)
    assert not used and not used_o
    assert rel_fro(dU.cpu().numpy(), want) < 1e-10


@pytest.mark.parametrize("R", [6, 33, 64, 112])
def test_gpu_pseudo_inverse_fallback_matches_oracle(oracle, R):
    """A singular V (two equal columns in every other factor, integer entries
    so that the Cholesky pivot is exactly 0 on every machine) takes the
    pseudo-inverse path on both sides; the results agree."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(100 + R)
    Us = []
    for d in (40, 30, 25):
        u = rng.integers(0, 3, size=(d, R)).astype(np.float64)
        u[:, 0] = 0.0
        u[0, 0] = 1.0
        u[:, 1] = u[:, 0]
        Us.append(u)
    G = _grams(Us)
    U = rng.random((200, R))
    want, used_o = oracle.pseudo_inverse(G, 0, U)
    dU = torch.from_numpy(U.copy()).cuda()
    t0 = time.perf_counter()
    used = ab.pseudo_inverse(torch.from_numpy(G).cuda(), 0, dU)
    dt = time.perf_counter() - t0
    assert used and used_o
    assert rel_fro(dU.cpu().numpy(), want) < 1e-9
    assert dt < 1.0  # parallel Jacobi: milliseconds, not a serial sweep per rotation
    dU32 = torch.from_numpy(U.astype(np.float32)).cuda()
    assert ab.pseudo_inverse(torch.from_numpy(G).cuda(), 0, dU32)
    assert rel_fro(dU32.cpu().numpy(), want) < 1e-5


@pytest.mark.parametrize("rank", [1, 5, 8, 13, 16, 27, 32, 33, 48, 64, 65])
def test_gpu_cpd_fused_row_update_matches_oracle(oracle, rank, monkeypatch):
    """Ranks up to 64 take the fused row-update + Gram pass (FP64 MMA), 65 the
    separate passes; both against the oracle (FP64), and the fused FP64 result
    against the separate passes (ALTOB_FUSED_APPLY=0)."""
    torch = pytest.importorskip("torch")
    dims, cidx, vals = synth.uniform_distinct((300, 200, 100), 60_000, seed=11)
    at = ab.create_alto(_coo(dims, cidx, vals), 16, 0)
    U, lam = oracle.random_init(dims, rank, 5)
    ot = oracle.create(dims, cidx, vals, 16, 64)

    def run(dtype):
        dU = [torch.from_numpy(u.astype(dtype)).cuda() for u in U]
        dl = torch.from_numpy(lam.astype(dtype)).cuda()
        fits = ab.cpd_alto(at if dtype == np.float64 else at32, ab.KruskalModel([int(d) for d in dims], rank, dU, dl),
                           6, 1e-30)
        return fits, [u.cpu().numpy() for u in dU], dl.cpu().numpy()

    at32 = ab.create_alto(_coo(dims, cidx, vals), 16, 0, val_dtype="f32")
    oU = [u.copy() for u in U]
    ofits = ot.cpd_als(oU, lam.copy(), rank, 6, 1e-30)
    fits, gU, glam = run(np.float64)
    np.testing.assert_allclose(fits, ofits, rtol=1e-9)
    for n in range(3):
        assert rel_fro(gU[n], oU[n]) < 1e-8, n
    monkeypatch.setenv("ALTOB_FUSED_APPLY", "0")
    fits0, gU0, glam0 = run(np.float64)
    monkeypatch.delenv("ALTOB_FUSED_APPLY")
    assert np.max(np.abs(fits - fits0)) < 1e-12
    for n in range(3):
        assert rel_fro(gU[n], gU0[n]) < 1e-11, n
    np.testing.assert_allclose(glam, glam0, rtol=1e-11)
    fits32, _, _ = run(np.float32)
    assert np.max(np.abs(fits32 - ofits)) < 1e-4


@pytest.mark.parametrize("rank", [16, 24, 32, 64])
def test_gpu_cpd_fused_row_update_unaligned_factors(rank):
    """Factor matrices that start 4 bytes past a 16-byte boundary take the
    scalar loads of the fused pass (and of the MTTKRP); same fits as aligned
    factors."""
    torch = pytest.importorskip("torch")
    dims, cidx, vals = synth.uniform_distinct((400, 150, 90), 50_000, seed=12)
    at = ab.create_alto(_coo(dims, cidx, vals), 16, 0, val_dtype="f32")
    M = ab.random_init_factors(dims, rank, 8, dtype=np.float32)

    def run(offset):
        dU = []
        for u in M.U:
            buf = torch.zeros(u.size + offset, dtype=torch.float32, device="cuda")
            v = buf[offset:].view(u.shape)
            v.copy_(torch.from_numpy(u))
            dU.append(v)
        dl = torch.from_numpy(M.lam.copy()).cuda()
        fits = ab.cpd_alto(at, ab.KruskalModel([int(d) for d in dims], rank, dU, dl), 5, 1e-30)
        return fits, [u.cpu().numpy() for u in dU]

    fa, ua = run(0)
    fu, uu = run(1)
    assert np.max(np.abs(fa - fu)) < 1e-6
    for n in range(3):
        assert rel_fro(uu[n], ua[n]) < 1e-4, n
