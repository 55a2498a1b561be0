"""Batched CP-ALS (altob_batch_*) on the GPU.  Every tensor of a batch must
give what a separate altob_cpd_als call gives on the same tensor and
initial model: fits within 1e-9 (FP64) / 1e-4 (FP32, also against the FP64
solve), the same stopping iteration, factors within the stated relative
Frobenius error."""
import numpy as np
import pytest

import alto_b200 as ab
from alto_b200 import synth
from conftest import rel_fro

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

# (dims, nnz, rank): orders 3-5, ranks in every lane class, low-reuse modes
# (nnz / dim <= 4, read through oidx) and high-reuse modes
SHAPES = [
    ((60, 50, 40), 8_000, 8),
    ((400, 30, 20), 20_000, 16),
    ((2000, 1500, 900), 5_000, 32),
    ((80, 70, 60, 20), 30_000, 24),
    ((25, 30, 35, 40, 15), 40_000, 16),
    ((3000, 40, 50), 12_000, 64),
    ((90, 80, 70, 60), 3_000, 8),
    ((30, 20, 25, 10, 12), 25_000, 32),
    ((500, 600, 700), 60_000, 10),
]


def _make(i, val_dtype):
    dims, nnz, rank = SHAPES[i]
    total = int(np.prod(dims))
    dims, cidx, vals = synth.uniform_distinct(dims, min(nnz, total // 2), seed=100 + i)
    at = ab.create_alto(ab.SparseTensor.from_arrays(dims, cidx, vals), 16, 0, val_dtype=val_dtype)
    return dims, at, rank


def _model(dims, rank, seed, dtype):
    M = ab.random_init_factors(dims, rank, seed, dtype=dtype)
    dU = [torch.from_numpy(u.copy()).cuda() for u in M.U]
    dl = torch.from_numpy(M.lam.copy()).cuda()
    return ab.KruskalModel([int(d) for d in dims], rank, dU, dl)


def _solve_each(items, dtype, iters, eps):
    out = []
    for k, (dims, at, rank) in enumerate(items):
        M = _model(dims, rank, 7 + k, dtype)
        fits = ab.cpd_alto(at, M, iters, eps)
        out.append((fits, M))
    return out


def _batch(items, dtype, iters, eps, autotune=False, use_graph=True, seeds=None):
    seeds = seeds if seeds is not None else [7 + k for k in range(len(items))]
    models = [_model(dims, rank, sd, dtype) for sd, (dims, at, rank) in zip(seeds, items)]
    b = ab.BatchCPD([at for _, at, _ in items], models, fit_capacity=iters)
    if autotune:
        b.autotune()
    fits, its = b.solve(iters, eps, use_graph=use_graph)
    b.close()
    return fits, its, models


def _items(dtype):
    vd = "f64" if dtype == np.float64 else "f32"
    return [_make(i, vd) for i in range(len(SHAPES))]


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_fp64_equals_separate_solves(use_graph):
    items = _items(np.float64)
    iters = 8
    ref = _solve_each(items, np.float64, iters, 1e-30)
    fits, its, models = _batch(items, np.float64, iters, 1e-30, use_graph=use_graph)
    for k, (rf, rM) in enumerate(ref):
        assert its[k] == len(rf) == iters
        assert np.max(np.abs(fits[k] - rf)) < 1e-9, k
        for n in range(len(rM.U)):
            assert rel_fro(models[k].U[n].cpu().numpy(), rM.U[n].cpu().numpy()) < 1e-7, (k, n)
        np.testing.assert_allclose(models[k].lam.cpu().numpy(), rM.lam.cpu().numpy(), rtol=1e-7)


def test_batch_fp32_matches_fp64_fit():
    items32 = _items(np.float32)
    items64 = _items(np.float64)
    iters = 10
    ref32 = _solve_each(items32, np.float32, iters, 1e-30)
    ref64 = _solve_each(items64, np.float64, iters, 1e-30)
    fits, its, models = _batch(items32, np.float32, iters, 1e-30, autotune=True)
    for k in range(len(items32)):
        assert its[k] == iters
        assert np.max(np.abs(fits[k] - ref32[k][0])) < 1e-4, k
        assert np.max(np.abs(fits[k] - ref64[k][0])) < 1e-4, k


def test_batch_stopping_rule_per_tensor():
    """Each tensor stops on its own |fit - prev| < eps, as its separate solve does."""
    items = _items(np.float64)
    iters, eps = 40, 1e-4
    ref = _solve_each(items, np.float64, iters, eps)
    fits, its, _ = _batch(items, np.float64, iters, eps)
    assert len(set(int(x) for x in its)) > 1  # the tensors stop at different iterations
    for k, (rf, _) in enumerate(ref):
        assert its[k] == len(rf), k
        np.testing.assert_allclose(fits[k, :its[k]], rf, atol=1e-9)
        assert np.all(fits[k, its[k]:] == 0)


def test_batch_result_same_alone_and_in_mix():
    """FP32: fits alone and in the mix within 1e-4.  FP64: factors too (in
    FP32 the atomics' order differs between the two launches, and random
    rank-16..24 problems amplify that rounding in the factors, not the fit)."""
    items = _items(np.float32)
    iters = 6
    mix_fits, _, _ = _batch(items, np.float32, iters, 1e-30)
    for k in (0, 3, 4):
        alone_fits, _, _ = _batch([items[k]], np.float32, iters, 1e-30, seeds=[7 + k])
        assert np.max(np.abs(alone_fits[0] - mix_fits[k])) < 1e-4
    items = _items(np.float64)
    mix_fits, _, mix_models = _batch(items, np.float64, iters, 1e-30)
    for k in (0, 3, 4):
        alone_fits, _, alone_models = _batch([items[k]], np.float64, iters, 1e-30, seeds=[7 + k])
        assert np.max(np.abs(alone_fits[0] - mix_fits[k])) < 1e-9
        for n in range(len(alone_models[0].U)):
            assert rel_fro(alone_models[0].U[n].cpu().numpy(), mix_models[k].U[n].cpu().numpy()) < 1e-7


def test_batch_autotune_keeps_factors_and_reports_classes():
    items = _items(np.float32)
    models = [_model(dims, rank, 7 + k, np.float32) for k, (dims, at, rank) in enumerate(items)]
    before = [[u.clone() for u in m.U] for m in models]
    b = ab.BatchCPD([at for _, at, _ in items], models, fit_capacity=4)
    b.autotune()
    torch.cuda.synchronize()
    for m, bu in zip(models, before):
        for u, v in zip(m.U, bu):
            assert torch.equal(u, v)
    text = b.describe()
    assert all(f"order={o}" in text for o in (3, 4, 5)) and "tuned_ms" in text
    b.close()


def test_batch_rejects_bad_arguments():
    dims, at, rank = _make(0, "f32")
    dims64, at64, _ = _make(1, "f64")
    m32 = _model(dims, rank, 1, np.float32)
    with pytest.raises(ab.AltobError) as e:  # FP64 model on FP32 values
        ab.BatchCPD([at], [_model(dims, rank, 1, np.float64)])
    assert e.value.status == ab.ERR_UNSUPPORTED
    with pytest.raises(ab.AltobError) as e:  # one value dtype per batch
        ab.BatchCPD([at, at64], [m32, _model(dims64, 4, 1, np.float32)])
    big = _model(dims, 113, 1, np.float32)
    with pytest.raises(ab.AltobError) as e:
        ab.BatchCPD([at], [big])
    assert e.value.status == ab.ERR_UNSUPPORTED
    b = ab.BatchCPD([at], [m32], fit_capacity=3)
    with pytest.raises(ab.AltobError) as e:
        b.solve(4, 0.0)
    assert e.value.status == ab.ERR_ARG
    b.close()


def test_batch_5mode_80bit_low_reuse_vs_reference():
    """A batch holding a 5-mode tensor with 80-bit keys (two index words) whose
    modes all have fiber reuse <= 4 (read through oidx, op_sched), beside two
    other tensors: each tensor's batched FP64 solve against the reference's
    own cpd_alto (oracle/_ref) from the same seeded initial model."""
    orc = pytest.importorskip("oracle.orc")
    if not orc.ref_available():
        pytest.skip("reference library oracle/_ref not built")
    ref = orc.RefLib()
    specs = [((50_000, 45_000, 40_000, 35_000, 60_000), 120_000, 16),
             ((500, 400, 300), 50_000, 8),
             ((3000, 2000, 50, 40), 40_000, 32)]
    items, coo = [], []
    for i, (dims, nnz, rank) in enumerate(specs):
        d, cidx, vals = synth.uniform_distinct(dims, nnz, seed=300 + i)
        at = ab.create_alto(ab.SparseTensor.from_arrays(d, cidx, vals), 16, 0)
        items.append((d, at, rank))
        coo.append((d, cidx, vals))
    info = items[0][1].info()
    assert info["alto_bits"] == 80 and info["lit_bits"] == 128 and info["is_oidx"]
    iters = 6
    fits, its, models = _batch(items, np.float64, iters, 1e-30, seeds=[21, 22, 23])
    for k, ((d, cidx, vals), (_, at, rank)) in enumerate(zip(coo, items)):
        rU, rlam, rfits = ref.cpd(d, cidx, vals, 16, at.info()["lit_bits"], rank, iters, 1e-30, 21 + k)
        assert its[k] == len(rfits) == iters
        assert np.max(np.abs(fits[k][:iters] - rfits)) < 1e-6, (k, fits[k], rfits)
        M = models[k]
        for n in range(len(d)):
            assert rel_fro(M.U[n].cpu().numpy(), rU[n]) < 1e-5, (k, n)
