"""Decomposition server on the GPU: every request's result is the same
served in a mix (concurrent workers, CP-ALS requests batched) as served
alone: CP-ALS fit within 1e-4 (FP32) / 1e-9 (FP64), CP-APR log-likelihood
within 1e-4 relative; admission keeps the running footprint inside the HBM
budget."""
import numpy as np
import pytest

import alto_b200 as ab
from alto_b200 import serve, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

STREAM = [  # (kind, dims, nnz, rank)
    ("als", (300, 200, 100), 60_000, 16),
    ("apr", (200, 150, 100, 40), 80_000, 8),
    ("als", (120, 90, 80, 60), 40_000, 32),
    ("als", (2000, 1500, 900), 20_000, 8),
    ("apr", (400, 300, 200), 50_000, 16),
    ("als", (50, 60, 70, 40, 30), 90_000, 16),
    ("als", (800, 700, 600), 150_000, 32),
    ("apr", (100, 90, 80, 70, 20), 60_000, 8),
    ("als", (1000, 40, 50), 30_000, 64),
]


def _inputs(dtype_als):
    out = []
    for k, (kind, dims, nnz, rank) in enumerate(STREAM):
        if kind == "als":
            cidx, vals = synth.uniform_coo_torch(dims, nnz, 500 + k, "cuda")
            vals = vals.to(dtype_als)
        else:
            cidx, vals = synth.poisson_kruskal_torch(dims, 8, nnz, 500 + k, "cuda")
        out.append((kind, dims, cidx, vals, rank))
    return out


def _submit(srv, k, item, ftype):
    kind, dims, cidx, vals, rank = item
    if kind == "als":
        return srv.submit_als(dims, cidx, vals, rank, max_iters=12, tol=1e-30, seed=900 + k, ftype=ftype)
    return srv.submit_apr(dims, cidx, vals, rank, max_iters=6, tol=1e-4, seed=900 + k, ftype=ftype, max_inner=5)


def _mix(items, ftype, **cfg):
    srv = serve.Server(**cfg)
    ids = [_submit(srv, k, it, ftype) for k, it in enumerate(items)]
    res = [srv.wait(i) for i in ids]
    st = srv.stats()
    srv.close()
    return res, st


def _alone(items, ftype):
    srv = serve.Server(workers=1, max_batch=1)
    res = [srv.wait(_submit(srv, k, it, ftype)) for k, it in enumerate(items)]
    srv.close()
    return res


@pytest.mark.parametrize("ftype", [ab.F32, ab.F64])
def test_served_results_same_alone_and_in_mix(ftype):
    items = _inputs(torch.float32 if ftype == ab.F32 else torch.float64)
    mix, _ = _mix(items, ftype, workers=3, max_batch=4)
    alone = _alone(items, ftype)
    assert max(r["batch_size"] for r in mix) > 1  # CP-ALS requests were batched
    tol = 1e-4 if ftype == ab.F32 else 1e-9
    for (kind, *_), m, a in zip(items, mix, alone):
        assert m["status"] == 0 and a["status"] == 0
        assert m["iters"] == a["iters"]
        if kind == "als":
            assert abs(m["fit"] - a["fit"]) < tol
        else:
            assert abs(m["loglik"] - a["loglik"]) <= (1e-4 if ftype == ab.F32 else 1e-9) * abs(a["loglik"])
        assert m["t_submit"] <= m["t_start"] <= m["t_end"]


def test_served_plain_fp64_matches_batched_fp64():
    items = _inputs(torch.float64)
    plain, _ = _mix(items, ab.F64, workers=1, max_batch=1, plain=True)
    batched, _ = _mix(items, ab.F64, workers=2, max_batch=8)
    for (kind, *_), p, b in zip(items, plain, batched):
        if kind == "als":
            assert abs(p["fit"] - b["fit"]) < 1e-9
        else:
            assert abs(p["loglik"] - b["loglik"]) <= 1e-9 * abs(p["loglik"])


def test_admission_respects_budget():
    items = _inputs(torch.float32)
    fps = []
    for k, (kind, dims, cidx, vals, rank) in enumerate(items):
        req = serve.Server.make_request(serve.ALS if kind == "als" else serve.APR, dims, cidx, vals, rank, 12, 1e-30,
                                        900 + k, ab.F32)
        fps.append(serve.footprint(req))
    budget = 1.5 * max(fps)  # at most one or two requests fit at a time
    res, st = _mix(items, ab.F32, workers=4, max_batch=4, hbm_budget_gb=budget / (1 << 30))
    assert all(r["status"] == 0 for r in res)
    assert st["peak_bytes"] <= budget
    assert st["used_bytes"] == 0
    # a request larger than the whole budget is refused, the rest still run
    small = max(fps) * 0.5
    res, _ = _mix(items[:3], ab.F32, workers=2, max_batch=2, hbm_budget_gb=small / (1 << 30))
    for r, fp in zip(res, fps[:3]):
        assert (r["status"] == ab.ERR_NOMEM) == (fp > small)


@pytest.mark.parametrize("policy", ["fifo", "least_work"])
def test_admission_policy_order(policy):
    """One worker, a long CP-APR request queued first and short CP-ALS
    requests behind it: arrival order runs the long one first, least-work
    order runs the short ones first; the results are the same either way."""
    dims = (200, 150, 100, 40)
    cidx, cnt = synth.poisson_kruskal_torch(dims, 8, 400_000, 77, "cuda")
    small = [synth.uniform_coo_torch((60, 50, 40), 5_000, 80 + k, "cuda") for k in range(3)]
    srv = serve.Server(workers=1, max_batch=1, policy=policy)
    # hold the worker with a first request so that the rest queue up together
    hold = srv.submit_apr(dims, cidx, cnt, 8, max_iters=3, tol=0.0, seed=1, max_inner=3)
    big = srv.submit_apr(dims, cidx, cnt, 8, max_iters=8, tol=0.0, seed=2, max_inner=5)
    ids = [srv.submit_als((60, 50, 40), c, v.float(), 8, max_iters=5, tol=0.0, seed=3 + k)
           for k, (c, v) in enumerate(small)]
    res = {i: srv.wait(i) for i in [hold, big] + ids}
    srv.close()
    assert all(r["status"] == 0 for r in res.values())
    short_done = max(res[i]["t_end"] for i in ids)
    if policy == "fifo":
        assert res[big]["t_end"] <= min(res[i]["t_start"] for i in ids)
    else:
        assert short_done <= res[big]["t_start"]
