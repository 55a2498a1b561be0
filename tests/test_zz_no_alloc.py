"""altob_loglik_noalloc: the log-likelihood for callers that cannot call
cudaMalloc (their device memory belongs to their own pool, or the CUDA
allocator must not be entered where they run).  It keeps its scratch in a
fixed array inside the library instead of allocating; its results must equal
those of altob_loglik.  Called through the C ABI, twice in a row, since every
call reuses the same fixed scratch.  This file is collected last."""
import ctypes as C

import numpy as np
import pytest

import alto_b200 as ab
from alto_b200 import synth

pytestmark = pytest.mark.gpu
TOL = {"f64": 1e-12, "f32": 1e-5}  # the parity tests' tolerances per model precision


def _call(fn, at, ftype, U, lam, rank, stream=None):
    ll = C.c_double(0.0)
    ptrs = (C.c_void_p * len(U))(*[u.data_ptr() for u in U])
    st = fn(at.handle, ftype, ptrs, lam.data_ptr(), rank, 1e-10, C.byref(ll), stream)
    assert st == 0, ab.lib().altob_last_error()
    return ll.value


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_loglik_noalloc_matches_loglik_on_two_calls(prec):
    """Two calls in a row with different factors and lambda (the second call
    finds the first one's values in the shared scratch); FP64 and FP32
    models; the second pair runs on a non-default stream."""
    torch = pytest.importorskip("torch")
    dims, cidx, vals = synth.poisson_kruskal((150, 120, 90, 30), 6, 80_000, seed=12)
    at = ab.create_alto(ab.SparseTensor.from_arrays(dims, cidx, vals), 8, 0, val_dtype="u32")
    rank = 16
    L = ab.lib()
    tol = TOL[prec]
    dt = torch.float64 if prec == "f64" else torch.float32
    ftype = ab.F64 if prec == "f64" else ab.F32
    side = torch.cuda.Stream()
    for call in range(2):
        U = synth.random_factors(dims, rank, seed=40 + call)
        lam = np.linspace(0.5, 2.0, rank) * (call + 1)
        UA = [torch.from_numpy(u.copy()).to(dt).cuda() for u in U]
        UB = [torch.from_numpy(u.copy()).to(dt).cuda() for u in U]
        lA = torch.from_numpy(lam.copy()).to(dt).cuda()
        lB = torch.from_numpy(lam.copy()).to(dt).cuda()
        torch.cuda.synchronize()
        stream = None if call == 0 else C.c_void_p(side.cuda_stream)
        want = _call(L.altob_loglik, at, ftype, UA, lA, rank, stream)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        got = _call(L.altob_loglik_noalloc, at, ftype, UB, lB, rank, stream)
        torch.cuda.synchronize()
        # nothing was allocated on the device by the call
        assert torch.cuda.mem_get_info()[0] == free_before
        assert abs(got - want) <= tol * abs(want), (call, got, want)
        for a, b in zip(UA, UB):
            a, b = a.double().cpu().numpy(), b.double().cpu().numpy()
            assert np.linalg.norm(a - b) <= tol * np.linalg.norm(a)
        np.testing.assert_allclose(lB.double().cpu().numpy(), lA.double().cpu().numpy(), rtol=tol)


def test_loglik_noalloc_rejects_rank_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    dims, cidx, vals = synth.poisson_kruskal((40, 30, 20), 3, 5_000, seed=13)
    at = ab.create_alto(ab.SparseTensor.from_arrays(dims, cidx, vals), 4, 0, val_dtype="u32")
    rank = 113
    U = [torch.rand(int(d), rank, dtype=torch.float64, device="cuda") for d in dims]
    lam = torch.ones(rank, dtype=torch.float64, device="cuda")
    ll = C.c_double(0.0)
    ptrs = (C.c_void_p * 3)(*[u.data_ptr() for u in U])
    st = ab.lib().altob_loglik_noalloc(at.handle, ab.F64, ptrs, lam.data_ptr(), rank, 1e-10, C.byref(ll), None)
    assert st == 1  # ALTOB_ERR_ARG
    assert b"maximum rank 112" in ab.lib().altob_last_error()
