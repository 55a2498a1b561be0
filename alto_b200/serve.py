"""Decomposition server (altob_server_*): requests arrive, are admitted
against an HBM budget, run concurrently on worker streams, and CP-ALS
requests queued together are solved as one batch.  No counterpart in the
reference, which decomposes one tensor per cpd64 run.

    srv = Server(hbm_budget_gb=150, workers=4, max_batch=32)
    rid = srv.submit_als(dims, d_cidx, d_vals, rank=32, max_iters=50, tol=1e-4, seed=1)
    res = srv.wait(rid)      # dict: status, fit, iters, batch_size, t_submit, t_start, t_end
    srv.close()

`replay` drives a timed request stream (arrival offsets in seconds) and
returns the per-request results plus latency percentiles and throughput.
"""
from __future__ import annotations

import ctypes as C
import threading
import time

import numpy as np

from . import (F32, F64, U32, Request, Result, ServerConfig, _check, _dev_ptr, lib)

ALS, APR = 0, 1


class Server:
    POLICIES = {"fifo": 0, "least_work": 1}

    def __init__(self, hbm_budget_gb=150.0, workers=4, max_batch=32, use_graph=True, autotune=True, plain=False,
                 policy="fifo"):
        cfg = ServerConfig(int(hbm_budget_gb * (1 << 30)), int(workers), int(max_batch), int(bool(use_graph)),
                           int(bool(autotune)), int(bool(plain)), self.POLICIES[policy])
        h = C.c_void_p()
        _check(lib().altob_server_create(C.byref(cfg), C.byref(h)))
        self.handle = h.value
        self._keep = {}  # request id -> device arrays (alive until waited for)
        self._lock = threading.Lock()

    @staticmethod
    def make_request(kind, dims, d_cidx, d_vals, rank, max_iters, tol, seed, ftype=F32, max_inner=10, nprtn=128):
        r = Request()
        r.kind = kind
        r.nmode = len(dims)
        for m, d in enumerate(dims):
            r.dims[m] = int(d)
        r.nnz = int(d_vals.shape[0])
        r.d_cidx = _dev_ptr(d_cidx)
        r.d_vals = _dev_ptr(d_vals)
        vd = str(d_vals.dtype)
        r.vdtype = F64 if "float64" in vd else F32 if "float32" in vd else U32
        r.ftype = ftype
        r.rank = int(rank)
        r.max_iters = int(max_iters)
        r.max_inner = int(max_inner)
        r.tol = float(tol)
        r.seed = int(seed) & 0xFFFFFFFF
        r.nprtn = int(nprtn)
        return r

    def submit(self, req: Request, keep=None):
        rid = C.c_uint64()
        _check(lib().altob_server_submit(self.handle, C.byref(req), C.byref(rid)))
        with self._lock:
            self._keep[rid.value] = keep
        return rid.value

    def submit_als(self, dims, d_cidx, d_vals, rank, max_iters=50, tol=1e-4, seed=1, ftype=F32):
        return self.submit(self.make_request(ALS, dims, d_cidx, d_vals, rank, max_iters, tol, seed, ftype),
                           (d_cidx, d_vals))

    def submit_apr(self, dims, d_cidx, d_vals, rank, max_iters=50, tol=1e-4, seed=1, ftype=F32, max_inner=10):
        return self.submit(self.make_request(APR, dims, d_cidx, d_vals, rank, max_iters, tol, seed, ftype,
                                             max_inner), (d_cidx, d_vals))

    def wait(self, rid):
        res = Result()
        _check(lib().altob_server_wait(self.handle, C.c_uint64(rid), C.byref(res)))
        with self._lock:
            self._keep.pop(rid, None)
        return {"status": res.status, "iters": res.iters, "batch_size": res.batch_size, "fit": res.fit,
                "loglik": res.loglik, "t_submit": res.t_submit, "t_start": res.t_start, "t_end": res.t_end,
                "latency": res.t_end - res.t_submit}

    def stats(self):
        used, peak = C.c_uint64(), C.c_uint64()
        q, r = C.c_int(), C.c_int()
        _check(lib().altob_server_stats(self.handle, C.byref(used), C.byref(peak), C.byref(q), C.byref(r)))
        return {"used_bytes": used.value, "peak_bytes": peak.value, "queued": q.value, "running": r.value}

    def clock(self):
        return lib().altob_server_clock(self.handle)

    def close(self):
        if getattr(self, "handle", None):
            _check(lib().altob_server_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def footprint(req: Request) -> int:
    b = C.c_uint64()
    _check(lib().altob_request_footprint(C.byref(req), C.byref(b)))
    return b.value


def replay(server: Server, requests, arrivals):
    """Submits requests[k] at server time arrivals[k] (seconds from the first
    submission), waits for all of them, and summarises the run.  Each entry
    of `requests` is (Request, keep-alive object)."""
    t0 = server.clock()
    ids = []
    for (req, keep), at in zip(requests, arrivals):
        while True:
            dt = t0 + at - server.clock()
            if dt <= 0:
                break
            time.sleep(min(dt, 0.002))
        ids.append(server.submit(req, keep))
    results = [server.wait(i) for i in ids]
    lat = np.array([r["latency"] for r in results])
    first = min(r["t_submit"] for r in results)
    last = max(r["t_end"] for r in results)
    ok = sum(1 for r in results if r["status"] == 0)
    return results, {"requests": len(results), "ok": ok, "makespan_s": last - first,
                     "solves_per_s": ok / (last - first) if last > first else None,
                     "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                     "mean_batch": float(np.mean([r["batch_size"] for r in results]))}
