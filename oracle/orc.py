"""ctypes bindings for the oracle (liborc.so) and the reference harness
(_ref/libaltoref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU legs.  The alto_b200 package never imports this module.

COO tensors are passed as (dims, cidx, vals) with cidx a (nmode, nnz)
uint64 array (0-based) and vals a float64 array.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_SO = os.path.join(HERE, "liborc.so")
REF_SO = os.path.join(HERE, "_ref", "libaltoref.so")
REF_SO_AVX512 = os.path.join(HERE, "_ref", "libaltoref_avx512.so")
REF_SO_PEXT = os.path.join(HERE, "_ref", "libaltoref_pext.so")
REF_SO_OPT = os.path.join(HERE, "_ref", "libaltoref_opt.so")
_AVX512 = ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl")


def host_isa():
    """'avx512' when the host CPU has the x86-64-v4 extensions, else 'avx2'."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    return "avx512" if all(x in flags for x in _AVX512) else "avx2"
    except OSError:
        pass
    return "unknown"


def ref_default_path():
    """The reference build for this host: x86-64-v4 (AVX-512) where the CPU
    has it (the reference's own -march=native would use it), else x86-64-v3."""
    if host_isa() == "avx512" and os.path.exists(REF_SO_AVX512):
        return REF_SO_AVX512
    return REF_SO

_u64p = C.POINTER(C.c_uint64)
_f64p = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int)


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _ptr_array(mats):
    arr = (C.POINTER(C.c_double) * len(mats))()
    for i, m in enumerate(mats):
        assert m.dtype == np.float64 and m.flags.c_contiguous
        arr[i] = m.ctypes.data_as(_f64p)
    return arr


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE, "liborc.so"], check=True)


def _coo_args(dims, cidx, vals):
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    cidx = np.ascontiguousarray(cidx, dtype=np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    nmode = dims.shape[0]
    assert cidx.shape == (nmode, vals.shape[0])
    return dims, cidx, vals, nmode, vals.shape[0]


class Oracle:
    """The CPU restatement (oracle/alto_oracle.c)."""

    def __init__(self):
        if not os.path.exists(ORC_SO) or os.path.getmtime(ORC_SO) < os.path.getmtime(
            os.path.join(HERE, "alto_oracle.c")
        ):
            build_oracle()
        L = C.CDLL(ORC_SO)
        L.orc_create.restype = C.c_int
        L.orc_create.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p, _f64p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_info.argtypes = [C.c_void_p, _i32p]
        L.orc_dump.argtypes = [C.c_void_p, _u64p, _f64p, _u64p, _u64p, _u64p, _u64p, _u64p]
        L.orc_mttkrp.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_uint64]
        L.orc_mttkrp_coo.argtypes = [C.c_int, C.c_uint64, _u64p, _f64p, C.c_int, C.c_void_p, C.c_uint64]
        L.orc_random_init.argtypes = [C.c_int, _u64p, C.c_uint64, C.c_uint, C.c_void_p, _f64p]
        L.orc_cpd_als.restype = C.c_int
        L.orc_cpd_als.argtypes = [C.c_void_p, C.c_void_p, _f64p, C.c_uint64, C.c_int, C.c_double, _f64p]
        L.orc_cp_apr.restype = C.c_int
        L.orc_cp_apr.argtypes = [C.c_void_p, C.c_void_p, _f64p, C.c_uint64, C.c_int, C.c_int, C.c_double,
                                 C.c_double, C.c_double, C.c_double, C.c_int, _f64p, _f64p]
        L.orc_phi.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_uint64, C.c_double, _f64p]
        L.orc_loglik.restype = C.c_double
        L.orc_loglik.argtypes = [C.c_void_p, C.c_void_p, _f64p, C.c_uint64, C.c_double]
        L.orc_gram.argtypes = [_f64p, C.c_uint64, C.c_uint64, _f64p]
        L.orc_pseudo_inverse.restype = C.c_int
        L.orc_pseudo_inverse.argtypes = [_f64p, C.c_int, C.c_int, _f64p, C.c_uint64, C.c_uint64]
        self.L = L

    # -- encoding --
    def create(self, dims, cidx, vals, nprtn, lit_bits):
        dims, cidx, vals, nmode, nnz = _coo_args(dims, cidx, vals)
        h = C.c_void_p()
        rc = self.L.orc_create(nmode, _p(dims, _u64p), nnz, _p(cidx, _u64p), _p(vals, _f64p),
                               int(nprtn), int(lit_bits), C.byref(h))
        if rc != 0:
            raise ValueError(f"orc_create failed rc={rc}")
        return OracleTensor(self, h, dims, nnz, nprtn)

    def pseudo_inverse(self, grams, mode, U):
        """U <- U V^-1 (or V^+), V = Hadamard of the Grams but `mode`; returns
        (U, used_pseudo_inverse)."""
        grams = np.ascontiguousarray(grams, dtype=np.float64)
        U = np.ascontiguousarray(U, dtype=np.float64).copy()
        used = self.L.orc_pseudo_inverse(_p(grams, _f64p), grams.shape[0], mode, _p(U, _f64p), U.shape[0], U.shape[1])
        return U, bool(used)

    def random_init(self, dims, rank, seed):
        dims = np.ascontiguousarray(dims, dtype=np.uint64)
        U = [np.zeros((int(d), rank)) for d in dims]
        lam = np.zeros(rank)
        self.L.orc_random_init(len(dims), _p(dims, _u64p), rank, seed, _ptr_array(U), _p(lam, _f64p))
        return U, lam

    def mttkrp_coo(self, dims, cidx, vals, mode, factors, rank):
        dims, cidx, vals, nmode, nnz = _coo_args(dims, cidx, vals)
        self.L.orc_mttkrp_coo(nmode, nnz, _p(cidx, _u64p), _p(vals, _f64p), mode, _ptr_array(factors), rank)

    def gram(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        G = np.zeros((U.shape[1], U.shape[1]))
        self.L.orc_gram(_p(U, _f64p), U.shape[0], U.shape[1], _p(G, _f64p))
        return G


class OracleTensor:
    def __init__(self, orc, h, dims, nnz, nprtn):
        self.orc, self.h, self.dims, self.nnz, self.nprtn = orc, h, dims, nnz, nprtn
        self.nmode = len(dims)

    def __del__(self):
        try:
            self.orc.L.orc_destroy(self.h)
        except Exception:
            pass

    def dump(self):
        nm, nnz, np_ = self.nmode, self.nnz, self.nprtn
        info = np.zeros(4, dtype=np.int32)
        self.orc.L.orc_info(self.h, _p(info, _i32p))
        out = dict(
            idx=np.zeros((nnz, 2), np.uint64), vals=np.zeros(nnz), prtn_ptr=np.zeros(np_ + 1, np.uint64),
            intervals=np.zeros((np_, nm, 2), np.uint64), masks=np.zeros((nm, 2), np.uint64),
            cr_masks=np.zeros((nm, 2), np.uint64), oidx=np.zeros((nm, nnz), np.uint64),
        )
        L = self.orc.L
        L.orc_dump(self.h, _p(out["idx"], _u64p), _p(out["vals"], _f64p), _p(out["prtn_ptr"], _u64p),
                   _p(out["intervals"], _u64p), _p(out["masks"], _u64p), _p(out["cr_masks"], _u64p),
                   _p(out["oidx"], _u64p))
        out["alto_bits"] = int(info[0])
        out["is_oidx"] = int(info[1])
        return out

    def mttkrp(self, mode, factors, rank):
        self.orc.L.orc_mttkrp(self.h, mode, _ptr_array(factors), rank)

    def cpd_als(self, U, lam, rank, max_iters, eps):
        fits = np.zeros(max_iters)
        it = self.orc.L.orc_cpd_als(self.h, _ptr_array(U), _p(lam, _f64p), rank, max_iters, eps, _p(fits, _f64p))
        return fits[:it]

    def cp_apr(self, U, lam, rank, max_iters, max_inner, eps=1e-5, eps_div_zero=1e-10, kappa_tol=1e-10,
               kappa=1e-2, dobench=False):
        out = np.zeros(8)
        kkt = np.zeros(max_iters)
        self.orc.L.orc_cp_apr(self.h, _ptr_array(U), _p(lam, _f64p), rank, max_iters, max_inner, eps,
                              eps_div_zero, kappa_tol, kappa, int(bool(dobench)), _p(out, _f64p), _p(kkt, _f64p))
        return dict(loglik=out[0], fit=out[1], kkt=out[2], outer=int(out[3]), inner=int(out[4]), kkt_trace=kkt)

    def phi(self, mode, U, rank, eps_div_zero=1e-10):
        out = np.zeros((int(self.dims[mode]), rank))
        self.orc.L.orc_phi(self.h, mode, _ptr_array(U), rank, eps_div_zero, _p(out, _f64p))
        return out

    def loglik(self, U, lam, rank, eps_div_zero=1e-10):
        return self.orc.L.orc_loglik(self.h, _ptr_array(U), _p(lam, _f64p), rank, eps_div_zero)


def ref_available():
    return os.path.exists(REF_SO)


class RefLib:
    """The reference itself, compiled by oracle/build_ref.sh."""

    def __init__(self, path=None):
        path = path or ref_default_path()
        self.path = path
        self.march = "x86-64-v4" if path == REF_SO_AVX512 else "x86-64-v3"
        L = C.CDLL(path)
        L.ref_max_threads.restype = C.c_int
        L.ref_create_dump.restype = C.c_int
        L.ref_create_dump.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p, _f64p, C.c_int, C.c_int, _u64p, _f64p,
                                      _u64p, _u64p, _u64p, _u64p, _u64p, _i32p]
        L.ref_mttkrp.restype = C.c_int
        L.ref_mttkrp.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p, _f64p, C.c_int, C.c_int, C.c_int,
                                 C.c_void_p, C.c_uint64]
        L.ref_cpd.restype = C.c_int
        L.ref_cpd.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p, _f64p, C.c_int, C.c_int, C.c_uint64, C.c_int,
                              C.c_double, C.c_uint, C.c_void_p, _f64p, _f64p]
        L.ref_apr.restype = C.c_int
        L.ref_apr.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p, _f64p, C.c_int, C.c_int, C.c_uint64, C.c_int,
                              C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_uint,
                              C.c_void_p, _f64p, _f64p]
        L.ref_bench_mttkrp.restype = C.c_double
        L.ref_bench_mttkrp.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p, _f64p, C.c_int, C.c_int, C.c_uint64,
                                       C.c_int, C.c_uint, _f64p]
        self.L = L

    def max_threads(self):
        return self.L.ref_max_threads()

    def create_dump(self, dims, cidx, vals, nprtn, lit_bits):
        dims, cidx, vals, nm, nnz = _coo_args(dims, cidx, vals)
        out = dict(
            idx=np.zeros((nnz, 2), np.uint64), vals=np.zeros(nnz), prtn_ptr=np.zeros(nprtn + 1, np.uint64),
            intervals=np.zeros((nprtn, nm, 2), np.uint64), masks=np.zeros((nm, 2), np.uint64),
            cr_masks=np.zeros((nm, 2), np.uint64), oidx=np.zeros((nm, nnz), np.uint64),
        )
        info = np.zeros(4, np.int32)
        self.L.ref_create_dump(nm, _p(dims, _u64p), nnz, _p(cidx, _u64p), _p(vals, _f64p), nprtn, lit_bits,
                               _p(out["idx"], _u64p), _p(out["vals"], _f64p), _p(out["prtn_ptr"], _u64p),
                               _p(out["intervals"], _u64p), _p(out["masks"], _u64p), _p(out["cr_masks"], _u64p),
                               _p(out["oidx"], _u64p), _p(info, _i32p))
        out["alto_bits"] = int(info[0])
        out["is_oidx"] = int(info[1])
        return out

    def mttkrp(self, dims, cidx, vals, nprtn, lit_bits, mode, factors, rank):
        dims, cidx, vals, nm, nnz = _coo_args(dims, cidx, vals)
        self.L.ref_mttkrp(nm, _p(dims, _u64p), nnz, _p(cidx, _u64p), _p(vals, _f64p), nprtn, lit_bits, mode,
                          _ptr_array(factors), rank)

    def cpd(self, dims, cidx, vals, nprtn, lit_bits, rank, max_iters, eps, seed):
        dims, cidx, vals, nm, nnz = _coo_args(dims, cidx, vals)
        U = [np.zeros((int(d), rank)) for d in dims]
        lam = np.zeros(rank)
        fits = np.zeros(max_iters)
        it = self.L.ref_cpd(nm, _p(dims, _u64p), nnz, _p(cidx, _u64p), _p(vals, _f64p), nprtn, lit_bits, rank,
                            max_iters, eps, seed, _ptr_array(U), _p(lam, _f64p), _p(fits, _f64p))
        return U, lam, fits[:it]

    def apr(self, dims, cidx, vals, nprtn, lit_bits, rank, max_iters, max_inner, eps, eps_div_zero, kappa_tol,
            kappa, dobench, seed):
        dims, cidx, vals, nm, nnz = _coo_args(dims, cidx, vals)
        U = [np.zeros((int(d), rank)) for d in dims]
        lam = np.zeros(rank)
        s = np.zeros(8)
        self.L.ref_apr(nm, _p(dims, _u64p), nnz, _p(cidx, _u64p), _p(vals, _f64p), nprtn, lit_bits, rank,
                       max_iters, max_inner, eps, eps_div_zero, kappa_tol, kappa, int(bool(dobench)), seed,
                       _ptr_array(U), _p(lam, _f64p), _p(s, _f64p))
        return U, lam, dict(loglik=s[0], fit=s[1], kkt=s[2], outer=int(s[3]), inner=int(s[4]))

    def read(self, path, binary=False, zero_based=0):
        """The reference's ImportSparseTensor: (dims, cidx (modes x nnz), vals)."""
        L = self.L
        L.ref_read_open.restype = C.c_void_p
        L.ref_read_open.argtypes = [C.c_char_p, C.c_int, C.c_uint64, _i32p, _u64p]
        L.ref_read_take.restype = None
        L.ref_read_take.argtypes = [C.c_void_p, _u64p, _u64p, _f64p]
        nm = np.zeros(1, np.int32)
        nnz = np.zeros(1, np.uint64)
        h = L.ref_read_open(path.encode(), int(bool(binary)), int(zero_based), _p(nm, _i32p), _p(nnz, _u64p))
        n, z = int(nm[0]), int(nnz[0])
        dims = np.zeros(n, np.uint64)
        cidx = np.zeros((n, z), np.uint64)
        vals = np.zeros(z)
        L.ref_read_take(h, _p(dims, _u64p), _p(cidx, _u64p), _p(vals, _f64p))
        return dims, cidx, vals

    def write(self, path, dims, cidx, vals, binary=False):
        """The reference's ExportSparseTensor of a COO tensor (cidx: modes x nnz)."""
        L = self.L
        L.ref_write.restype = None
        L.ref_write.argtypes = [C.c_char_p, C.c_int, C.c_int, _u64p, C.c_uint64, _u64p, _f64p]
        dims, cidx, vals, nm, nnz = _coo_args(dims, cidx, vals)
        L.ref_write(path.encode(), int(bool(binary)), nm, _p(dims, _u64p), nnz, _p(cidx, _u64p), _p(vals, _f64p))

    def prtn_ids(self, dims, cidx, vals, nprtn, lit_bits):
        """OPT_ALTO partition ids (a -DOPT_ALTO build only)."""
        dims, cidx, vals, nm, nnz = _coo_args(dims, cidx, vals)
        L = self.L
        L.ref_prtn_ids.restype = C.c_int
        L.ref_prtn_ids.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p, _f64p, C.c_int, C.c_int, _u64p, _u64p, _u64p]
        pid, pm = np.zeros(nprtn, np.uint64), np.zeros(nprtn, np.uint64)
        mm = np.zeros((nprtn, nm), np.uint64)
        rc = L.ref_prtn_ids(nm, _p(dims, _u64p), nnz, _p(cidx, _u64p), _p(vals, _f64p), nprtn, lit_bits,
                            _p(pid, _u64p), _p(pm, _u64p), _p(mm, _u64p))
        if rc != 0:
            raise RuntimeError("this reference build has no OPT_ALTO")
        return dict(prtn_id=pid, prtn_mask=pm, prtn_mode_masks=mm)

    def bench_mttkrp(self, dims, cidx, vals, nprtn, lit_bits, rank, iters, seed):
        dims, cidx, vals, nm, nnz = _coo_args(dims, cidx, vals)
        cs = np.zeros(1)
        t = self.L.ref_bench_mttkrp(nm, _p(dims, _u64p), nnz, _p(cidx, _u64p), _p(vals, _f64p), nprtn, lit_bits,
                                    rank, iters, seed, _p(cs, _f64p))
        return t, float(cs[0])


REF_SO_POISSON = os.path.join(HERE, "_ref", "libaltoref_poisson.so")


class RefPoisson:
    """The reference's own Poisson generator (PoissonGeneratorRun,
    src/poisson_generator.cpp:337-375), compiled by oracle/build_ref.sh."""

    def __init__(self, path=REF_SO_POISSON):
        L = C.CDLL(path)
        L.refp_run.restype = C.c_void_p
        L.refp_run.argtypes = [C.c_int, _u64p, C.c_uint64, C.c_uint64, C.c_int, _u64p, C.c_void_p, _f64p]
        L.refp_take.restype = None
        L.refp_take.argtypes = [C.c_void_p, _u64p, _f64p]
        self.L = L

    def run(self, dims, num_edges, rank, nthreads):
        """(cidx (modes x nnz), vals, U list, lambda) for `nthreads` OpenMP threads."""
        dims = np.ascontiguousarray(dims, np.uint64)
        nm = dims.shape[0]
        U = [np.zeros((int(d), rank)) for d in dims]
        lam = np.zeros(rank)
        nnz = np.zeros(1, np.uint64)
        h = self.L.refp_run(nm, _p(dims, _u64p), int(num_edges), int(rank), int(nthreads), _p(nnz, _u64p),
                            _ptr_array(U), _p(lam, _f64p))
        z = int(nnz[0])
        cidx = np.zeros((nm, z), np.uint64)
        vals = np.zeros(z)
        self.L.refp_take(h, _p(cidx, _u64p), _p(vals, _f64p))
        return cidx, vals, U, lam
