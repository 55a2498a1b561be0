"""alto_b200 -- B200-native ALTO: linearized sparse-tensor build, MTTKRP on
every mode from one tensor copy, CP-ALS and CP-APR, behind the reference's
operator names (IntelLabs/ALTO v0.1.2):

    create_alto        include/alto.hpp:108     -> create_alto()
    mttkrp_alto_par    include/alto.hpp:617     -> mttkrp_alto_par()
    cpd_alto           include/cpd.hpp:43       -> cpd_alto()
    cp_apr_alto        include/apr.hpp:984      -> cp_apr_alto()
    ImportSparseTensor src/sptensor.cpp:165     -> ImportSparseTensor()
    KruskalModelRandomInit src/kruskal_model.cpp:109 -> KruskalModelRandomInit()

Everything runs through the C ABI of libaltob.so (include/altob.h).  There
is no CPU fallback: if the library or a CUDA device is missing, the calls
raise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaltob.so")

F64, F32, U32 = 0, 1, 2
_DT = {"f64": F64, "float64": F64, "f32": F32, "float32": F32, "u32": U32, "uint32": U32}
_NP = {F64: np.float64, F32: np.float32, U32: np.uint32}
ALGOS = {"auto": 0, "tiled": 1, "atomic": 2, "atomic_cr": 3, "op_sched": 4}
MAX_MODES = 5
# altob_status codes (include/altob.h)
OK, ERR_ARG, ERR_BITS, ERR_CUDA, ERR_NOMEM, ERR_IO, ERR_UNSUPPORTED, ERR_NOT_FOUND = range(8)


class AltobError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"altob error {status}: {msg}")
        self.status = status


class _Info(C.Structure):
    _fields_ = [
        ("nmode", C.c_int), ("nprtn", C.c_int), ("lit_bits", C.c_int), ("alto_bits", C.c_int),
        ("is_oidx", C.c_int), ("val_dtype", C.c_int), ("nnz", C.c_uint64),
        ("dims", C.c_uint64 * MAX_MODES), ("mode_masks", (C.c_uint64 * 2) * MAX_MODES),
        ("cr_masks", (C.c_uint64 * 2) * MAX_MODES), ("alto_mask", C.c_uint64 * 2),
        ("alto_cr_mask", C.c_uint64 * 2), ("device_bytes", C.c_uint64), ("key_bytes", C.c_uint64),
        ("nruns", C.c_int), ("plan_modes", C.c_int), ("plan_bytes", C.c_uint64), ("tma_err", C.c_int),
    ]


class _Coo(C.Structure):
    _fields_ = [("nmode", C.c_int), ("nnz", C.c_uint64), ("dims", C.c_uint64 * MAX_MODES),
                ("cidx", C.POINTER(C.c_uint64)), ("vals", C.POINTER(C.c_double))]


_lib = None


class Request(C.Structure):
    """altob_request (include/altob.h)."""
    _fields_ = [("kind", C.c_int), ("nmode", C.c_int), ("dims", C.c_uint64 * MAX_MODES), ("nnz", C.c_uint64),
                ("d_cidx", C.c_void_p), ("d_vals", C.c_void_p), ("vdtype", C.c_int), ("ftype", C.c_int),
                ("rank", C.c_uint64), ("max_iters", C.c_int), ("max_inner", C.c_int), ("tol", C.c_double),
                ("seed", C.c_uint), ("nprtn", C.c_int)]


class Result(C.Structure):
    """altob_result (include/altob.h)."""
    _fields_ = [("status", C.c_int), ("iters", C.c_int), ("batch_size", C.c_int), ("fit", C.c_double),
                ("loglik", C.c_double), ("t_submit", C.c_double), ("t_start", C.c_double), ("t_end", C.c_double)]


class ServerConfig(C.Structure):
    """altob_server_config (include/altob.h)."""
    _fields_ = [("hbm_budget", C.c_uint64), ("workers", C.c_int), ("max_batch", C.c_int), ("use_graph", C.c_int),
                ("autotune", C.c_int), ("plain", C.c_int), ("policy", C.c_int)]

# name -> (restype, argtypes); the exported C ABI of include/altob.h
_vp, _u64, _i, _d = C.c_void_p, C.c_uint64, C.c_int, C.c_double
_u64p, _dp = C.POINTER(C.c_uint64), C.POINTER(C.c_double)
SIGNATURES = {
    "altob_status_string": (C.c_char_p, [_i]),
    "altob_last_error": (C.c_char_p, []),
    "altob_version": (C.c_char_p, []),
    "altob_create": (_i, [_i, _u64p, _u64, _u64p, _vp, _i, _i, _i, _vp, C.POINTER(_vp)]),
    "altob_create_device": (_i, [_i, _u64p, _u64, _vp, _vp, _i, _i, _i, _vp, C.POINTER(_vp)]),
    "altob_destroy": (_i, [_vp]),
    "altob_slice": (_i, [_vp, _u64, _u64, _i, _vp, C.POINTER(_vp)]),
    "altob_dump_alt_pext": (_i, [_vp, _u64p, _u64p, C.POINTER(_i), _vp]),
    "altob_partition_ids": (_i, [_vp, _u64p, _u64p, _u64p, _vp]),
    "altob_cpd_als_sharded": (_i, [_vp, _i, _vp, _vp, _u64, _i, _d, _dp, C.POINTER(_i), _vp, _vp, _vp]),
    "altob_get_info": (_i, [_vp, C.POINTER(_Info)]),
    "altob_dump": (_i, [_vp, _u64p, _vp, _u64p, _u64p, _u64p, _vp]),
    "altob_mttkrp": (_i, [_vp, _i, _i, _vp, _u64, _i, _i, _vp]),
    "altob_mttkrp_host": (_i, [_vp, _i, _i, _vp, _u64, _i, _vp]),
    "altob_mttkrp_sweep_host": (_i, [_vp, _i, _vp, _u64, _i, _i, _vp]),
    "altob_cpd_als": (_i, [_vp, _i, _vp, _vp, _u64, _i, _d, _dp, C.POINTER(_i), _vp]),
    "altob_cp_apr": (_i, [_vp, _i, _vp, _vp, _u64, _i, _i, _d, _d, _d, _d, _i, _dp, _vp]),
    "altob_phi": (_i, [_vp, _i, _i, _vp, _u64, _d, _vp, _vp]),
    "altob_loglik": (_i, [_vp, _i, _vp, _vp, _u64, _d, _dp, _vp]),
    "altob_loglik_noalloc": (_i, [_vp, _i, _vp, _vp, _u64, _d, _dp, _vp]),
    "altob_read_tns": (_i, [C.c_char_p, _i, C.POINTER(C.POINTER(_Coo))]),
    "altob_read_bin": (_i, [C.c_char_p, C.POINTER(C.POINTER(_Coo))]),
    "altob_write_bin": (_i, [C.c_char_p, C.POINTER(_Coo)]),
    "altob_write_tns": (_i, [C.c_char_p, C.POINTER(_Coo)]),
    "altob_coo_free": (None, [C.POINTER(_Coo)]),
    "altob_cpd_als_host": (_i, [_vp, _i, _vp, _vp, _u64, _i, _d, _dp, C.POINTER(_i), _vp]),
    "altob_cp_apr_host": (_i, [_vp, _i, _vp, _vp, _u64, _i, _i, _d, _d, _d, _d, _i, _dp, _vp]),
    "altob_kruskal_random_init": (_i, [_i, _u64p, _u64, C.c_uint, _i, _vp, _vp]),
    "altob_poisson_tensor": (_i, [_i, _u64p, _u64, _u64, _i, _vp, _dp, C.POINTER(C.POINTER(_Coo)), _vp]),
    "altob_pseudo_inverse": (_i, [_vp, _i, _i, _u64, _vp, _u64, _i, C.POINTER(_i), _vp]),
    "altob_batch_create": (_i, [_vp, _i, _u64p, _i, _vp, _vp, _i, _vp, C.POINTER(_vp)]),
    "altob_batch_autotune": (_i, [_vp, _i, _vp]),
    "altob_batch_cpd_als": (_i, [_vp, _i, _d, _dp, C.POINTER(_i), _i, _vp]),
    "altob_batch_describe": (_i, [_vp, C.c_char_p, C.c_size_t]),
    "altob_batch_destroy": (_i, [_vp]),
    "altob_request_footprint": (_i, [C.POINTER(Request), _u64p]),
    "altob_server_create": (_i, [C.POINTER(ServerConfig), C.POINTER(_vp)]),
    "altob_server_clock": (C.c_double, [_vp]),
    "altob_server_submit": (_i, [_vp, C.POINTER(Request), _u64p]),
    "altob_server_wait": (_i, [_vp, C.c_uint64, C.POINTER(Result)]),
    "altob_server_stats": (_i, [_vp, _u64p, _u64p, C.POINTER(_i), C.POINTER(_i)]),
    "altob_server_destroy": (_i, [_vp]),
}


def lib():
    """Loads libaltob.so (built in-tree by `make -C alto_b200`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {HERE}`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        L = lib()
        raise AltobError(status, f"{L.altob_status_string(status).decode()}: {L.altob_last_error().decode()}")


def _stream_ptr(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


def _dev_ptr(x):
    """Device pointer of a torch CUDA tensor or a raw integer address."""
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise ValueError("expected a CUDA tensor")
        if not x.is_contiguous():
            raise ValueError("expected a contiguous tensor")
        return x.data_ptr()
    raise TypeError(f"not a device array: {type(x)}")


def _ptr_array(ptrs):
    arr = (C.c_void_p * len(ptrs))()
    for i, p in enumerate(ptrs):
        arr[i] = p
    return arr


# --------------------------------------------------------------------------
# Sparse tensors (SparseTensor, include/sptensor.hpp:8-25)

@dataclass
class SparseTensor:
    dims: np.ndarray           # uint64 [nmodes]
    cidx: np.ndarray           # uint64 [nmodes, nnz], 0-based
    vals: np.ndarray           # float64 [nnz]

    @property
    def nmodes(self):
        return int(self.dims.shape[0])

    @property
    def nnz(self):
        return int(self.vals.shape[0])

    @staticmethod
    def from_arrays(dims, cidx, vals):
        return SparseTensor(np.ascontiguousarray(dims, np.uint64), np.ascontiguousarray(cidx, np.uint64),
                            np.ascontiguousarray(vals, np.float64))


def _coo_to_tensor(p):
    c = p.contents
    nm, nnz = c.nmode, c.nnz
    dims = np.array([c.dims[i] for i in range(nm)], np.uint64)
    cidx = np.ctypeslib.as_array(c.cidx, shape=(nm * nnz,)).reshape(nm, nnz).copy() if nnz else \
        np.zeros((nm, 0), np.uint64)
    vals = np.ctypeslib.as_array(c.vals, shape=(nnz,)).copy() if nnz else np.zeros(0)
    lib().altob_coo_free(p)
    return SparseTensor(dims, cidx, vals)


TEXT_FORMAT, BINARY_FORMAT = 0, 1


def ImportSparseTensor(path, fmt=TEXT_FORMAT, zero_based=0):
    """ImportSparseTensor (src/sptensor.cpp:165-258)."""
    p = C.POINTER(_Coo)()
    if fmt == TEXT_FORMAT:
        _check(lib().altob_read_tns(path.encode(), int(zero_based), C.byref(p)))
    else:
        _check(lib().altob_read_bin(path.encode(), C.byref(p)))
    return _coo_to_tensor(p)


def ExportSparseTensor(path, fmt, X: SparseTensor):
    """ExportSparseTensor (src/sptensor.cpp:23-70)."""
    coo = _Coo()
    coo.nmode = X.nmodes
    coo.nnz = X.nnz
    for i in range(X.nmodes):
        coo.dims[i] = int(X.dims[i])
    cidx = np.ascontiguousarray(X.cidx, np.uint64)
    vals = np.ascontiguousarray(X.vals, np.float64)
    coo.cidx = cidx.ctypes.data_as(_u64p)
    coo.vals = vals.ctypes.data_as(_dp)
    if fmt == TEXT_FORMAT:
        _check(lib().altob_write_tns(path.encode(), C.byref(coo)))
    else:
        _check(lib().altob_write_bin(path.encode(), C.byref(coo)))


# --------------------------------------------------------------------------
# ALTO tensors (AltoTensor<LIT>, include/alto.hpp:27-54)

class AltoTensor:
    """Device-resident ALTO encoding; owns an altob_tensor handle."""

    def __init__(self, handle):
        self._h = handle

    @property
    def handle(self):
        if not self._h:
            raise ValueError("tensor destroyed")
        return self._h

    def info(self):
        inf = _Info()
        _check(lib().altob_get_info(self.handle, C.byref(inf)))
        nm = inf.nmode
        return dict(
            nmode=nm, nprtn=inf.nprtn, lit_bits=inf.lit_bits, alto_bits=inf.alto_bits, is_oidx=inf.is_oidx,
            val_dtype=inf.val_dtype, nnz=inf.nnz, dims=[inf.dims[i] for i in range(nm)],
            masks=np.array([[inf.mode_masks[i][0], inf.mode_masks[i][1]] for i in range(nm)], np.uint64),
            cr_masks=np.array([[inf.cr_masks[i][0], inf.cr_masks[i][1]] for i in range(nm)], np.uint64),
            alto_mask=(inf.alto_mask[0], inf.alto_mask[1]), device_bytes=inf.device_bytes,
            key_bytes=inf.key_bytes, nruns=inf.nruns, plan_modes=inf.plan_modes, plan_bytes=inf.plan_bytes,
            tma_err=inf.tma_err,
        )

    def dump_alt_pext(self, stream=None):
        """The keys, mode masks and field positions of the reference's
        ALT_PEXT encoding (altob_dump_alt_pext)."""
        inf = self.info()
        nnz, nm = inf["nnz"], inf["nmode"]
        idx = np.zeros((nnz, 2), np.uint64)
        masks = np.zeros((nm, 2), np.uint64)
        pos = (C.c_int * nm)()
        _check(lib().altob_dump_alt_pext(self.handle, idx.ctypes.data_as(_u64p), masks.ctypes.data_as(_u64p), pos,
                                         _stream_ptr(stream)))
        return dict(idx=idx, masks=masks, mode_pos=list(pos))

    def partition_ids(self, stream=None):
        """OPT_ALTO partition subspace ids, masks and mode masks
        (altob_partition_ids)."""
        inf = self.info()
        npr, nm = inf["nprtn"], inf["nmode"]
        pid, pmask = np.zeros(npr, np.uint64), np.zeros(npr, np.uint64)
        mm = np.zeros((npr, nm), np.uint64)
        _check(lib().altob_partition_ids(self.handle, pid.ctypes.data_as(_u64p), pmask.ctypes.data_as(_u64p),
                                         mm.ctypes.data_as(_u64p), _stream_ptr(stream)))
        return dict(prtn_id=pid, prtn_mask=pmask, prtn_mode_masks=mm)

    def slice(self, begin, end, nprtn, stream=None):
        """Nonzeros [begin, end) of the ALTO stream as a tensor of its own
        (one GPU's share of a sharded solve; altob_slice)."""
        h = C.c_void_p()
        _check(lib().altob_slice(self.handle, int(begin), int(end), int(nprtn), _stream_ptr(stream), C.byref(h)))
        return AltoTensor(h)

    @property
    def nmode(self):
        return self.info()["nmode"]

    @property
    def dims(self):
        return self.info()["dims"]

    def dump(self, stream=None):
        """Encoding in the reference layout (idx words, vals, prtn_ptr,
        intervals, oidx)."""
        inf = self.info()
        nnz, nm, np_ = inf["nnz"], inf["nmode"], inf["nprtn"]
        idx = np.zeros((nnz, 2), np.uint64)
        vals = np.zeros(nnz, _NP[inf["val_dtype"]])
        prtn = np.zeros(np_ + 1, np.uint64)
        iv = np.zeros((np_, nm, 2), np.uint64)
        oidx = np.zeros((nm, nnz), np.uint64)
        _check(lib().altob_dump(self.handle, idx.ctypes.data_as(_u64p), vals.ctypes.data_as(C.c_void_p),
                                prtn.ctypes.data_as(_u64p), iv.ctypes.data_as(_u64p), oidx.ctypes.data_as(_u64p),
                                _stream_ptr(stream)))
        return dict(idx=idx, vals=vals, prtn_ptr=prtn, intervals=iv, oidx=oidx, masks=inf["masks"],
                    cr_masks=inf["cr_masks"], alto_bits=inf["alto_bits"], is_oidx=inf["is_oidx"])

    def destroy(self):
        if self._h:
            lib().altob_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def create_alto(X: SparseTensor, nprtn: int, lit_bits: int = 0, val_dtype="f64", stream=None) -> AltoTensor:
    """create_alto (include/alto.hpp:108-294) from a host COO tensor."""
    vdt = _DT[val_dtype] if isinstance(val_dtype, str) else int(val_dtype)
    dims = np.ascontiguousarray(X.dims, np.uint64)
    cidx = np.ascontiguousarray(X.cidx, np.uint64)
    vals = np.ascontiguousarray(X.vals, _NP[vdt])
    h = C.c_void_p()
    _check(lib().altob_create(X.nmodes, dims.ctypes.data_as(_u64p), X.nnz, cidx.ctypes.data_as(_u64p),
                              vals.ctypes.data_as(C.c_void_p), vdt, int(nprtn), int(lit_bits),
                              _stream_ptr(stream), C.byref(h)))
    return AltoTensor(h)


def create_alto_device(nmodes, dims, nnz, d_cidx, d_vals, nprtn, lit_bits=0, val_dtype="f64", stream=None):
    """create_alto from device-resident COO arrays (torch tensors or raw
    pointers): d_cidx uint64 [nmodes*nnz], d_vals in val_dtype."""
    vdt = _DT[val_dtype] if isinstance(val_dtype, str) else int(val_dtype)
    dims = np.ascontiguousarray(dims, np.uint64)
    h = C.c_void_p()
    _check(lib().altob_create_device(int(nmodes), dims.ctypes.data_as(_u64p), int(nnz), _dev_ptr(d_cidx),
                                     _dev_ptr(d_vals), vdt, int(nprtn), int(lit_bits), _stream_ptr(stream),
                                     C.byref(h)))
    return AltoTensor(h)


def destroy_alto(at: AltoTensor):
    at.destroy()


# --------------------------------------------------------------------------
# MTTKRP

def _ftype_of(arrs):
    a = arrs[0]
    dt = str(a.dtype)
    if "float64" in dt:
        return F64
    if "float32" in dt:
        return F32
    raise TypeError(f"factor dtype must be float32 or float64, got {dt}")


def mttkrp_alto_par(target_mode: int, factors: Sequence, rank: int, at: AltoTensor, algo="auto",
                    accumulate=True, stream=None):
    """mttkrp_alto_par (include/alto.hpp:617-623): factors[target_mode] +=
    MTTKRP.  `factors` are numpy arrays (host; copied in and the target
    copied back) or CUDA tensors (device; updated in place on `stream`)."""
    ft = _ftype_of(factors)
    a = ALGOS[algo] if isinstance(algo, str) else int(algo)
    if isinstance(factors[0], np.ndarray):
        if not accumulate:
            factors[target_mode][...] = 0
        ptrs = [f.ctypes.data for f in factors]
        for f in factors:
            assert f.flags.c_contiguous
        _check(lib().altob_mttkrp_host(at.handle, int(target_mode), ft, _ptr_array(ptrs), int(rank), a,
                                       _stream_ptr(stream)))
    else:
        ptrs = [_dev_ptr(f) for f in factors]
        _check(lib().altob_mttkrp(at.handle, int(target_mode), ft, _ptr_array(ptrs), int(rank),
                                  int(bool(accumulate)), a, _stream_ptr(stream)))


def mttkrp_sweep_host(at: AltoTensor, factors: Sequence[np.ndarray], rank: int, iters=1, algo="auto",
                      stream=None):
    """`iters` sweeps of mttkrp_alto_par over every mode on host factors
    (the reference's -p benchmark loop, src/main.cpp:476-495)."""
    ft = _ftype_of(factors)
    a = ALGOS[algo] if isinstance(algo, str) else int(algo)
    ptrs = [f.ctypes.data for f in factors]
    _check(lib().altob_mttkrp_sweep_host(at.handle, ft, _ptr_array(ptrs), int(rank), int(iters), a,
                                         _stream_ptr(stream)))


def calculate_phi(at: AltoTensor, mode: int, factors: Sequence, rank: int, phi, eps_div_zero=1e-10,
                  stream=None):
    """CalculatePhi_alto_par (include/apr.hpp:297-303) on device arrays."""
    ft = _ftype_of(factors)
    ptrs = [_dev_ptr(f) for f in factors]
    _check(lib().altob_phi(at.handle, int(mode), ft, _ptr_array(ptrs), int(rank), float(eps_div_zero),
                           _dev_ptr(phi), _stream_ptr(stream)))


# --------------------------------------------------------------------------
# Kruskal models (include/kruskal_model.hpp:8-15)

@dataclass
class KruskalModel:
    dims: List[int]
    rank: int
    U: List[np.ndarray] = field(default_factory=list)
    lam: Optional[np.ndarray] = None

    @property
    def mode(self):
        return len(self.dims)


def CreateKruskalModel(mode, dims, rank, dtype=np.float64):
    """CreateKruskalModel (src/kruskal_model.cpp:80-106)."""
    dims = [int(d) for d in dims[:mode]]
    return KruskalModel(dims, int(rank), [np.zeros((d, rank), dtype) for d in dims], np.zeros(rank, dtype))


def KruskalModelRandomInit(M: KruskalModel, seed: int):
    """KruskalModelRandomInit (src/kruskal_model.cpp:109-125): lambda = 1,
    U = (FType)rand()/RAND_MAX from glibc srand(seed), mode by mode."""
    ft = _ftype_of(M.U)
    dims = np.array(M.dims, np.uint64)
    ptrs = [u.ctypes.data for u in M.U]
    _check(lib().altob_kruskal_random_init(M.mode, dims.ctypes.data_as(_u64p), M.rank, int(seed) & 0xFFFFFFFF, ft,
                                           _ptr_array(ptrs), M.lam.ctypes.data))


def poisson_tensor(dims, num_edges, rank, nthreads=1, stream=None):
    """PoissonGeneratorRun (src/poisson_generator.cpp:337-375) as cpd64 -d
    runs it (MakeSparseTensor, src/main.cpp:652-675), with the random streams
    of `nthreads` OpenMP threads: (SparseTensor of counts, true model)."""
    dims = np.ascontiguousarray(dims, np.uint64)
    nm = dims.shape[0]
    U = [np.zeros((int(d), int(rank))) for d in dims]
    lam = np.zeros(int(rank))
    p = C.POINTER(_Coo)()
    _check(lib().altob_poisson_tensor(nm, dims.ctypes.data_as(_u64p), int(num_edges), int(rank), int(nthreads),
                                      _ptr_array([u.ctypes.data for u in U]), lam.ctypes.data_as(_dp), C.byref(p),
                                      _stream_ptr(stream)))
    return _coo_to_tensor(p), KruskalModel([int(d) for d in dims], int(rank), U, lam)


def random_init_factors(dims, rank, seed, dtype=np.float64):
    M = CreateKruskalModel(len(dims), dims, rank, dtype)
    KruskalModelRandomInit(M, seed)
    return M


def _is_host(arrs):
    return isinstance(arrs[0], np.ndarray)


def cpd_alto(at: AltoTensor, M: KruskalModel, max_iters: int, epsilon: float, stream=None):
    """cpd_alto (include/cpd.hpp:43-186).  Updates M in place and returns
    the per-iteration fits (cpd_fit_alto, cpd.hpp:189-271).  M holds numpy
    arrays (host model) or CUDA tensors (device model)."""
    ft = _ftype_of(M.U)
    fits = np.zeros(max_iters)
    it = C.c_int(0)
    if _is_host(M.U):
        ptrs = [u.ctypes.data for u in M.U]
        _check(lib().altob_cpd_als_host(at.handle, ft, _ptr_array(ptrs), M.lam.ctypes.data, M.rank, int(max_iters),
                                        float(epsilon), fits.ctypes.data_as(_dp), C.byref(it), _stream_ptr(stream)))
    else:
        ptrs = [_dev_ptr(u) for u in M.U]
        _check(lib().altob_cpd_als(at.handle, ft, _ptr_array(ptrs), _dev_ptr(M.lam), M.rank, int(max_iters),
                                   float(epsilon), fits.ctypes.data_as(_dp), C.byref(it), _stream_ptr(stream)))
    return fits[:it.value]


def pseudo_inverse(grams, mode, U, stream=None):
    """pseudo_inverse (include/cpd.hpp:546-646) on the device: U <- U V^-1
    (Cholesky) or U V^+ with V the Hadamard product of the Grams of every
    mode but `mode`.  grams: CUDA FP64 tensor (nmode, R, R); U: CUDA tensor
    (rows, R), updated in place.  Returns True when the pseudo-inverse was
    used."""
    used = C.c_int(0)
    _check(lib().altob_pseudo_inverse(_dev_ptr(grams), int(grams.shape[0]), int(mode), int(U.shape[1]),
                                      _dev_ptr(U), int(U.shape[0]), _ftype_of([U]), C.byref(used),
                                      _stream_ptr(stream)))
    return bool(used.value)


def cp_apr_alto(at: AltoTensor, M: KruskalModel, max_iters: int, max_inner_iters: int, epsilon=1e-5,
                eps_div_zero=1e-10, kappa_tol=1e-10, kappa=1e-2, dobench=False, stream=None):
    """cp_apr_alto (include/apr.hpp:984-1376).  Updates M in place; returns
    {loglik, fit, kkt, outer, inner} as the reference prints them."""
    ft = _ftype_of(M.U)
    out = np.zeros(5)
    args = (M.rank, int(max_iters), int(max_inner_iters), float(epsilon), float(eps_div_zero), float(kappa_tol),
            float(kappa), int(bool(dobench)), out.ctypes.data_as(_dp), _stream_ptr(stream))
    if _is_host(M.U):
        ptrs = [u.ctypes.data for u in M.U]
        _check(lib().altob_cp_apr_host(at.handle, ft, _ptr_array(ptrs), M.lam.ctypes.data, *args))
    else:
        ptrs = [_dev_ptr(u) for u in M.U]
        _check(lib().altob_cp_apr(at.handle, ft, _ptr_array(ptrs), _dev_ptr(M.lam), *args))
    return dict(loglik=out[0], fit=out[1], kkt=out[2], outer=int(out[3]), inner=int(out[4]))


def tt_logLikelihood(at: AltoTensor, M: KruskalModel, eps_div_zero=1e-10, stream=None):
    """tt_logLikelihood (include/apr.hpp:851-982) on a device model; like the
    reference it moves lambda into mode 0 and renormalises that mode."""
    ft = _ftype_of(M.U)
    ptrs = [_dev_ptr(u) for u in M.U]
    ll = C.c_double(0.0)
    _check(lib().altob_loglik(at.handle, ft, _ptr_array(ptrs), _dev_ptr(M.lam), M.rank, float(eps_div_zero),
                              C.byref(ll), _stream_ptr(stream)))
    return ll.value


class BatchCPD:
    """Many independent CP-ALS solves in batched launches (no counterpart in
    the reference; each tensor follows cpd_alto, include/cpd.hpp:43-186).

    tensors: AltoTensor handles; models: KruskalModel with CUDA tensors (all
    FP32 or all FP64).  The models are updated in place by every solve().
    The handle keeps references to both so their memory outlives it."""

    def __init__(self, tensors, models, fit_capacity=64, stream=None):
        if len(tensors) != len(models) or not tensors:
            raise ValueError("need one model per tensor")
        ft = _ftype_of(models[0].U)
        self._tensors, self._models = list(tensors), list(models)
        self.count = len(tensors)
        self.fit_capacity = int(fit_capacity)
        n = self.count
        th = (C.c_void_p * n)(*[t.handle for t in tensors])
        ranks = (C.c_uint64 * n)(*[m.rank for m in models])
        self._rows = []
        for m in models:
            if _ftype_of(m.U) != ft:
                raise ValueError("all models need one dtype")
            self._rows.append(_ptr_array([_dev_ptr(u) for u in m.U]))
        fac = (C.c_void_p * n)(*[C.cast(r, C.c_void_p).value for r in self._rows])
        lam = (C.c_void_p * n)(*[_dev_ptr(m.lam) for m in models])
        h = C.c_void_p()
        _check(lib().altob_batch_create(th, n, ranks, ft, fac, lam, self.fit_capacity, _stream_ptr(stream),
                                        C.byref(h)))
        self.handle = h.value

    def autotune(self, force=True, stream=None):
        _check(lib().altob_batch_autotune(self.handle, int(bool(force)), _stream_ptr(stream)))

    def solve(self, max_iters, epsilon, use_graph=True, stream=None):
        """Returns (fits[count, max_iters], iters[count])."""
        fits = np.zeros((self.count, max_iters))
        iters = np.zeros(self.count, dtype=np.int32)
        _check(lib().altob_batch_cpd_als(self.handle, int(max_iters), float(epsilon), fits.ctypes.data_as(_dp),
                                         iters.ctypes.data_as(C.POINTER(_i)), int(bool(use_graph)),
                                         _stream_ptr(stream)))
        return fits, iters

    def describe(self):
        buf = C.create_string_buffer(1 << 16)
        _check(lib().altob_batch_describe(self.handle, buf, len(buf)))
        return buf.value.decode()

    def close(self):
        if getattr(self, "handle", None):
            lib().altob_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def status_of(fn, *args):
    try:
        fn(*args)
        return 0
    except AltobError as e:
        return e.status


def version():
    return lib().altob_version().decode()
