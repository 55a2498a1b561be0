"""Sharded MTTKRP and CP-ALS: one tensor split across GPUs.

The reference (IntelLabs/ALTO) runs on one node.  Its own parallel split is
the equal-nnz contiguous partition of the ALTO stream (prtn_alto,
include/alto.hpp:822-836) with each partition's output rows bounded by its
mode intervals (alto.hpp:874-899); here each GPU takes one such partition:

* every GPU builds the tensor's ALTO stream (or receives it) and keeps the
  slice [begin, end) of `shard_bounds` for its rank (`AltoTensor.slice`);
* MTTKRP: each GPU computes the partial rows of its slice into a full
  I_n x R buffer, and one all-reduce (sum) over the GPUs completes it;
* CP-ALS (`altob_cpd_als_sharded`): the same partial MTTKRP per mode plus
  an all-reduce, after which every GPU runs the dense update (R x R Grams,
  solve, normalisation, fit) on identical data; the fit is all-reduced with
  max so the stopping rule agrees everywhere, and the tensor norm once.

The exchanges go through an all-reduce callback.  `nccl_allreduce` makes one
from a torch.distributed process group (one process per GPU, NCCL over
NVLink); `host_allreduce` does the same for host buffers over a CPU (gloo)
group.  Factors are replicated, so the data path has exactly one collective
per mode.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import (AltoTensor, KruskalModel, _check, _dev_ptr, _dp, _ftype_of, _ptr_array, _stream_ptr, F32, F64,
               lib)

REDUCE_SUM, REDUCE_MAX = 0, 1
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_void_p, C.c_void_p)
_ERR_CUDA = 3  # ALTOB_ERR_CUDA


def shard_bounds(nnz, world):
    """[begin, end) of every rank: contiguous ranges of ceil(nnz / world)
    nonzeros of the ALTO stream (the last ones may be short or empty), the
    rule of prtn_alto (alto.hpp:822-836)."""
    per = -(-int(nnz) // int(world)) if world > 0 else 0
    return [(min(r * per, nnz), min((r + 1) * per, nnz)) for r in range(world)]


class _DeviceView:
    """A raw device buffer as an array torch can wrap without copying."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


_TYPESTR = {F64: "<f8", F32: "<f4"}


def _torch_op(dist, op):
    return dist.ReduceOp.MAX if op == REDUCE_MAX else dist.ReduceOp.SUM


def nccl_allreduce(group=None):
    """An all-reduce callback for altob_cpd_als_sharded over a
    torch.distributed (NCCL) process group: the buffer is wrapped in place and
    reduced on the solver's stream.  Keep the returned object alive while the
    solve runs."""
    import torch
    import torch.distributed as dist

    def fn(buf, count, dtype, op, stream, user):
        try:
            t = torch.as_tensor(_DeviceView(buf, count, _TYPESTR[dtype]), device="cuda")
            s = torch.cuda.ExternalStream(int(stream)) if stream else torch.cuda.default_stream()
            with torch.cuda.stream(s):
                dist.all_reduce(t, op=_torch_op(dist, op), group=group)
            return 0
        except Exception:  # noqa: BLE001 - reported to the library as a status
            return _ERR_CUDA

    return ALLREDUCE_FN(fn)


def host_allreduce(group=None):
    """The same callback for host buffers over a CPU (gloo) group."""
    import torch
    import torch.distributed as dist

    def fn(buf, count, dtype, op, stream, user):
        try:
            ctype = C.c_double if dtype == F64 else C.c_float
            arr = np.ctypeslib.as_array((ctype * int(count)).from_address(int(buf)))
            t = torch.from_numpy(arr)
            dist.all_reduce(t, op=_torch_op(dist, op), group=group)
            return 0
        except Exception:  # noqa: BLE001
            return _ERR_CUDA

    return ALLREDUCE_FN(fn)


class ShardedTensor:
    """One rank's slice of a tensor sharded over `world` GPUs."""

    def __init__(self, full: AltoTensor, rank: int, world: int, nprtn: int = 256, stream=None):
        nnz = full.info()["nnz"]
        self.rank, self.world = int(rank), int(world)
        self.bounds = shard_bounds(nnz, world)[rank]
        self.local = full.slice(self.bounds[0], self.bounds[1], nprtn, stream)
        self.dims = full.info()["dims"]

    def mttkrp(self, mode, factors, rank, allreduce, stream=None):
        """factors[mode] = the full MTTKRP (overwritten): this slice's
        partial rows, then the all-reduce (sum) over the GPUs."""
        from . import mttkrp_alto_par
        mttkrp_alto_par(mode, factors, rank, self.local, accumulate=False, stream=stream)
        out = factors[mode]
        st = _stream_ptr(stream)
        rc = allreduce(_dev_ptr(out), int(out.numel()), _ftype_of([out]), REDUCE_SUM, st, None)
        if rc != 0:
            _check(rc)

    def cpd_als(self, M: KruskalModel, max_iters, epsilon, allreduce, stream=None):
        """cpd_alto (cpd.hpp:43-186) on the sharded tensor; every rank calls it
        with the same initial model and gets the same result."""
        ft = _ftype_of(M.U)
        fits = np.zeros(max_iters)
        it = C.c_int(0)
        ptrs = [_dev_ptr(u) for u in M.U]
        _check(lib().altob_cpd_als_sharded(self.local.handle, ft, _ptr_array(ptrs), _dev_ptr(M.lam), M.rank,
                                           int(max_iters), float(epsilon), fits.ctypes.data_as(_dp), C.byref(it),
                                           C.cast(allreduce, C.c_void_p), None, _stream_ptr(stream)))
        return fits[:it.value]
