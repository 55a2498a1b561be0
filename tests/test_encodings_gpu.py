"""The reference's alternative encodings, from a tensor handle, against the
reference's own -DALT_PEXT and -DOPT_ALTO builds (oracle/_ref): ALT_PEXT
keys (alto.hpp:212-244, CR bits included) and mode masks, bit for bit; the
ALT_PEXT build's MTTKRP (1e-12); the OPT_ALTO partition subspace ids
(alto.hpp:838-868), bit for bit."""
import os

import numpy as np
import pytest

import alto_b200 as ab
from alto_b200 import synth
from conftest import rel_fro

pytestmark = pytest.mark.gpu
orc = pytest.importorskip("oracle.orc")

CASES = [
    # dims, nnz, nprtn: modes in and out of shortest-first order, low fiber
    # reuse (CR bits), 4 and 5 modes
    ((300, 1000, 5000), 50_000, 8),
    ((5000, 1000, 300), 50_000, 8),
    ((40_000, 30_000, 20_000), 30_000, 16),
    ((64, 128, 256, 512), 80_000, 12),
    ((20, 30, 40, 50, 60), 40_000, 5),
]


def _lib(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.basename(path)} not built")
    return orc.RefLib(path)


@pytest.mark.parametrize("case", CASES)
def test_alt_pext_keys_and_masks(case):
    ref = _lib(orc.REF_SO_PEXT)
    dims, nnz, nprtn = case
    d, cidx, vals = synth.uniform_distinct(dims, nnz, seed=nnz % 71)
    want = ref.create_dump(d, cidx, vals, nprtn, 64)
    at = ab.create_alto(ab.SparseTensor.from_arrays(d, cidx, vals), nprtn, 64)
    got = at.dump_alt_pext()
    assert np.array_equal(got["idx"], want["idx"])
    assert np.array_equal(got["masks"], want["masks"])


@pytest.mark.parametrize("case", [CASES[0], CASES[1], CASES[3]])
def test_alt_pext_build_mttkrp_matches(case):
    """The ALT_PEXT build's MTTKRP (pext with field positions) against the
    device kernel."""
    torch = pytest.importorskip("torch")
    ref = _lib(orc.REF_SO_PEXT)
    dims, nnz, nprtn = case
    d, cidx, vals = synth.uniform_distinct(dims, nnz, seed=3)
    at = ab.create_alto(ab.SparseTensor.from_arrays(d, cidx, vals), nprtn, 64)
    rank = 16
    for mode in range(len(dims)):
        U = synth.random_factors(d, rank, seed=mode)
        want = [u if m != mode else np.zeros_like(u) for m, u in enumerate(U)]
        ref.mttkrp(d, cidx, vals, nprtn, 64, mode, want, rank)
        dU = [torch.from_numpy(u).cuda() for u in U]
        ab.mttkrp_alto_par(mode, dU, rank, at, accumulate=False)
        assert rel_fro(dU[mode].cpu().numpy(), want[mode]) < 1e-12, mode


@pytest.mark.parametrize("case", CASES + [((4_800_000, 1_800_000, 1_800_000), 200_000, 32)])
def test_opt_alto_partition_ids(case):
    ref = _lib(orc.REF_SO_OPT)
    dims, nnz, nprtn = case
    d, cidx, vals = synth.uniform_distinct(dims, nnz, seed=11)
    at = ab.create_alto(ab.SparseTensor.from_arrays(d, cidx, vals), nprtn, 0)
    lit = at.info()["lit_bits"]
    want = ref.prtn_ids(d, cidx, vals, nprtn, lit)
    got = at.partition_ids()
    for k in ("prtn_id", "prtn_mask", "prtn_mode_masks"):
        assert np.array_equal(got[k], want[k]), k


def test_alt_pext_refuses_31_bit_modes():
    d, cidx, vals = synth.uniform_distinct((1 << 31, 100, 100), 1000, seed=1)
    at = ab.create_alto(ab.SparseTensor.from_arrays(d, cidx, vals), 4, 0)
    with pytest.raises(ab.AltobError):
        at.dump_alt_pext()
