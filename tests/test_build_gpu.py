"""ALTO build on the GPU (linearize, radix sort, oidx, partitions,
intervals, CR bits) against the reference's encoding: bit-exact."""
import numpy as np
import pytest

import alto_b200 as ab
from alto_b200 import synth
from conftest import golden_cases, load_golden, same_oidx
from helpers import pext_rows

pytestmark = pytest.mark.gpu


def _coo(dims, cidx, vals):
    return ab.SparseTensor.from_arrays(dims, cidx, vals)


def _check_against(d, ref, dims, nnz):
    assert d["alto_bits"] == ref["alto_bits"]
    assert d["is_oidx"] == ref["is_oidx"]
    np.testing.assert_array_equal(d["masks"], ref["masks"])
    np.testing.assert_array_equal(d["cr_masks"], ref["cr_masks"])
    np.testing.assert_array_equal(d["idx"], ref["idx"])
    np.testing.assert_array_equal(d["vals"].astype(np.float64), ref["vals"])
    np.testing.assert_array_equal(d["prtn_ptr"], ref["prtn_ptr"])
    np.testing.assert_array_equal(d["intervals"], ref["intervals"])
    if d["is_oidx"] and nnz:
        for n in range(len(dims)):
            if nnz // int(dims[n]) > 4:
                continue
            keys = pext_rows(d["idx"], d["masks"][n])
            assert same_oidx(lambda o: keys[o.astype(np.int64)], d["oidx"][n], ref["oidx"][n])


@pytest.mark.parametrize("name", golden_cases("enc_"))
def test_gpu_encoding_matches_reference_fixture(name):
    g = load_golden(name)
    at = ab.create_alto(_coo(g["dims"], g["cidx"], g["vals"]), int(g["nprtn"]), int(g["lit_bits"]))
    ref = {k[4:]: g[k] for k in g if k.startswith("enc_")}
    ref["alto_bits"] = int(ref["alto_bits"])
    ref["is_oidx"] = int(ref["is_oidx"])
    _check_against(at.dump(), ref, g["dims"], g["vals"].shape[0])


CASES = [
    # dims, nnz, nprtn, lit_bits, seed
    ((1000, 800, 600), 200_000, 64, 64, 1),        # config-1 shape (reduced nnz)
    ((1000, 800, 600), 50_000, 3, 128, 2),
    ((7, 9, 11, 5, 3), 2_000, 13, 64, 3),           # 5 modes, tiny dims
    ((100_000, 70_000, 50_000), 30_000, 8, 64, 4),  # low reuse: oidx + CR bits
    ((3_000, 2, 40_000, 17), 40_000, 6, 128, 5),    # mixed reuse
    ((65_536, 65_536, 65_536, 65_536, 8), 20_000, 7, 128, 6),  # 67 bits
]


@pytest.mark.parametrize("case", CASES)
def test_gpu_encoding_matches_oracle(oracle, case):
    dims, nnz, nprtn, lit, seed = case
    dims_a, cidx, vals = synth.uniform_distinct(dims, nnz, seed)
    at = ab.create_alto(_coo(dims_a, cidx, vals), nprtn, lit)
    ref = oracle.create(dims_a, cidx, vals, nprtn, lit).dump()
    _check_against(at.dump(), ref, dims_a, nnz)


def test_gpu_encoding_zipf_65_bits(oracle):
    dims, cidx, vals = synth.zipf_tensor((4_800_000, 1_800_000, 1_800_000), 200_000, seed=7)
    at = ab.create_alto(_coo(dims, cidx, vals), 16, 0)
    assert at.info()["lit_bits"] == 128
    ref = oracle.create(dims, cidx, vals, 16, 128).dump()
    _check_against(at.dump(), ref, dims, vals.shape[0])


def test_gpu_encoding_edge_cases(oracle):
    # a mode of length 1 (0 ALTO bits), more partitions than nonzeros
    dims, cidx, vals = synth.uniform_distinct((1, 50, 40), 10, seed=8)
    at = ab.create_alto(_coo(dims, cidx, vals), 32, 64)
    ref = oracle.create(dims, cidx, vals, 32, 64).dump()
    _check_against(at.dump(), ref, dims, 10)
    # a single nonzero
    dims, cidx, vals = synth.uniform_distinct((5, 6, 7), 1, seed=9)
    at = ab.create_alto(_coo(dims, cidx, vals), 1, 64)
    ref = oracle.create(dims, cidx, vals, 1, 64).dump()
    _check_against(at.dump(), ref, dims, 1)


def test_gpu_empty_tensor():
    dims = np.array([10, 20, 30], np.uint64)
    at = ab.create_alto(_coo(dims, np.zeros((3, 0), np.uint64), np.zeros(0)), 4, 64)
    inf = at.info()
    assert inf["nnz"] == 0 and inf["alto_bits"] == 4 + 5 + 5
    d = at.dump()
    np.testing.assert_array_equal(d["prtn_ptr"], np.zeros(5, np.uint64))


def test_gpu_create_errors():
    dims = np.array([1 << 31, 1 << 31, 1 << 31], np.uint64)  # 93 ALTO bits
    X = _coo(dims, np.zeros((3, 1), np.uint64), np.ones(1))
    with pytest.raises(ab.AltobError) as e:
        ab.create_alto(X, 1, 64)
    assert e.value.status == 2  # ALTOB_ERR_BITS
    dims = np.array([1 << 40, 2], np.uint64)
    X = _coo(dims, np.zeros((2, 1), np.uint64), np.ones(1))
    with pytest.raises(ab.AltobError) as e:
        ab.create_alto(X, 1, 128)
    assert e.value.status == 6  # dimension beyond the 32-bit row index
    X = _coo(np.array([10, 10], np.uint64), np.array([[3], [10]], np.uint64), np.ones(1))
    with pytest.raises(ab.AltobError) as e:
        ab.create_alto(X, 1, 64)  # coordinate == dimension
    assert e.value.status == 1
