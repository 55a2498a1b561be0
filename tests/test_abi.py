"""The C ABI library loads and exports every symbol include/altob.h
declares; host-only entry points work without a GPU.  CPU only."""
import os
import re

import numpy as np
import pytest

import alto_b200 as ab
from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "altob.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"ALTOB_API[^;(]*?\b(altob_\w+)\s*\(", text, flags=re.S)))


def test_library_exports_every_declared_symbol():
    L = ab.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(ab.SIGNATURES), "Python bindings and header disagree"


def test_status_strings_and_version():
    L = ab.lib()
    assert L.altob_status_string(0) == b"ok"
    assert b"argument" in L.altob_status_string(1)
    assert b"sm_100a" in L.altob_version()


def test_null_arguments_are_errors_not_crashes():
    L = ab.lib()
    assert L.altob_destroy(None) == 0
    assert L.altob_get_info(None, None) == 1
    assert L.altob_mttkrp(None, 0, 0, None, 8, 1, 0, None) == 1


def test_tns_round_trip(tmp_path):
    dims = np.array([4, 5, 6], np.uint64)
    cidx = np.array([[0, 3, 1, 2], [4, 0, 2, 2], [5, 1, 0, 3]], np.uint64)
    vals = np.array([1.5, -2.0, 3.25, 1e-3])
    X = ab.SparseTensor.from_arrays(dims, cidx, vals)
    p = str(tmp_path / "t.tns")
    ab.ExportSparseTensor(p, ab.TEXT_FORMAT, X)
    Y = ab.ImportSparseTensor(p, ab.TEXT_FORMAT)
    np.testing.assert_array_equal(Y.cidx, cidx)
    np.testing.assert_allclose(Y.vals, vals)
    np.testing.assert_array_equal(Y.dims, dims)  # dims = largest index seen


def test_tns_reader_reference_rules(tmp_path):
    # comments and empty lines skipped; dims from the largest index; tabs;
    # 0-based reading with the reference's dims = max index + zero_based
    p = str(tmp_path / "r.tns")
    with open(p, "w") as f:
        f.write("# a comment\n\n1 2 3 1.0\n4\t1 1 2.5\n\n2 2 7 -1e2\n")
    Y = ab.ImportSparseTensor(p, ab.TEXT_FORMAT)
    np.testing.assert_array_equal(Y.dims, [4, 2, 7])
    np.testing.assert_array_equal(Y.cidx, [[0, 3, 1], [1, 0, 1], [2, 0, 6]])
    np.testing.assert_allclose(Y.vals, [1.0, 2.5, -100.0])
    Z = ab.ImportSparseTensor(p, ab.TEXT_FORMAT, zero_based=1)
    np.testing.assert_array_equal(Z.dims, [5, 3, 8])
    np.testing.assert_array_equal(Z.cidx, [[1, 4, 2], [2, 1, 2], [3, 1, 7]])


def test_tns_reader_large_parallel(tmp_path):
    from alto_b200 import synth
    dims, cidx, vals = synth.uniform_distinct((300, 200, 100), 200_000, seed=2)
    X = ab.SparseTensor.from_arrays(dims, cidx, vals)
    p = str(tmp_path / "big.tns")
    ab.ExportSparseTensor(p, ab.TEXT_FORMAT, X)
    Y = ab.ImportSparseTensor(p, ab.TEXT_FORMAT)
    np.testing.assert_array_equal(Y.cidx, cidx)
    np.testing.assert_allclose(Y.vals, vals, rtol=1e-5)  # %g keeps 6 digits


def test_readers_match_the_reference_reader(tmp_path):
    """altob_read_tns / altob_read_bin against the reference's own
    ImportSparseTensor (src/sptensor.cpp:75-258, compiled under oracle/_ref):
    the same dims, coordinates and values, bit for bit, for the rule cases
    (comments, empty lines, tabs, 1- and 0-based) and generated files."""
    from alto_b200 import synth
    from oracle.orc import RefLib, ref_available
    if not ref_available():
        pytest.skip("reference library not built")
    ref = RefLib()
    rules = str(tmp_path / "r.tns")
    with open(rules, "w") as f:
        f.write("# a comment\n\n1 2 3 1.0\n4\t1 1 2.5\n\n2 2 7 -1e2\n")
    files = [(rules, False, 0), (rules, False, 1)]
    for k, (shape, nnz) in enumerate([((300, 200, 100), 200_000), ((50, 40, 30, 20, 7), 30_000)]):
        dims, cidx, vals = synth.uniform_distinct(shape, nnz, seed=11 + k)
        X = ab.SparseTensor.from_arrays(dims, cidx, vals)
        for binary in (False, True):
            p = str(tmp_path / (f"g{k}." + ("bin" if binary else "tns")))
            ab.ExportSparseTensor(p, ab.BINARY_FORMAT if binary else ab.TEXT_FORMAT, X)
            files.append((p, binary, 0))
    for p, binary, zb in files:
        rd, rc, rv = ref.read(p, binary=binary, zero_based=zb)
        if binary:
            Y = ab.ImportSparseTensor(p, ab.BINARY_FORMAT)
        else:
            Y = ab.ImportSparseTensor(p, ab.TEXT_FORMAT, zero_based=zb)
        np.testing.assert_array_equal(Y.dims, rd, err_msg=p)
        np.testing.assert_array_equal(Y.cidx, rc, err_msg=p)
        np.testing.assert_array_equal(Y.vals, rv, err_msg=p)
    # files written by the reference's ExportSparseTensor (src/sptensor.cpp:23-70)
    dims, cidx, vals = synth.uniform_distinct((300, 200, 100), 50_000, seed=7)
    p = str(tmp_path / "ref.tns")
    ref.write(p, dims, cidx, vals)
    rd, rc, rv = ref.read(p)
    Y = ab.ImportSparseTensor(p, ab.TEXT_FORMAT)
    np.testing.assert_array_equal(Y.dims, rd)
    np.testing.assert_array_equal(Y.cidx, rc)
    np.testing.assert_array_equal(Y.vals, rv)
    # its binary writer stores the 4-byte mode count as 8 bytes, the upper 4
    # being struct padding (src/sptensor.cpp:59): the reference's own reader
    # can then abort on its mode-count assert, so only this reader reads it
    p = str(tmp_path / "ref.bin")
    ref.write(p, dims, cidx, vals, binary=True)
    Y = ab.ImportSparseTensor(p, ab.BINARY_FORMAT)
    np.testing.assert_array_equal(Y.dims, dims)
    np.testing.assert_array_equal(Y.cidx, cidx)
    np.testing.assert_array_equal(Y.vals, vals)


ODD_TNS = {
    "crlf": "1 2 3 1.0\r\n2 1 1 2.0\r\n",
    "multi_space": "1  2   3 1.0\n2 1 1   2.0\n",
    "leading_space": " 1 2 3 1.0\n 2 1 1 2.0\n",
    "tabs": "1\t2\t3\t1.0\n2\t1\t1\t2.0\n",
    "no_final_newline": "1 2 3 1.0\n2 1 1 2.0",
    "exponents": "1 2 3 1e-300\n2 1 1 -2.5E+10\n",
    "comment_between": "1 2 3 1.0\n# c\n2 1 1 2.0\n",
}


@pytest.mark.parametrize("name", sorted(ODD_TNS))
def test_tns_odd_formatting_matches_the_reference_reader(tmp_path, name):
    """Line endings, repeated and leading separators, a missing final newline,
    exponents and comments between data lines read as the reference reads
    them (src/sptensor.cpp:75-161)."""
    from oracle.orc import RefLib, ref_available
    if not ref_available():
        pytest.skip("reference library not built")
    p = str(tmp_path / "odd.tns")
    with open(p, "w", newline="") as f:
        f.write(ODD_TNS[name])
    rd, rc, rv = RefLib().read(p)
    Y = ab.ImportSparseTensor(p, ab.TEXT_FORMAT)
    np.testing.assert_array_equal(Y.dims, rd)
    np.testing.assert_array_equal(Y.cidx, rc)
    np.testing.assert_array_equal(Y.vals, rv)


def test_tns_trailing_whitespace(tmp_path):
    """A separator before the newline: the reference counts the newline as
    one more token (one mode too many, every value read as 0); this reader
    ignores trailing whitespace."""
    p = str(tmp_path / "trail.tns")
    with open(p, "w") as f:
        f.write("1 2 3 1.0 \n2 1 1 2.0\t\n")
    Y = ab.ImportSparseTensor(p, ab.TEXT_FORMAT)
    np.testing.assert_array_equal(Y.dims, [2, 2, 3])
    np.testing.assert_array_equal(Y.cidx, [[0, 1], [1, 0], [2, 0]])
    np.testing.assert_array_equal(Y.vals, [1.0, 2.0])


def test_binary_round_trip_and_errors(tmp_path):
    dims = np.array([7, 8], np.uint64)
    cidx = np.array([[1, 6], [7, 0]], np.uint64)
    vals = np.array([0.5, 0.25])
    X = ab.SparseTensor.from_arrays(dims, cidx, vals)
    p = str(tmp_path / "t.bin")
    ab.ExportSparseTensor(p, ab.BINARY_FORMAT, X)
    Y = ab.ImportSparseTensor(p, ab.BINARY_FORMAT)
    np.testing.assert_array_equal(Y.cidx, cidx)
    np.testing.assert_array_equal(Y.vals, vals)
    with open(p, "r+b") as f:
        f.truncate(40)
    with pytest.raises(ab.AltobError) as e:
        ab.ImportSparseTensor(p, ab.BINARY_FORMAT)
    assert e.value.status == 5
    with pytest.raises(ab.AltobError):
        ab.ImportSparseTensor(str(tmp_path / "missing.tns"))


def test_random_init_matches_glibc_reference_stream(oracle):
    M = ab.random_init_factors([30, 20, 10], 7, 1234)
    U, lam = oracle.random_init([30, 20, 10], 7, 1234)
    for a, b in zip(M.U, U):
        np.testing.assert_array_equal(a, b)
    M32 = ab.random_init_factors([30, 20, 10], 7, 1234, dtype=np.float32)
    np.testing.assert_allclose(M32.U[2], U[2].astype(np.float32), rtol=1e-7)
