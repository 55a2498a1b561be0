"""Pins the oracle (oracle/alto_oracle.c) to fixtures written by the
reference itself (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from alto_b200 import synth
from conftest import golden_cases, load_golden, rel_fro, same_oidx
from helpers import mttkrp_from_golden, pext_rows

ENC = golden_cases("enc_")


@pytest.mark.parametrize("name", ENC)
def test_oracle_encoding_matches_reference(oracle, name):
    g = load_golden(name)
    t = oracle.create(g["dims"], g["cidx"], g["vals"], int(g["nprtn"]), int(g["lit_bits"]))
    d = t.dump()
    assert d["alto_bits"] == int(g["enc_alto_bits"])
    assert d["is_oidx"] == int(g["enc_is_oidx"])
    np.testing.assert_array_equal(d["masks"], g["enc_masks"])
    np.testing.assert_array_equal(d["cr_masks"], g["enc_cr_masks"])
    np.testing.assert_array_equal(d["idx"], g["enc_idx"])  # bit-exact, CR bits included
    np.testing.assert_array_equal(d["vals"], g["enc_vals"])
    np.testing.assert_array_equal(d["prtn_ptr"], g["enc_prtn_ptr"])
    np.testing.assert_array_equal(d["intervals"], g["enc_intervals"])
    if d["is_oidx"]:
        nnz = g["vals"].shape[0]
        for n in range(len(g["dims"])):
            if nnz // int(g["dims"][n]) > 4:
                continue
            keys = pext_rows(d["idx"], d["masks"][n])
            assert same_oidx(lambda o: keys[o.astype(np.int64)], d["oidx"][n], g["enc_oidx"][n])


@pytest.mark.parametrize("name", [n for n in ENC if "mttkrp0_rows" in load_golden(n)])
def test_oracle_mttkrp_matches_reference(oracle, name):
    g = load_golden(name)
    rank = int(g["rank"])
    t = oracle.create(g["dims"], g["cidx"], g["vals"], int(g["nprtn"]), int(g["lit_bits"]))
    for mode in range(len(g["dims"])):
        U, want = mttkrp_from_golden(g, mode, synth)
        t.mttkrp(mode, U, rank)
        assert rel_fro(U[mode], want) < 1e-12


def test_oracle_cpd_matches_reference(oracle):
    g = load_golden("cpd_u3")
    rank = int(g["rank"])
    U, lam = oracle.random_init(g["dims"], rank, int(g["seed"]))
    t = oracle.create(g["dims"], g["cidx"], g["vals"], int(g["nprtn"]), 64)
    fits = t.cpd_als(U, lam, rank, int(g["max_iters"]), 1e-30)
    assert len(fits) == len(g["fits"])
    # the reference prints fits with %g (6 significant digits)
    np.testing.assert_allclose(fits, g["fits"], rtol=2e-6, atol=0)
    for n in range(len(U)):
        assert rel_fro(U[n], g[f"U{n}"]) < 1e-9
    np.testing.assert_allclose(lam, g["lam"], rtol=1e-9)


def test_oracle_cpd_convergence_matches_reference(oracle):
    g = load_golden("cpd_conv4")
    rank = int(g["rank"])
    U, lam = oracle.random_init(g["dims"], rank, int(g["seed"]))
    t = oracle.create(g["dims"], g["cidx"], g["vals"], int(g["nprtn"]), 64)
    fits = t.cpd_als(U, lam, rank, int(g["max_iters"]), float(g["eps"]))
    assert len(fits) == len(g["fits"])  # same stopping iteration
    np.testing.assert_allclose(fits, g["fits"], rtol=2e-6)
    for n in range(len(U)):
        assert rel_fro(U[n], g[f"U{n}"]) < 1e-9


@pytest.mark.parametrize("name", ["apr_bench", "apr_eps"])
def test_oracle_cp_apr_matches_reference(oracle, name):
    g = load_golden(name)
    rank = int(g["rank"])
    U, lam = oracle.random_init(g["dims"], rank, int(g["seed"]))
    t = oracle.create(g["dims"], g["cidx"], g["vals"], int(g["nprtn"]), 64)
    r = t.cp_apr(U, lam, rank, int(g["max_iters"]), int(g["max_inner"]), float(g["eps"]), 1e-10, 1e-10, 1e-2,
                 bool(g["dobench"]))
    assert r["outer"] == int(g["outer"]) and r["inner"] == int(g["inner"])
    np.testing.assert_allclose(r["loglik"], g["loglik"], rtol=1e-6)  # printed with %e
    np.testing.assert_allclose(r["fit"], g["fit"], rtol=1e-6)
    np.testing.assert_allclose(r["kkt"], g["kkt"], rtol=1e-6)
    for n in range(len(U)):
        assert rel_fro(U[n], g[f"U{n}"]) < 1e-9
    np.testing.assert_allclose(lam, g["lam"], rtol=1e-9)


def test_oracle_coo_mttkrp_agrees_with_alto_order(oracle):
    dims, cidx, vals = synth.uniform_distinct((40, 30, 20), 3000, seed=3)
    t = oracle.create(dims, cidx, vals, 5, 64)
    for mode in range(3):
        A = synth.random_factors(dims, 6, seed=mode)
        B = [a.copy() for a in A]
        t.mttkrp(mode, A, 6)
        oracle.mttkrp_coo(dims, cidx, vals, mode, B, 6)
        assert rel_fro(A[mode], B[mode]) < 1e-13


def test_oracle_rejects_too_many_bits(oracle):
    dims = np.array([1 << 40, 1 << 30], np.uint64)
    with pytest.raises(ValueError):
        oracle.create(dims, np.zeros((2, 1), np.uint64), np.ones(1), 1, 64)
