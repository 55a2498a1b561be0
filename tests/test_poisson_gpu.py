"""The device Poisson generator (altob_poisson_tensor, cpd64 -d) against the
reference's own PoissonGeneratorRun (oracle/_ref, the reference compiled from
its sources) for the same OpenMP thread count: the tensor (coordinates,
counts) bit for bit; the model (factors and lambda) bit for bit on one
thread, and within 1e-13 (relative) on several, where the reference adds its
column sums in an OpenMP reduction whose order is not fixed."""
import numpy as np
import pytest

import alto_b200 as ab

pytestmark = pytest.mark.gpu
orc = pytest.importorskip("oracle.orc")

CASES = [
    # dims, num_edges, rank, threads
    ((30, 20, 10), 5_000, 3, 1),
    ((200, 150, 100, 20), 400_000, 8, 1),     # several 100,000-draw batches
    ((2000, 1000, 500), 250_000, 10, 4),      # four streams
    ((64, 64, 64, 64, 64), 120_000, 5, 3),    # order 5, uneven chunks
]


@pytest.fixture(scope="module")
def refp():
    import os
    if not os.path.exists(orc.REF_SO_POISSON):
        pytest.skip("reference generator library oracle/_ref/libaltoref_poisson.so not built")
    return orc.RefPoisson()


@pytest.mark.parametrize("case", CASES)
def test_poisson_generator_matches_reference(refp, case):
    dims, edges, rank, threads = case
    rc, rv, rU, rlam = refp.run(dims, edges, rank, threads)
    X, M = ab.poisson_tensor(dims, edges, rank, nthreads=threads)
    for n in range(len(dims)):
        if threads == 1:
            assert np.array_equal(M.U[n], rU[n]), n
        else:
            np.testing.assert_allclose(M.U[n], rU[n], rtol=1e-13, atol=0)
    if threads == 1:
        assert np.array_equal(M.lam, rlam)
    else:
        np.testing.assert_allclose(M.lam, rlam, rtol=1e-13)
    assert X.nnz == rv.shape[0]
    assert np.array_equal(X.cidx, rc)
    assert np.array_equal(X.vals, rv)
    assert X.vals.sum() == edges  # every draw became an edge


def test_poisson_generator_errors():
    with pytest.raises(ab.AltobError):
        ab.poisson_tensor((10, 2, 10), 100, 3)  # a dimension below the rank
    with pytest.raises(ab.AltobError):
        ab.poisson_tensor((10, 10), 0, 3)
