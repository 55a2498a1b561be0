"""Host-side pieces of the server and of the workload generators (no GPU):
the footprint estimate, and the seeded stream / tensor generators."""
import numpy as np
import pytest

import alto_b200 as ab
from alto_b200 import serve, synth


class _Fake:
    """Stands in for a device array in make_request (pointer + dtype + shape)."""

    def __init__(self, n, dtype):
        self.shape = (n,)
        self.dtype = dtype

    def data_ptr(self):
        return 0x1000

    is_cuda = True

    def is_contiguous(self):
        return True


def _req(kind, dims, nnz, rank, ftype=ab.F32):
    vals = _Fake(nnz, "torch.float32" if kind == serve.ALS else "torch.int32")
    return serve.Server.make_request(kind, dims, _Fake(nnz, "torch.int64"), vals, rank, 50, 1e-4, 1, ftype)


def test_footprint_grows_with_nnz_rank_and_dtype():
    base = serve.footprint(_req(serve.ALS, (1000, 800, 600), 1_000_000, 16))
    assert base >= 1_000_000 * 48  # the build's peak
    assert serve.footprint(_req(serve.ALS, (1000, 800, 600), 2_000_000, 16)) > base
    assert serve.footprint(_req(serve.ALS, (1000, 800, 600), 1_000_000, 64)) > base
    assert serve.footprint(_req(serve.ALS, (1000, 800, 600), 1_000_000, 16, ab.F64)) > base
    assert serve.footprint(_req(serve.APR, (1000, 800, 600), 1_000_000, 16)) > base


def test_footprint_rejects_bad_order():
    r = _req(serve.ALS, (10, 10, 10), 100, 4)
    r.nmode = 7
    with pytest.raises(ab.AltobError):
        serve.footprint(r)


def test_served_stream_shape():
    s = synth.served_stream(4000, 3)
    arr = np.array([x[0] for x in s])
    rate = len(s) / arr[-1]
    assert 185 < rate < 215  # Poisson arrivals at 200 / s
    frac = np.mean([x[1] == "als" for x in s])
    assert 0.67 < frac < 0.73
    nnz = np.array([x[3] for x in s])
    assert nnz.min() >= 50_000 and nnz.max() <= 20_000_000
    assert set(x[4] for x in s) == {16, 32, 64}
    assert all(x[2] == (20_000, 10_000, 5_000, 200) for x in s)
    assert synth.served_stream(10, 3) == s[:10]


def test_poisson_kruskal_counts_are_merged_and_seeded():
    torch = pytest.importorskip("torch")
    c1, v1 = synth.poisson_kruskal_torch((60, 50, 40, 10), 8, 50_000, 4, "cpu")
    c2, v2 = synth.poisson_kruskal_torch((60, 50, 40, 10), 8, 50_000, 4, "cpu")
    assert torch.equal(c1, c2) and torch.equal(v1, v2)
    assert int(v1.sum()) == 50_000 and v1.dtype == torch.int32
    keys = set(map(tuple, c1.t().tolist()))
    assert len(keys) == c1.shape[1]  # no repeated coordinate after merging
    for m, d in enumerate((60, 50, 40, 10)):
        assert 0 <= int(c1[m].min()) and int(c1[m].max()) < d
