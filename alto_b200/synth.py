"""Seeded synthetic sparse tensors with the shapes and value distributions of
the benchmark configurations (the reference measures on FROSTT tensors that
are not available offline; these stand in for them).

All generators are deterministic for a given seed and independent of the
thread count.  They return (dims, cidx, vals) with cidx a (nmode, nnz)
uint64 array (0-based) and vals float64.
"""
from __future__ import annotations

import numpy as np


def uniform_distinct(dims, nnz, seed, low=0.0):
    """`nnz` distinct coordinates drawn uniformly without replacement;
    values uniform in (0, 1] (config 1: 1000x800x600, 1M nonzeros)."""
    dims = [int(d) for d in dims]
    total = int(np.prod(np.array(dims, dtype=object)))
    if nnz > total:
        raise ValueError("more nonzeros than coordinates")
    rng = np.random.default_rng(seed)
    if total < 2**62:
        picked = np.zeros(0, np.int64)
        while picked.size < nnz:
            need = int((nnz - picked.size) * 1.2) + 16
            cand = rng.integers(0, total, size=need, dtype=np.int64)
            picked = np.unique(np.concatenate([picked, cand]))
        picked = rng.permutation(picked)[:nnz]
        cidx = np.zeros((len(dims), nnz), np.uint64)
        rem = picked.copy()
        for n in range(len(dims) - 1, -1, -1):
            cidx[n] = (rem % dims[n]).astype(np.uint64)
            rem //= dims[n]
    else:
        cidx = np.stack([rng.integers(0, d, size=nnz * 2, dtype=np.int64) for d in dims]).astype(np.uint64)
        _, first = np.unique(cidx.T, axis=0, return_index=True)
        first = np.sort(first)[:nnz]
        if first.size < nnz:
            raise ValueError("could not draw enough distinct coordinates")
        cidx = np.ascontiguousarray(cidx[:, first])
    vals = 1.0 - rng.random(nnz)  # (0, 1]
    return np.array(dims, np.uint64), cidx, vals


def zipf_indices(rng, n, dim, s):
    """`n` draws of a Zipf(s) distribution truncated to [1, dim], returned
    0-based.  Draws above dim are redrawn (exact truncation)."""
    out = rng.zipf(s, size=n)
    bad = out > dim
    while bad.any():
        out[bad] = rng.zipf(s, size=int(bad.sum()))
        bad = out > dim
    return (out - 1).astype(np.uint64)


def merge_duplicates(dims, cidx, vals):
    """Sums values of repeated coordinates; output sorted lexicographically."""
    nm = cidx.shape[0]
    order = np.lexsort(cidx[::-1])
    c = cidx[:, order]
    v = vals[order]
    if c.shape[1] == 0:
        return c, v
    new = np.ones(c.shape[1], bool)
    new[1:] = np.any(c[:, 1:] != c[:, :-1], axis=0)
    run = np.cumsum(new) - 1
    out_v = np.zeros(int(new.sum()))
    np.add.at(out_v, run, v)
    return np.ascontiguousarray(c[:, new]), out_v


def zipf_tensor(dims, draws, seed, s=1.1, lognormal=True):
    """Config 2 shape: each mode index drawn independently from Zipf(s) over
    its dimension, duplicates merged by summing, values log-normal(0, 1)."""
    rng = np.random.default_rng(seed)
    cidx = np.stack([zipf_indices(rng, draws, int(d), s) for d in dims])
    vals = rng.lognormal(0.0, 1.0, size=draws) if lognormal else 1.0 - rng.random(draws)
    cidx, vals = merge_duplicates(np.array(dims), cidx, vals)
    return np.array(dims, np.uint64), cidx, vals


def poisson_kruskal(dims, rank, total_counts, seed, shape=0.3, scale=1.0):
    """Config 3 shape: Poisson counts from a Kruskal model with Gamma(shape,
    scale) factor entries (columns normalised to probabilities, unit weights).
    Each of `total_counts` events picks a component uniformly and then one
    index per mode from that component's column; repeated coordinates are
    merged into counts."""
    rng = np.random.default_rng(seed)
    nm = len(dims)
    cols = []
    for d in dims:
        A = rng.gamma(shape, scale, size=(int(d), rank))
        A /= A.sum(axis=0, keepdims=True)
        cols.append(np.cumsum(A, axis=0))
    comp = rng.integers(0, rank, size=total_counts)
    cidx = np.zeros((nm, total_counts), np.uint64)
    for n in range(nm):
        u = rng.random(total_counts)
        cdf = cols[n]
        idx = np.empty(total_counts, np.int64)
        for r in range(rank):
            sel = comp == r
            idx[sel] = np.searchsorted(cdf[:, r], u[sel], side="right")
        cidx[n] = np.minimum(idx, int(dims[n]) - 1).astype(np.uint64)
    cidx, vals = merge_duplicates(np.array(dims), cidx, np.ones(total_counts))
    return np.array(dims, np.uint64), cidx, vals


def random_factors(dims, rank, seed):
    """Uniform(0,1) factor matrices from numpy (for parity inputs)."""
    rng = np.random.default_rng(seed)
    return [rng.random((int(d), rank)) for d in dims]


# ------------------------------------------------- batched / served streams

def batch_shapes(count, seed, ranks=(8, 16, 32, 64), dim_range=(100, 50_000), nnz_range=(10_000, 2_000_000),
                 orders=(3, 4, 5)):
    """Shapes of the batched CP-ALS workload: order uniform over `orders`,
    every dimension log-uniform in dim_range, nnz log-uniform in nnz_range,
    rank uniform over `ranks`.  Returns [(dims, nnz, rank), ...]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nm = int(rng.choice(orders))
        dims = tuple(int(round(np.exp(rng.uniform(np.log(dim_range[0]), np.log(dim_range[1]))))) for _ in range(nm))
        nnz = int(round(np.exp(rng.uniform(np.log(nnz_range[0]), np.log(nnz_range[1])))))
        out.append((dims, nnz, int(rng.choice(ranks))))
    return out


def uniform_coo_torch(dims, nnz, seed, device):
    """`nnz` coordinates drawn uniformly (with replacement; repeated
    coordinates stay separate nonzeros, which CP-ALS treats as their sum) and
    values uniform in (0, 1], generated on `device`.  Returns (cidx int64
    (nmode, nnz), vals float64)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    cidx = torch.stack([torch.randint(0, int(d), (nnz,), generator=g, device=device, dtype=torch.int64)
                        for d in dims]).contiguous()
    vals = 1.0 - torch.rand(nnz, generator=g, device=device, dtype=torch.float64)
    return cidx, vals


def poisson_kruskal_torch(dims, rank, total_counts, seed, device, shape=0.3, scale=1.0):
    """poisson_kruskal on `device`: each of `total_counts` events picks a
    component uniformly, then one index per mode from that component's
    Gamma(shape, scale) column (normalised); repeated coordinates are merged
    into INT32 counts.  Returns (cidx int64 (nmode, nnz), vals int32)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    rng = np.random.default_rng(seed)  # the factor columns (dims x rank) are small: drawn on the host
    comp = torch.randint(0, rank, (total_counts,), generator=g, device=device)
    idx = []
    for d in dims:
        d = int(d)
        A = torch.from_numpy(rng.gamma(shape, scale, size=(d, rank))).to(device)
        A /= A.sum(dim=0, keepdim=True)
        cdf = torch.cumsum(A, 0)
        cdf /= cdf[-1:].clone()
        # column r of the flattened table holds r + cdf[:, r], so one sorted search serves every component
        flat = (cdf.t() + torch.arange(rank, device=device, dtype=torch.float64)[:, None]).reshape(-1)
        u = torch.rand(total_counts, generator=g, device=device, dtype=torch.float64) * (1 - 1e-12)
        pos = torch.searchsorted(flat, u + comp.double(), right=True)
        idx.append((pos - comp * d).clamp_(0, d - 1))
    # merge repeated coordinates: lexicographic order by stable sorts, last mode first
    order = torch.arange(total_counts, device=device)
    for i in reversed(idx):
        order = order[torch.sort(i[order], stable=True).indices]
    cs = torch.stack([i[order] for i in idx])
    new = torch.ones(total_counts, dtype=torch.bool, device=device)
    new[1:] = (cs[:, 1:] != cs[:, :-1]).any(dim=0)
    seg = torch.cumsum(new.to(torch.int64), 0) - 1
    nnz = int(seg[-1].item()) + 1
    counts = torch.zeros(nnz, dtype=torch.int32, device=device).index_add_(0, seg, torch.ones_like(seg, dtype=torch.int32))
    return cs[:, new].contiguous(), counts


CONFIG3_DIMS = (20_000, 10_000, 5_000, 200)


def served_stream(count, seed, rate=200.0, als_frac=0.7, ranks=(16, 32, 64), nnz_range=(50_000, 20_000_000),
                  dims=CONFIG3_DIMS, model_rank=8):
    """The served request stream: Poisson arrivals at `rate` per second;
    each request is CP-ALS (probability als_frac) or CP-APR on a tensor
    generated as the CP-APR benchmark tensor is: `dims` (4-mode 20,000 x
    10,000 x 5,000 x 200), Poisson counts from a rank-`model_rank`
    Gamma(0.3, 1) Kruskal model (poisson_kruskal_torch) with a count total
    log-uniform in nnz_range; CP-ALS requests decompose the counts as FP32
    values.  Rank uniform over `ranks`.
    Returns [(arrival_s, kind, dims, total_counts, rank, seed), ...]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(count):
        t += rng.exponential(1.0 / rate)
        kind = "als" if rng.random() < als_frac else "apr"
        nnz = int(round(np.exp(rng.uniform(np.log(nnz_range[0]), np.log(nnz_range[1])))))
        out.append((t, kind, tuple(int(d) for d in dims), nnz, int(rng.choice(ranks)), int(rng.integers(1, 2**31))))
    return out


def zipf_tensor_torch(dims, draws, s, seed, device):
    """Config-2 tensor generated on the device: inverse-CDF Zipf draws per
    mode, duplicate coordinates merged by summing log-normal values."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    idx = []
    for d in dims:
        k = torch.arange(1, d + 1, dtype=torch.float64, device=device)
        cdf = torch.cumsum(k.pow(-s), 0)
        cdf /= cdf[-1].clone()
        u = torch.rand(draws, dtype=torch.float64, device=device, generator=g)
        i = torch.searchsorted(cdf, u, right=True).clamp_(max=d - 1)
        idx.append(i)
        del k, cdf, u
    vals = torch.exp(torch.randn(draws, dtype=torch.float64, device=device, generator=g))
    low = idx[1] * dims[2] + idx[2]
    o1 = torch.sort(low, stable=True).indices
    o2 = torch.sort(idx[0][o1], stable=True).indices
    order = o1[o2]
    del o1, o2
    i0, lo, v = idx[0][order], low[order], vals[order]
    del idx, low, vals, order
    new = torch.ones_like(i0, dtype=torch.bool)
    new[1:] = (i0[1:] != i0[:-1]) | (lo[1:] != lo[:-1])
    seg = torch.cumsum(new.to(torch.int64), 0) - 1
    nnz = int(seg[-1].item()) + 1
    vs = torch.zeros(nnz, dtype=torch.float64, device=device).index_add_(0, seg, v)
    keep = new.nonzero().squeeze(1)
    i0, lo = i0[keep], lo[keep]
    cidx = torch.stack([i0, lo // dims[2], lo % dims[2]]).contiguous()
    return cidx, vs.to(torch.float32), nnz
