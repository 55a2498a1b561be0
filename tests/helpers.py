"""Shared helpers for the parity tests."""
import numpy as np


def pext_rows(idx_words, mask_words):
    """Mode indices of 128-bit keys (lo, hi words) under a mask: a plain
    bit-by-bit extract, independent of the code under test."""
    lo, hi = idx_words[:, 0].astype(object), idx_words[:, 1].astype(object)
    keys = [int(l) | (int(h) << 64) for l, h in zip(lo, hi)]
    m = int(mask_words[0]) | (int(mask_words[1]) << 64)
    bits = [b for b in range(128) if (m >> b) & 1]
    out = np.zeros(len(keys), np.uint64)
    for i, k in enumerate(keys):
        v = 0
        for j, b in enumerate(bits):
            v |= ((k >> b) & 1) << j
        out[i] = v
    return out


def mttkrp_from_golden(g, mode, synth):
    """Reference MTTKRP output (dense) for a golden case and mode."""
    dims = g["dims"]
    rank = int(g["rank"])
    U = synth.random_factors(dims, rank, seed=100 + mode)
    out = U[mode].copy()
    rows = g[f"mttkrp{mode}_rows"]
    out[rows] += g[f"mttkrp{mode}_delta"]
    return U, out
