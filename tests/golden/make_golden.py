"""Writes the golden fixtures in this directory from the REFERENCE itself.

The reference (IntelLabs/ALTO) is compiled from its own sources by
oracle/build_ref.sh into oracle/_ref/libaltoref.so; this script calls its
create_alto, mttkrp_alto_par, cpd_alto and cp_apr_alto through
oracle/ref_harness.cpp and stores inputs and outputs as .npz files.

    python oracle/build_ref.sh && python tests/golden/make_golden.py

Inputs are small seeded synthetic tensors (alto_b200/synth.py); factor
matrices for MTTKRP come from numpy's seeded generator; CP-ALS / CP-APR start
from the reference's own KruskalModelRandomInit(seed).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from alto_b200 import synth  # noqa: E402
from oracle.orc import RefLib  # noqa: E402

# name: (generator, nprtn, lit_bits, rank, mttkrp?)
CASES = {
    "u3": (lambda: synth.uniform_distinct((45, 37, 29), 2500, seed=11), 7, 64, 8, True),
    "u3_lit128": (lambda: synth.uniform_distinct((45, 37, 29), 2500, seed=11), 4, 128, 8, True),
    "mixed4": (lambda: synth.uniform_distinct((200, 3000, 50, 7), 5000, seed=12), 6, 64, 8, True),
    "low3_64": (lambda: synth.uniform_distinct((5000, 4000, 3000), 6000, seed=13), 8, 64, 4, True),
    "low5_66bits": (lambda: synth.uniform_distinct((8192, 8000, 6000, 5000, 9000), 3000, seed=14), 5, 128, 4,
                    True),
    "z3_65bits": (lambda: synth.zipf_tensor((4_800_000, 1_800_000, 1_800_000), 3000, seed=15), 4, 128, 0, False),
    "odd_rank": (lambda: synth.uniform_distinct((60, 70, 80), 4000, seed=16), 3, 64, 5, True),
}


def gen_case(ref, name):
    gen, nprtn, lit, rank, do_mttkrp = CASES[name]
    dims, cidx, vals = gen()
    out = dict(dims=dims, cidx=cidx, vals=vals, nprtn=np.int64(nprtn), lit_bits=np.int64(lit),
               rank=np.int64(rank))
    enc = ref.create_dump(dims, cidx, vals, nprtn, lit)
    for k in ("idx", "vals", "prtn_ptr", "intervals", "masks", "cr_masks", "oidx"):
        out["enc_" + k] = enc[k]
    out["enc_alto_bits"] = np.int64(enc["alto_bits"])
    out["enc_is_oidx"] = np.int64(enc["is_oidx"])
    if do_mttkrp:
        for mode in range(len(dims)):
            U = synth.random_factors(dims, rank, seed=100 + mode)
            init = U[mode].copy()
            ref.mttkrp(dims, cidx, vals, nprtn, lit, mode, U, rank)
            delta = U[mode] - init
            rows = np.nonzero(np.any(delta != 0, axis=1))[0]
            out[f"mttkrp{mode}_rows"] = rows.astype(np.int64)
            out[f"mttkrp{mode}_delta"] = delta[rows]
    return out


def gen_cpd(ref):
    dims, cidx, vals = synth.uniform_distinct((45, 37, 29), 2500, seed=11)
    U, lam, fits = ref.cpd(dims, cidx, vals, 7, 64, 8, 12, 1e-30, 5)
    out = dict(dims=dims, cidx=cidx, vals=vals, nprtn=np.int64(7), rank=np.int64(8), max_iters=np.int64(12),
               seed=np.int64(5), fits=fits, lam=lam)
    for n, u in enumerate(U):
        out[f"U{n}"] = u
    return out


def gen_cpd_conv(ref):
    """Converging run (epsilon 1e-4) to pin the stopping rule."""
    dims, cidx, vals = synth.uniform_distinct((30, 40, 20, 10), 3000, seed=21)
    U, lam, fits = ref.cpd(dims, cidx, vals, 5, 64, 6, 50, 1e-4, 9)
    out = dict(dims=dims, cidx=cidx, vals=vals, nprtn=np.int64(5), rank=np.int64(6), max_iters=np.int64(50),
               eps=np.float64(1e-4), seed=np.int64(9), fits=fits, lam=lam)
    for n, u in enumerate(U):
        out[f"U{n}"] = u
    return out


def gen_apr(ref, dobench):
    dims, cidx, vals = synth.poisson_kruskal((30, 25, 20), 4, 6000, seed=31)
    U, lam, s = ref.apr(dims, cidx, vals, 6, 64, 5, 6, 5, 1e-4, 1e-10, 1e-10, 1e-2, dobench, 7)
    out = dict(dims=dims, cidx=cidx, vals=vals, nprtn=np.int64(6), rank=np.int64(5), max_iters=np.int64(6),
               max_inner=np.int64(5), eps=np.float64(1e-4), seed=np.int64(7), dobench=np.int64(dobench),
               loglik=np.float64(s["loglik"]), fit=np.float64(s["fit"]), kkt=np.float64(s["kkt"]),
               outer=np.int64(s["outer"]), inner=np.int64(s["inner"]), lam=lam)
    for n, u in enumerate(U):
        out[f"U{n}"] = u
    return out


def gen_config1_fits(ref):
    """Fit trajectory of the config-1 workload (1000x800x600, 1M distinct
    nonzeros, rank 16, 20 iterations, glibc srand(1) factors)."""
    dims, cidx, vals = synth.uniform_distinct((1000, 800, 600), 1_000_000, seed=1)
    U, lam, fits = ref.cpd(dims, cidx, vals, 8, 64, 16, 20, 1e-30, 1)
    return dict(fits=fits, lam=lam, nprtn=np.int64(8), seed=np.int64(1), data_seed=np.int64(1))


def main():
    ref = RefLib()
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, f"enc_{name}.npz"), **gen_case(ref, name))
        print("wrote", name)
    np.savez_compressed(os.path.join(HERE, "cpd_u3.npz"), **gen_cpd(ref))
    np.savez_compressed(os.path.join(HERE, "cpd_conv4.npz"), **gen_cpd_conv(ref))
    np.savez_compressed(os.path.join(HERE, "apr_bench.npz"), **gen_apr(ref, 1))
    np.savez_compressed(os.path.join(HERE, "apr_eps.npz"), **gen_apr(ref, 0))
    np.savez_compressed(os.path.join(HERE, "cpd_config1_fits.npz"), **gen_config1_fits(ref))
    print("done")


if __name__ == "__main__":
    main()
