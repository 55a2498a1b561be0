"""The cpd64 command-line driver (the reference's flags, src/main.cpp:70-92)
built on the C++ drop-in header: usage on the host, and on the GPU the
CP-ALS fit lines and CP-APR summary lines the reference printed for the same
tensor, seed and partitions."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "alto_b200", "bin", "cpd64")
needs_cli = pytest.mark.skipif(not os.path.exists(CLI), reason="bin/cpd64 is built by make -C alto_b200")


def _write_tns(path, cidx, vals):
    with open(path, "w") as f:
        f.write("# written by the CLI test\n")
        for k in range(len(vals)):
            f.write(" ".join(str(int(c) + 1) for c in cidx[:, k]) + f" {float(vals[k]):.17g}\n")


def _run(args):
    return subprocess.run([CLI] + [str(a) for a in args], capture_output=True, text=True, timeout=300)


@needs_cli
def test_cli_usage_and_missing_input():
    r = _run(["-h"])
    assert r.returncode == 0 and "--rank" in r.stdout and "-l, --model" in r.stdout
    r = _run(["-l", "als"])
    assert r.returncode != 0 and "no input" in r.stderr


@pytest.mark.gpu
@needs_cli
def test_cli_cp_als_prints_the_reference_fits(tmp_path):
    g = load_golden("cpd_u3")
    path = tmp_path / "t.tns"
    _write_tns(path, g["cidx"], g["vals"])
    r = _run(["-l", "als", "-i", path, "--rank", int(g["rank"]), "-m", int(g["max_iters"]), "-e", "1e-30",
              "-x", int(g["seed"]), "--nprtn", int(g["nprtn"])])
    assert r.returncode == 0, r.stderr
    fits = [float(m) for m in re.findall(r"it: \d+\s+fit: (\S+)", r.stdout)]
    np.testing.assert_allclose(fits, g["fits"], rtol=2e-5)  # both printed with %g


@pytest.mark.gpu
@needs_cli
def test_cli_cp_apr_prints_the_reference_summary(tmp_path):
    g = load_golden("apr_eps")
    path = tmp_path / "t.tns"
    _write_tns(path, g["cidx"], g["vals"])
    r = _run(["-l", "apr", "-i", path, "--rank", int(g["rank"]), "-m", int(g["max_iters"]), "-n",
              int(g["max_inner"]), "-e", repr(float(g["eps"])), "-x", int(g["seed"]), "--nprtn", int(g["nprtn"])])
    assert r.returncode == 0, r.stderr
    ll = float(re.search(r"Final log-likelihood = (\S+)", r.stdout).group(1))
    outer = int(re.search(r"Total outer iterations = (\d+)", r.stdout).group(1))
    inner = int(re.search(r"Total inner iterations = (\d+)", r.stdout).group(1))
    assert (outer, inner) == (int(g["outer"]), int(g["inner"]))
    np.testing.assert_allclose(ll, g["loglik"], rtol=1e-6)


@pytest.mark.gpu
@needs_cli
def test_cli_check_and_bench_modes(tmp_path):
    g = load_golden("cpd_u3")
    path = tmp_path / "t.tns"
    _write_tns(path, g["cidx"], g["vals"])
    r = _run(["-l", "als", "-i", path, "--rank", 8, "-c", "-x", 3])
    assert r.returncode == 0, r.stderr
    assert r.stderr.count("Results of mttkrp_alto is correct") == 3
    r = _run(["-l", "als", "-i", path, "--rank", 8, "-p", "-m", 3, "-t", 1])
    assert r.returncode == 0 and "ALTO runtime:" in r.stdout


@pytest.mark.gpu
@needs_cli
def test_cli_generates_the_reference_poisson_tensor():
    """cpd64 -d dims -s sparsity -r rank (MakeSparseTensor, main.cpp:652-675)
    draws the tensor the reference's generator draws with the same OpenMP
    thread count (the nonzero count it prints; the full tensor is compared
    in test_poisson_gpu.py)."""
    orc = pytest.importorskip("oracle.orc")
    if not os.path.exists(orc.REF_SO_POISSON):
        pytest.skip("reference generator library not built")
    dims, sparsity, rank = (40, 30, 20), 0.5, 4
    edges = int(sparsity * 40 * 30 * 20)
    _, rv, _, _ = orc.RefPoisson().run(dims, edges, rank, 2)
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run([CLI, "-d", "40,30,20", "-s", str(sparsity), "-r", str(rank), "-l", "als", "-m", "2",
                        "-x", "3"], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr
    m = re.search(r"Creating a new tensor: [0-9.e+-]+ s \((\d+) nonzeros\)", r.stdout)
    assert m and int(m.group(1)) == rv.shape[0], r.stdout
