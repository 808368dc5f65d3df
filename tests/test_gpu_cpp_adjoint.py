"""The differentiated solvers of the b200 C++ API (graphblas/b200/algorithms.hpp)
through tests/cpp/diff_driver.cpp: the forward CG is ALP's own
algorithms::conjugate_gradient compiled for b200, followed by
grb::algorithms::conjugate_gradient_adjoint; personalised PageRank runs the
PersonalisedPageRank class.  Checked against the plain-C restatement's CG (for x
and for lambda = A^{-T} (x - x*)) with the gradient assembled on the host as
-lambda_i x_j, and against the numpy restatement of personalised PageRank."""
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from oracle import ppr as O
from oracle.oracle import FP64, crs_to_coo

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
DRIVER = ROOT / "_build" / "cpp" / "diff_driver_b200"


def run(what, d):
    if not DRIVER.exists():
        pytest.fail(f"{DRIVER} is not built (build() compiles it where the ALP sources exist)")
    r = subprocess.run([str(DRIVER), what, str(d)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    out = {}
    for line in r.stdout.splitlines():
        k, v = line.split()
        out.setdefault(k, []).append(int(v))
    return out


def write_coo(path, n, I, J, V):
    with open(path, "wb") as f:
        np.array([n, len(I)], np.int64).tofile(f)
        np.asarray(I, np.uint32).tofile(f)
        np.asarray(J, np.uint32).tofile(f)
        np.asarray(V, np.float64).tofile(f)


def key(i, j, n):
    return np.asarray(i, np.int64) * n + np.asarray(j, np.int64)


def test_cg_adjoint_cpp_api(cuda, oracle):
    """27-point 8^3 pattern, off-diagonals -U(0.5, 1.5) symmetric, diagonal
    1.05 |row sum|; L = 0.5 ||x - x*||^2."""
    I, J, _ = oracle.stencil_coo((8, 8, 8), 1.0, 1.0)
    n = 512
    lo, hi = np.minimum(I, J).astype(np.int64), np.maximum(I, J).astype(np.int64)
    V = -(0.5 + (np.sin(lo * 12.9898 + hi * 78.233) * 43758.5453 % 1.0 + 1.0) % 1.0)
    off = I != J
    rowsum = np.bincount(I[off], weights=np.abs(V[off]), minlength=n)
    V = np.where(off, V, 1.05 * rowsum[I])
    rng = np.random.default_rng(3)
    b, xs = rng.standard_normal(n), rng.standard_normal(n)
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        write_coo(d / "A.bin", n, I, J, V)
        b.tofile(d / "b.bin")
        xs.tofile(d / "xstar.bin")
        out = run("cg", d)
        x = np.fromfile(d / "x.bin")
        lam = np.fromfile(d / "lambda.bin")
        grad = np.fromfile(d / "grad.bin")
        order = np.fromfile(d / "order.bin", np.uint32).reshape(-1, 2)
    assert out["rc"] == [0]
    rp, col, vals = oracle.coo_to_crs(n, I, J, V, FP64)
    rc, xo, ito, _ = oracle.cg(rp, col, vals, b, np.zeros(n), 5000, 1e-12)
    assert rc == 0 and out["iterations_fwd"] == [ito]
    np.testing.assert_allclose(x, xo, rtol=0, atol=1e-10 * np.abs(xo).max())
    # A is symmetric: A^T lambda = x - x* on the same storage
    rc, lo_, ita, _ = oracle.cg(rp, col, vals, x - xs, np.zeros(n), 5000, 1e-12)
    assert rc == 0 and abs(out["iterations_adj"][0] - ita) <= 1
    np.testing.assert_allclose(lam, lo_, rtol=0, atol=1e-9 * np.abs(lo_).max())
    assert len(order) == len(I)
    np.testing.assert_allclose(grad, -lam[order[:, 0]] * x[order[:, 1]], rtol=1e-14, atol=0)


def test_personalised_pagerank_cpp_api(cuda, oracle):
    rp, col, w = oracle.rmat(8, seed=13, vtype=FP64)
    n = len(rp) - 1
    rows, cols = crs_to_coo(rp, col)
    S = 10
    rng = np.random.default_rng(8)
    seeds = rng.integers(0, n, S)
    g = rng.standard_normal((n, S))
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        write_coo(d / "W.bin", n, rows, cols, w)
        with open(d / "seeds.bin", "wb") as f:
            np.array([S], np.int64).tofile(f)
            np.asarray(seeds, np.int64).tofile(f)
        g.reshape(-1).tofile(d / "g.bin")
        out = run("ppr", d)
        X = np.fromfile(d / "X.bin").reshape(n, S)
        L = np.fromfile(d / "Lambda.bin").reshape(n, S)
        grad = np.fromfile(d / "grad.bin")
        order = np.fromfile(d / "order.bin", np.uint32).reshape(-1, 2)
    assert out["rc"] == [0]
    xo, ito, _ = O.forward(rp, col, w, seeds, conv=1e-10)
    np.testing.assert_array_equal(out["iterations_fwd"], ito)
    np.testing.assert_allclose(X, xo, rtol=1e-11, atol=1e-11 * np.abs(xo).max())
    lo, itao, _ = O.adjoint(rp, col, w, seeds, g, conv=1e-10)
    np.testing.assert_array_equal(out["iterations_adj"], itao)
    np.testing.assert_allclose(L, lo, rtol=1e-11, atol=1e-11 * np.abs(lo).max())
    go = O.grad_weights(rp, col, w, xo, lo)
    # map the iterator's order onto the restatement's CRS order
    pos = {k: p for p, k in enumerate(key(rows, cols, n).tolist())}
    idx = np.array([pos[k] for k in key(order[:, 0], order[:, 1], n).tolist()])
    np.testing.assert_allclose(grad, go[idx], rtol=1e-9, atol=1e-9 * np.abs(go).max())
