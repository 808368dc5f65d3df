"""The personalised-PageRank restatement (oracle/ppr.py) pinned on the CPU:
the mean over all seeds against the compiled ALP reference's simple_pagerank,
and its adjoint gradient against central finite differences of itself."""
import numpy as np

from oracle import ppr as O
from oracle.oracle import FP64, VOID, crs_to_coo


def no_dangling_unit_graph(R, scale, seed):
    rp, col, _ = R.rmat(scale, seed=seed, vtype=VOID)
    n = len(rp) - 1
    rows, cols = crs_to_coo(rp, col)
    have = set(zip(rows.tolist(), cols.tolist()))
    extra = np.array([i for i in range(n) if (i, i) not in have], np.uint32)
    I = np.concatenate([rows, extra])
    J = np.concatenate([cols, extra])
    order = np.lexsort((J, I))
    I, J = I[order], J[order]
    rp2 = np.concatenate([[0], np.cumsum(np.bincount(I, minlength=n))]).astype(np.int64)
    return n, rp2, I, J


def test_mean_over_seeds_is_reference_pagerank(oracle, reference):
    n, rp, I, J = no_dangling_unit_graph(oracle, 6, 5)
    V = np.ones(len(J))
    x, it, _ = O.forward(rp, J, V, np.arange(n), conv=0.0, max_iter=200)
    rc, pr, itr, _ = reference.pagerank(n, I, J, V, alpha=0.85, conv=0.0, max_iter=200)
    assert rc in (0, 8) and itr == 200 and (it == 200).all()
    np.testing.assert_allclose(x.mean(1), pr, rtol=1e-12, atol=1e-16)


def test_all_dangling_rows_give_the_seed_vector(oracle):
    """No edges: every row dangles, so the teleport term is alpha * 1 + 1 - alpha
    = 1 and x = e_seed after the first iteration; the second sees no change."""
    n = 8
    rp = np.zeros(n + 1, np.int64)
    x, it, res = O.forward(rp, np.zeros(0, np.int64), np.zeros(0), [2], conv=1e-12)
    e = np.zeros((n, 1))
    e[2, 0] = 1
    np.testing.assert_allclose(x, e, atol=1e-16)
    assert it[0] == 2 and res[0] == 0.0


def test_gradient_matches_central_differences(oracle):
    rp, col, w = oracle.rmat(6, seed=9, vtype=FP64)
    w = 0.5 + w
    n = len(rp) - 1
    rng = np.random.default_rng(4)
    seeds = rng.integers(0, n, 4)
    target = rng.standard_normal((n, 4)) * 0.01

    def loss(wv):
        x, _, _ = O.forward(rp, col, wv, seeds, conv=0.0, max_iter=300)
        return 0.5 * ((x - target) ** 2).sum(), x

    L0, x = loss(w)
    lam, _, _ = O.adjoint(rp, col, w, seeds, x - target, conv=0.0, max_iter=300)
    g = O.grad_weights(rp, col, w, x, lam)
    h = 1e-6
    for k in rng.choice(len(col), 12, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (loss(wp)[0] - loss(wm)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * abs(g[k]) + 1e-7 * np.abs(g).max(), (k, fd, g[k])


def test_c_restatement_equals_numpy_restatement(oracle):
    """ppr_oracle.c (the benchmark-scale checker) against oracle/ppr.py on a
    weighted R-MAT graph with dangling rows: the same iteration counts, and
    iterates equal to the last bits (same sums in the same order)."""
    rp, col, w = oracle.rmat(9, seed=21, vtype=FP64)
    n = len(rp) - 1
    rng = np.random.default_rng(7)
    seeds = rng.integers(0, n, 11)
    seeds[3] = seeds[7]                      # a repeated seed
    x, it, res = O.forward(rp, col, w, seeds, conv=1e-10)
    xc, itc, resc = oracle.ppr_forward(rp, col, w, seeds, conv=1e-10)
    assert (it == itc).all()
    np.testing.assert_allclose(xc, x, rtol=1e-14, atol=1e-300)
    np.testing.assert_allclose(resc, res, rtol=1e-12, atol=1e-300)
    g = rng.standard_normal((n, len(seeds)))
    lam, ita, _ = O.adjoint(rp, col, w, seeds, g, conv=1e-10)
    lamc, itac, _ = oracle.ppr_adjoint(rp, col, w, seeds, g, conv=1e-10)
    assert (ita == itac).all()
    np.testing.assert_allclose(lamc, lam, rtol=1e-13, atol=1e-13 * np.abs(lam).max())
    gr = O.grad_weights(rp, col, w, x, lam)
    grc = oracle.ppr_grad(rp, col, w, x, lam)
    np.testing.assert_allclose(grc, gr, rtol=1e-11, atol=1e-13 * np.abs(gr).max())
    # a warm start and a budget stop
    x2, it2, _ = O.forward(rp, col, w, seeds, conv=0.0, max_iter=5, x0=x)
    x2c, it2c, _ = oracle.ppr_forward(rp, col, w, seeds, conv=0.0, max_iter=5, x0=x)
    assert (it2 == 5).all() and (it2c == 5).all()
    np.testing.assert_allclose(x2c, x2, rtol=1e-14, atol=1e-300)
