"""TEST INFRASTRUCTURE ONLY: numpy restatement of personalised PageRank over a
weighted graph and of its adjoint, the checker of alpb_ppr_* (only tests/ use
it; the product never does).

The forward iteration is algorithms::simple_pagerank
(include/graphblas/algorithms/simple_pagerank.hpp:146-533) with the uniform
teleport vector replaced by a one-hot one per seed and the out-degree count
replaced by the weighted out-degree d_i = sum_j w_ij:

* the row scale is alpha / d_i, zero for a dangling row (:281-289);
* each iteration pre-scales x by it and sums the mass of the dangling rows
  apart (:324-357), forms (alpha * dangling + 1 - alpha) (:390), multiplies
  (vxm over L, :400), adds the teleport term and measures the L1 change
  (:440-470); a seed stops after the iteration whose change is <= conv (:490)
  or at max_iter;
* the initial guess is 1/n (:215).

With unit weights and no dangling rows, the mean of the personalised vectors
over all n seeds is simple_pagerank's vector (linearity in the teleport
vector); the tests pin this restatement to the compiled reference that way.

Adjoint (implicit function theorem on the fixed point
x = alpha M x + alpha v 1_D^T x + (1 - alpha) v, M_ji = w_ij / d_i):
  lambda = alpha M^T lambda + alpha 1_D lambda[seed] + dL/dx,
  dL/dw_ij = alpha / d_i sum_s x_is (lambda_js - (M^T lambda_s)_i).
"""
from __future__ import annotations

import numpy as np


def _rows(rp):
    return np.repeat(np.arange(len(rp) - 1), np.diff(rp))


def degrees(rp, w):
    n = len(rp) - 1
    return np.bincount(_rows(rp), weights=np.asarray(w, np.float64), minlength=n)


def _gather_cols(n, rows, cols, w, y):
    """acc[j] = sum_i w_ij y[i], summed in storage order."""
    acc = np.zeros((n, y.shape[1]))
    np.add.at(acc, cols, w[:, None] * y[rows])
    return acc


def forward(rp, col, w, seeds, alpha=0.85, conv=1e-9, max_iter=1000, x0=None):
    """Returns (x [n, S], iterations [S], residuals [S])."""
    n = len(rp) - 1
    seeds = np.asarray(seeds, np.int64)
    S = len(seeds)
    rows, cols, w = _rows(rp), np.asarray(col, np.int64), np.asarray(w, np.float64)
    d = degrees(rp, w)
    dangling = d == 0
    rs = np.where(dangling, 0.0, alpha / np.where(dangling, 1.0, d))
    x = np.full((n, S), 1.0 / n) if x0 is None else np.array(x0, np.float64, copy=True)
    term = alpha * x[dangling].sum(0) + 1 - alpha
    active = np.ones(S, bool)
    iters = np.zeros(S, np.int64)
    res = np.zeros(S)
    k = 0
    while active.any() and k < max_iter:
        k += 1
        y = x * rs[:, None]
        nw = _gather_cols(n, rows, cols, w, y)
        nw[seeds, np.arange(S)] += term
        r = np.abs(x - nw).sum(0)
        dng = nw[dangling].sum(0)
        for s in np.flatnonzero(active):
            x[:, s] = nw[:, s]
            res[s] = r[s]
            iters[s] = k
            term[s] = alpha * dng[s] + 1 - alpha
            if (conv != 0 and r[s] <= conv) or k >= max_iter:
                active[s] = False
    return x, iters, res


def adjoint(rp, col, w, seeds, g, alpha=0.85, conv=1e-9, max_iter=1000):
    """lambda for dL/dx = g; returns (lambda [n, S], iterations, residuals)."""
    n = len(rp) - 1
    seeds = np.asarray(seeds, np.int64)
    S = len(seeds)
    rows, cols, w = _rows(rp), np.asarray(col, np.int64), np.asarray(w, np.float64)
    d = degrees(rp, w)
    dangling = d == 0
    inv_d = np.where(dangling, 0.0, 1.0 / np.where(dangling, 1.0, d))
    g = np.asarray(g, np.float64)
    lam = g.copy()
    active = np.ones(S, bool)
    iters = np.zeros(S, np.int64)
    res = np.zeros(S)
    k = 0
    while active.any() and k < max_iter:
        k += 1
        term = alpha * lam[seeds, np.arange(S)]
        acc = np.zeros((n, S))
        np.add.at(acc, rows, w[:, None] * lam[cols])
        nw = alpha * (acc * inv_d[:, None]) + np.where(dangling[:, None], term[None, :], 0.0) + g
        r = np.abs(nw - lam).sum(0)
        for s in np.flatnonzero(active):
            lam[:, s] = nw[:, s]
            res[s] = r[s]
            iters[s] = k
            if (conv != 0 and r[s] <= conv) or k >= max_iter:
                active[s] = False
    return lam, iters, res


def grad_weights(rp, col, w, x, lam, alpha=0.85):
    """dL/dw for every stored edge (CRS order)."""
    n = len(rp) - 1
    rows, cols, w = _rows(rp), np.asarray(col, np.int64), np.asarray(w, np.float64)
    d = degrees(rp, w)
    dangling = d == 0
    inv_d = np.where(dangling, 0.0, 1.0 / np.where(dangling, 1.0, d))
    acc = np.zeros_like(lam)
    np.add.at(acc, rows, w[:, None] * lam[cols])
    mu = acc * inv_d[:, None]
    c = (x * mu).sum(1)
    dot = (x[rows] * lam[cols]).sum(1)
    return alpha * inv_d[rows] * (dot - c[rows])
