"""Personalised PageRank and its adjoint (alpb_ppr_*) against the numpy
restatement (oracle/ppr.py), central finite differences, and -- through the
mean over all seeds -- the compiled ALP reference's simple_pagerank.

Parity bars (FP64): forward and adjoint iterates within a relative 1e-11 of
the restatement with the same per-seed iteration counts; gradients within a
relative 1e-9 of the restatement and 1e-5 of central differences (h = 1e-6)."""
import ctypes as C

import numpy as np
import pytest

from oracle import ppr as O

pytestmark = pytest.mark.gpu


class Ppr:
    """Thin host wrapper over the C-ABI (device tensors in, device tensors out)."""

    def __init__(self, rp, col, w, nseeds):
        import torch
        from alp_b200 import _abi as abi
        from alp_b200 import device as dev
        self.n = len(rp) - 1
        self.nnz = len(col)
        self.S = nseeds
        self.rp = torch.from_numpy(np.asarray(rp, np.int64)).cuda()
        self.col = torch.from_numpy(np.asarray(col, np.int32)).cuda() if self.nnz else \
            torch.zeros(1, dtype=torch.int32, device="cuda")
        self.w = torch.from_numpy(np.asarray(w, np.float64)).cuda() if self.nnz else \
            torch.zeros(1, dtype=torch.float64, device="cuda")
        self.h = C.c_void_p()
        abi.call("alpb_ppr_create", C.byref(self.h), self.n, self.nnz, dev.ptr(self.rp),
                 dev.ptr(self.col), dev.ptr(self.w), nseeds, dev.stream_ptr())

    def info(self):
        from alp_b200 import _abi as abi
        v = [C.c_int64() for _ in range(4)]
        abi.call("alpb_ppr_info", self.h, *[C.byref(x) for x in v])
        return [x.value for x in v]

    def set_weights(self, w):
        import torch
        from alp_b200 import _abi as abi
        from alp_b200 import device as dev
        self.w = torch.from_numpy(np.asarray(w, np.float64)).cuda()
        abi.call("alpb_ppr_set_weights", self.h, dev.ptr(self.w), dev.stream_ptr())

    def solve(self, seeds, alpha=0.85, conv=1e-9, max_iter=1000, x0=None, expect_rc=0):
        import torch
        from alp_b200 import _abi as abi
        from alp_b200 import device as dev
        sd = np.ascontiguousarray(seeds, np.int64)
        x = torch.zeros(self.n * self.S, dtype=torch.float64, device="cuda") if x0 is None else \
            torch.from_numpy(np.ascontiguousarray(x0, np.float64).reshape(-1)).cuda()
        it = (C.c_int64 * self.S)()
        res = (C.c_double * self.S)()
        rc = abi.lib().alpb_ppr_solve(self.h, sd.ctypes.data_as(C.c_void_p), alpha, conv,
                                      max_iter, dev.ptr(x), int(x0 is not None), it, res,
                                      dev.stream_ptr())
        torch.cuda.synchronize()
        assert rc == expect_rc, abi.lib().alpb_last_error()
        return x, np.array(it), np.array(res)

    def adjoint(self, g, conv=1e-9, max_iter=1000):
        import torch
        from alp_b200 import _abi as abi
        from alp_b200 import device as dev
        lam = torch.empty_like(g)
        it = (C.c_int64 * self.S)()
        res = (C.c_double * self.S)()
        abi.call("alpb_ppr_adjoint", self.h, dev.ptr(g), dev.ptr(lam), conv, max_iter, it, res,
                 dev.stream_ptr())
        torch.cuda.synchronize()
        return lam, np.array(it), np.array(res)

    def grad(self, x, lam):
        import torch
        from alp_b200 import _abi as abi
        from alp_b200 import device as dev
        g = torch.empty(max(self.nnz, 1), dtype=torch.float64, device="cuda")
        abi.call("alpb_ppr_grad_weights", self.h, dev.ptr(x), dev.ptr(lam), dev.ptr(g),
                 dev.stream_ptr())
        torch.cuda.synchronize()
        return g[:self.nnz].cpu().numpy()

    def close(self):
        from alp_b200 import _abi as abi
        abi.lib().alpb_ppr_destroy(self.h)


def host(x, n, S):
    return x.view(n, S).cpu().numpy()


def rmat_weighted(oracle, scale, seed=7):
    """R-MAT graph (restatement's generator) with U(0,1) weights; dangling rows present."""
    from oracle.oracle import FP64
    rp, col, w = oracle.rmat(scale, seed=seed, vtype=FP64)
    return rp, col, w


@pytest.mark.parametrize("scale,S", [(8, 5), (9, 16), (10, 64), (9, 100), (8, 33)])
def test_forward_adjoint_gradient_match_restatement(cuda, oracle, scale, S):
    import torch
    rp, col, w = rmat_weighted(oracle, scale)
    n = len(rp) - 1
    rng = np.random.default_rng(scale * 1000 + S)
    seeds = rng.integers(0, n, S)
    seeds[-1] = seeds[0]                      # a repeated seed
    P = Ppr(rp, col, w, S)
    x, it, res = P.solve(seeds, conv=1e-10)
    xo, ito, reso = O.forward(rp, col, w, seeds, conv=1e-10)
    np.testing.assert_array_equal(it, ito)
    xh = host(x, n, S)
    np.testing.assert_allclose(xh, xo, rtol=1e-11, atol=1e-11 * np.abs(xo).max())
    # a residual sums |x_k - x_{k-1}| of iterates equal to ~1e-16 relative; the
    # differences are ~1e-5 of x near convergence, so ~1e-11 relative is all
    # the residual itself can carry: compare it loosely
    np.testing.assert_allclose(res, reso, rtol=1e-3, atol=1e-20)
    np.testing.assert_allclose(xh[:, 0], xh[:, -1], rtol=0, atol=0)
    # L = sum c * x  ->  dL/dx = c
    c = rng.standard_normal((n, S))
    g = torch.from_numpy(c.reshape(-1)).cuda()
    lam, ita, resa = P.adjoint(g, conv=1e-10)
    lo, itao, _ = O.adjoint(rp, col, w, seeds, c, conv=1e-10)
    np.testing.assert_array_equal(ita, itao)
    lh = host(lam, n, S)
    np.testing.assert_allclose(lh, lo, rtol=1e-11, atol=1e-11 * np.abs(lo).max())
    gr = P.grad(x, lam)
    gro = O.grad_weights(rp, col, w, xh, lh)
    np.testing.assert_allclose(gr, gro, rtol=1e-9, atol=1e-9 * np.abs(gro).max())
    P.close()


def test_multi_chunk_rows_present(cuda, oracle):
    rp, col, w = rmat_weighted(oracle, 10)
    P = Ppr(rp, col, w, 8)
    ch_ccs, mu_ccs, ch_crs, mu_crs = P.info()
    P.close()
    n = len(rp) - 1
    assert ch_crs >= n and ch_ccs >= n
    assert mu_crs > 0 and mu_ccs > 0          # hubs of more than 32 edges both ways
    assert np.diff(rp).max() > 64


def loss_of(P, seeds, target, n, S):
    x, _, _ = P.solve(seeds, conv=0.0, max_iter=400)
    xh = host(x, n, S)
    return 0.5 * ((xh - target) ** 2).sum(), x, xh


def test_gradient_matches_central_differences(cuda, oracle):
    """L = 0.5 ||x - x*||^2 over 16 seeds; 64 random edges; h = 1e-6."""
    import torch
    rp, col, w = rmat_weighted(oracle, 8, seed=11)
    w = 0.5 + w                              # keep w +- h positive
    n, S = len(rp) - 1, 16
    rng = np.random.default_rng(2)
    seeds = rng.integers(0, n, S)
    target = rng.standard_normal((n, S)) * 0.01
    P = Ppr(rp, col, w, S)
    L0, x, xh = loss_of(P, seeds, target, n, S)
    g = torch.from_numpy((xh - target).reshape(-1)).cuda()
    lam, _, _ = P.adjoint(g, conv=0.0, max_iter=400)
    grad = P.grad(x, lam)
    picks = rng.choice(len(col), 64, replace=False)
    h = 1e-6
    fd = []
    for k in picks:
        wp = w.copy()
        wp[k] += h
        P.set_weights(wp)
        Lp, _, _ = loss_of(P, seeds, target, n, S)
        wp[k] -= 2 * h
        P.set_weights(wp)
        Lm, _, _ = loss_of(P, seeds, target, n, S)
        fd.append((Lp - Lm) / (2 * h))
    P.close()
    fd = np.array(fd)
    np.testing.assert_allclose(grad[picks], fd, rtol=1e-5, atol=1e-6 * np.abs(grad).max())


def test_mean_over_all_seeds_is_reference_pagerank(cuda, reference):
    """Unit weights, no dangling rows: the mean of the personalised vectors over
    all n seeds is simple_pagerank's vector, here from the compiled reference."""
    from oracle.oracle import Restatement, VOID, crs_to_coo
    R = Restatement()
    rp, col, _ = R.rmat(7, seed=5, vtype=VOID)
    n = len(rp) - 1
    # add the missing self loops so no row is dangling
    rows, cols = crs_to_coo(rp, col)
    have = set(zip(rows.tolist(), cols.tolist()))
    extra = [(i, i) for i in range(n) if (i, i) not in have]
    I = np.concatenate([rows, np.array([e[0] for e in extra], np.uint32)])
    J = np.concatenate([cols, np.array([e[1] for e in extra], np.uint32)])
    order = np.lexsort((J, I))
    I, J = I[order], J[order]
    rp2 = np.concatenate([[0], np.cumsum(np.bincount(I, minlength=n))]).astype(np.int64)
    V = np.ones(len(J))
    assert np.diff(rp2).min() >= 1
    P = Ppr(rp2, J, V, n)
    x, it, _ = P.solve(np.arange(n), conv=0.0, max_iter=300)
    P.close()
    assert (it == 300).all()
    mean = host(x, n, n).mean(1)
    # conv = 0: both run all 300 iterations (the reference then reports FAILED)
    rc, pr, itr, _ = reference.pagerank(n, I, J, V, alpha=0.85, conv=0.0, max_iter=300)
    assert rc in (0, 8) and itr == 300
    np.testing.assert_allclose(mean, pr, rtol=1e-12, atol=1e-15)
    assert abs(mean.sum() - 1) < 1e-12


def test_empty_graph_all_dangling(cuda):
    """No edges: every row dangles and x_s = e_seed exactly in one step."""
    n, S = 50, 3
    P = Ppr(np.zeros(n + 1, np.int64), np.zeros(0, np.uint32), np.zeros(0), S)
    x, it, res = P.solve([3, 7, 3], conv=1e-12)
    xh = host(x, n, S)
    P.close()
    e = np.zeros((n, S))
    e[3, 0] = e[7, 1] = e[3, 2] = 1.0
    np.testing.assert_allclose(xh, e, rtol=0, atol=1e-15)
    rp, col, w = np.zeros(n + 1, np.int64), np.zeros(0, np.int64), np.zeros(0)
    xo, ito, _ = O.forward(rp, col, w, [3, 7, 3], conv=1e-12)
    np.testing.assert_array_equal(it, ito)


def test_not_converged_returns_failed(cuda, oracle):
    rp, col, w = rmat_weighted(oracle, 8)
    P = Ppr(rp, col, w, 4)
    x, it, res = P.solve([0, 1, 2, 3], conv=1e-12, max_iter=5, expect_rc=8)
    P.close()
    assert (it == 5).all() and (res > 1e-12).all()
    xo, ito, _ = O.forward(rp, col, w, [0, 1, 2, 3], conv=1e-12, max_iter=5)
    np.testing.assert_allclose(host(x, len(rp) - 1, 4), xo, rtol=1e-12, atol=1e-15)


def test_initial_guess_given(cuda, oracle):
    rp, col, w = rmat_weighted(oracle, 8)
    n, S = len(rp) - 1, 8
    seeds = np.arange(S) * 5
    x0 = np.random.default_rng(1).random((n, S))
    P = Ppr(rp, col, w, S)
    x, it, _ = P.solve(seeds, conv=1e-9, x0=x0)
    P.close()
    xo, ito, _ = O.forward(rp, col, w, seeds, conv=1e-9, x0=x0)
    np.testing.assert_array_equal(it, ito)
    np.testing.assert_allclose(host(x, n, S), xo, rtol=1e-11, atol=1e-13)


def test_errors(cuda, oracle):
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    rp, col, w = rmat_weighted(oracle, 6)
    P = Ppr(rp, col, w, 2)
    lam = torch.zeros(P.n * 2, dtype=torch.float64, device="cuda")
    it = (C.c_int64 * 2)()
    res = (C.c_double * 2)()
    # adjoint before any solve
    assert abi.lib().alpb_ppr_adjoint(P.h, dev.ptr(lam), dev.ptr(torch.zeros_like(lam)), 1e-9, 10,
                                      it, res, dev.stream_ptr()) == 7
    P.solve([1, 2], expect_rc=0)
    # seed out of range
    sd = np.array([0, P.n], np.int64)
    x = torch.zeros_like(lam)
    assert abi.lib().alpb_ppr_solve(P.h, sd.ctypes.data_as(C.c_void_p), 0.85, 1e-9, 10,
                                    dev.ptr(x), 0, it, res, dev.stream_ptr()) == 3
    # dl_dx and lambda the same buffer
    assert abi.lib().alpb_ppr_adjoint(P.h, dev.ptr(lam), dev.ptr(lam), 1e-9, 10, it, res,
                                      dev.stream_ptr()) == 4
    # negative weight: rejected, and the handle keeps the previous weights
    wn = w.copy()
    wn[3] = -1.0
    wt = torch.from_numpy(wn).cuda()
    assert abi.lib().alpb_ppr_set_weights(P.h, dev.ptr(wt), dev.stream_ptr()) == 7
    x2, it2, _ = P.solve([1, 2], expect_rc=0)
    xo, ito, _ = O.forward(rp, col, w, [1, 2], conv=1e-9)
    np.testing.assert_array_equal(it2, ito)
    np.testing.assert_allclose(host(x2, P.n, 2), xo, rtol=1e-11, atol=1e-15)
    P.close()
    h = C.c_void_p()
    assert abi.lib().alpb_ppr_create(C.byref(h), P.n, P.nnz, dev.ptr(P.rp), dev.ptr(P.col),
                                     dev.ptr(P.w), 129, dev.stream_ptr()) == 6


class PprFunction:
    """torch.autograd shim over the C-ABI (tests only): weights -> x."""

    @staticmethod
    def make(P, seeds, conv=1e-12):
        import torch

        class F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, w):
                P.set_weights(w.detach().cpu().numpy())
                x, _, _ = P.solve(seeds, conv=conv)
                ctx.save_for_backward(x)
                return x.view(P.n, P.S).clone()

            @staticmethod
            def backward(ctx, gx):
                (x,) = ctx.saved_tensors
                lam, _, _ = P.adjoint(gx.contiguous().view(-1), conv=conv)
                return torch.from_numpy(P.grad(x, lam)).to(gx.device)

        return F.apply


def test_autograd_shim(cuda, oracle):
    import torch
    rp, col, w = rmat_weighted(oracle, 8, seed=3)
    n, S = len(rp) - 1, 8
    seeds = np.arange(S) * 7
    P = Ppr(rp, col, w, S)
    f = PprFunction.make(P, seeds)
    wt = torch.tensor(w, dtype=torch.float64, device="cuda", requires_grad=True)
    x = f(wt)
    loss = (x[:, 0] ** 2).sum() + x[:, 1:].sum()
    loss.backward()
    xo, _, _ = O.forward(rp, col, w, seeds, conv=1e-12)
    go = np.zeros((n, S))
    go[:, 0] = 2 * xo[:, 0]
    go[:, 1:] = 1.0
    lo, _, _ = O.adjoint(rp, col, w, seeds, go, conv=1e-12)
    gro = O.grad_weights(rp, col, w, xo, lo)
    P.close()
    np.testing.assert_allclose(wt.grad.cpu().numpy(), gro, rtol=1e-8,
                               atol=1e-8 * np.abs(gro).max())


def test_hub_rows_summed_in_groups(cuda):
    """A hub with ~3000 out-edges and ~3000 in-edges: its rows span more than
    32 x 32 nonzeroes in both storages, so their chunk partials are summed in
    groups before the row sum."""
    import torch
    rng = np.random.default_rng(17)
    n = 3072
    I = [0] * (n - 1) + list(range(1, n)) + rng.integers(0, n, 5 * n).tolist()
    J = list(range(1, n)) + [0] * (n - 1) + rng.integers(0, n, 5 * n).tolist()
    keys = np.unique(np.asarray(I, np.int64) * n + np.asarray(J, np.int64))
    rows, cols = keys // n, keys % n
    rp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int64)
    w = rng.uniform(0.5, 1.5, len(cols))
    assert np.diff(rp).max() > 32 * 32 and np.bincount(cols, minlength=n).max() > 32 * 32
    S = 8
    seeds = np.concatenate([[0], rng.integers(1, n, S - 1)])
    # a fixed number of iterations (tolerance 0): the grouped sums round
    # differently from the restatement's sequential ones, which can move a
    # residual that sits at the tolerance across it
    P = Ppr(rp, cols, w, S)
    x, it, _ = P.solve(seeds, conv=0.0, max_iter=300)
    xo, ito, _ = O.forward(rp, cols, w, seeds, conv=0.0, max_iter=300)
    np.testing.assert_array_equal(it, ito)
    xh = host(x, n, S)
    np.testing.assert_allclose(xh, xo, rtol=1e-11, atol=1e-11 * np.abs(xo).max())
    g = rng.standard_normal((n, S))
    lam, ita, _ = P.adjoint(torch.from_numpy(g.reshape(-1)).cuda(), conv=0.0, max_iter=300)
    lo, itao, _ = O.adjoint(rp, cols, w, seeds, g, conv=0.0, max_iter=300)
    np.testing.assert_array_equal(ita, itao)
    lh = host(lam, n, S)
    np.testing.assert_allclose(lh, lo, rtol=1e-11, atol=1e-11 * np.abs(lo).max())
    gr = P.grad(x, lam)
    gro = O.grad_weights(rp, cols, w, xh, lh)
    P.close()
    np.testing.assert_allclose(gr, gro, rtol=1e-9, atol=1e-9 * np.abs(gro).max())
