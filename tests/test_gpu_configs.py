"""Parity at the benchmark's configurations: every workload bench.py times is
checked here at the size it is timed at (or, where the CPU checker cannot
finish in minutes, at the largest size it can, plus size-independent checks
at the full size).

* simple_pagerank on the R-MAT scale-22 pattern with unit weights (alpha 0.85,
  conv 1e-9) against the C restatement of algorithms::simple_pagerank;
* the differentiated CG on the 27-point 64^3 pattern with the benchmark's
  values (off-diagonals -U(0.5, 1.5), symmetric; diagonal 1.05 |row sum|):
  x, lambda and dL/dA against the restatement's CG forward, CG on A^T and
  -lambda_i x_j, and against central differences with h = 1e-6 on 64 entries;
* batched CG on the 256 shifted Poisson systems (sides log-uniform in
  [32, 512]), every instance against the restatement's CG;
* HPCG with 8 right-hand sides at 64^3 with 3 coarser levels against
  grb::algorithms::hpcg run unchanged on the reference backend (the largest
  grid it finishes in seconds per right-hand side), and at the benchmark's
  256^3 the true residual ||b - A x|| of every right-hand side, from an
  independent product;
* personalised PageRank with 64 seeds at R-MAT scale 20 against the C form of
  the numpy restatement (forward, adjoint, gradient), and at the benchmark's
  scale 24 the mass of every seed's vector and central differences on the 16
  edges of largest gradient.

Bars: the same iteration counts (batched CG: within one), FP64 results within
the relative tolerances stated at each check.
"""
import concurrent.futures as cf
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
FP64 = 3


def _dev():
    from alp_b200 import device
    return device


# ----------------------------------------------------------- PageRank s22 --
def test_pagerank_rmat22_config(cuda, oracle):
    """R-MAT scale 22, edge factor 16, seed 42, unit weights: the benchmark's
    PageRank.  Iterations equal, scores within 1e-10 relative."""
    import torch
    from test_gpu_solvers import pagerank_device
    dev = _dev()
    A = dev.rmat(22, vtype=FP64, seed=42)
    L = dev.CRS(A.m, A.n, A.nnz, A.offsets, A.indices,
                torch.ones(A.nnz, dtype=torch.float64, device="cuda"), FP64)
    del A
    LT = dev.transpose(L)
    rc, pr, it, res = pagerank_device(L, LT)
    assert rc == 0
    o, i, v = L.to_host()
    to, ti, tv = LT.to_host()
    del L, LT
    torch.cuda.empty_cache()
    rc2, pr2, it2, res2 = oracle.pagerank(o, i, v, to, ti, tv)
    assert rc2 == 0
    assert it == it2, (it, it2)
    np.testing.assert_allclose(pr, pr2, rtol=1e-10, atol=1e-10 * np.abs(pr2).max())
    # the L1 residual sums 4 M differences of iterates that agree to ~1e-13
    # relative (sums in another order), each ~1e-16 of the scores at
    # convergence: it carries only a few digits, so it is compared loosely
    assert res <= 1e-9 and res2 <= 1e-9
    assert abs(res - res2) <= 1e-2 * res2
    assert abs(pr.sum() - 1.0) < 1e-8


# ------------------------------------------------------- adjoint CG 64^3 --
def test_adjoint_cg_64_config(cuda, oracle):
    """The differentiated-CG workload exactly as benchmarked (27-point 64^3,
    value seed 11, b seed 5, x* seed 6, tolerance 1e-12): x, lambda = dL/db
    and dL/dA within 1e-10 relative of the restatement, then central
    differences on 64 stored entries (symmetric pairs perturbed together)."""
    import torch
    from alp_b200 import _abi as abi
    from test_gpu_adjoint import cg_solve
    dev = _dev()
    sp = dev.stream_ptr()
    A = dev.stencil((64, 64, 64), 1.0, 1.0, ref_order=False)
    abi.call("alpb_gen_sym_dd_values", dev.ptr(A.offsets), dev.ptr(A.indices), A.m, 11, 0.5, 1.5,
             1.05, dev.ptr(A.values), sp)
    At = dev.transpose(A)
    b = torch.empty(A.m, dtype=torch.float64, device="cuda")
    xs = torch.empty_like(b)
    abi.call("alpb_gen_normal", dev.ptr(b), A.m, 5, 1, sp)
    abi.call("alpb_gen_normal", dev.ptr(xs), A.m, 6, 1, sp)
    tol = 1e-12
    x = torch.zeros_like(b)
    itf, res = C.c_int64(), C.c_double()
    abi.call("alpb_cg_solve", A.m, dev.ptr(A.offsets), dev.ptr(A.indices), dev.ptr(A.values),
             dev.ptr(b), dev.ptr(x), 5000, tol, C.byref(itf), C.byref(res), None, None, sp)
    g = x - xs
    lam = torch.zeros_like(b)
    gv = torch.empty_like(A.values)
    ita = C.c_int64()
    abi.call("alpb_cg_adjoint", A.m, dev.ptr(A.offsets), dev.ptr(A.indices), dev.ptr(A.values),
             dev.ptr(At.offsets), dev.ptr(At.indices), dev.ptr(At.values), dev.ptr(x), dev.ptr(g),
             dev.ptr(lam), dev.ptr(gv), 5000, tol, C.byref(ita), C.byref(res), None, None, sp)
    torch.cuda.synchronize()
    o, i, v = A.to_host()
    hb, hxs = b.cpu().numpy(), xs.cpu().numpy()
    rc, xr, itr, _ = oracle.cg(o, i, v, hb, np.zeros(A.m), 5000, tol)
    assert rc == 0 and abs(itr - itf.value) <= 1, (itr, itf.value)
    cp, row, tv = oracle.transpose(A.m, A.n, o, i, v, FP64)
    rc, lr, itl, _ = oracle.cg(cp, row, tv, xr - hxs, np.zeros(A.m), 5000, tol)
    assert rc == 0 and abs(itl - ita.value) <= 1, (itl, ita.value)
    rows = np.repeat(np.arange(A.m), np.diff(o))
    g_ref = -lr[rows] * xr[i]
    hx, hl, hg = x.cpu().numpy(), lam.cpu().numpy(), gv.cpu().numpy()
    np.testing.assert_allclose(hx, xr, rtol=0, atol=1e-10 * np.abs(xr).max())
    np.testing.assert_allclose(hl, lr, rtol=0, atol=1e-10 * np.abs(lr).max())
    np.testing.assert_allclose(hg, g_ref, rtol=0, atol=1e-10 * np.abs(g_ref).max())

    # central differences, formed exactly as in test_gpu_adjoint: with
    # x- = x(theta - h) and d = x+ - x- solved from A(theta+h) d = (A(theta-h)
    # - A(theta+h)) x-, L+ - L- = 0.5 d . (2 (x- - x*) + d)
    key = rows.astype(np.int64) * A.m + i
    order = np.argsort(key)
    partner = order[np.searchsorted(key[order], i.astype(np.int64) * A.m + rows)]
    h = 1e-6
    rng = np.random.default_rng(64)
    base = A.values.clone()
    worst = 0.0
    for k in rng.choice(A.nnz, size=64, replace=False):
        k = int(k)
        p = int(partner[k])
        vp, vm = base.clone(), base.clone()
        vp[k] += h
        vm[k] -= h
        dvals = [(k, 2 * h)]
        if p != k:
            vp[p] += h
            vm[p] -= h
            dvals.append((p, 2 * h))
        xm = cg_solve(A, vm, b, to_floor=True)
        rhs = torch.zeros_like(b)
        for pos, dv in dvals:
            rhs[int(rows[pos])] -= dv * xm[int(i[pos])]
        d = cg_solve(A, vp, rhs, to_floor=True)
        fd = 0.5 * float((d * (2 * (xm - xs) + d)).sum()) / (2 * h)
        an = hg[k] + (hg[p] if p != k else 0.0)
        worst = max(worst, abs(fd - an) / max(abs(an), 1e-3 * np.abs(hg).max()))
    assert worst < 1e-5, worst


# ---------------------------------------------------- batched CG, 256 sys --
def test_batched_cg_256_config(cuda, oracle):
    """The benchmark's 256 shifted 2-D Poisson systems (rng seed 2024: sides
    log-uniform in [32, 512], shifts U(0.01, 1); b ~ N(0, 1) from the device
    generator, seed 2024), relative tolerance 1e-8, solved in one
    graph-captured launch: every instance against the restatement's CG
    (iterations within one, x within 1e-9 relative)."""
    from test_gpu_batched import batched_solve, make_batch
    nseg = 256
    rng = np.random.default_rng(2024)
    sides = np.round(np.exp(rng.uniform(np.log(32), np.log(512), nseg))).astype(np.int64)
    shifts = rng.uniform(0.01, 1.0, nseg)
    A, b, tR, seg = make_batch(sides, shifts, seed=2024)
    rc, x, it, res, conv = batched_solve(A, b, tR, nseg, 20000, 1e-8, capture=True)
    assert rc == 0 and conv.all()
    o, i, v = A.to_host()
    hb, hx = b.cpu().numpy(), x.cpu().numpy()

    def one(s):
        r0, r1 = int(seg[s]), int(seg[s + 1])
        srp = o[r0:r1 + 1] - o[r0]
        scol = (i[o[r0]:o[r1]].astype(np.int64) - r0).astype(np.uint32)
        rc2, x2, it2, _ = oracle.cg(srp, scol, v[o[r0]:o[r1]], hb[r0:r1], np.zeros(r1 - r0),
                                    20000, 1e-8)
        return s, rc2, x2, it2

    with cf.ThreadPoolExecutor(max_workers=16) as ex:   # the C solver releases the GIL
        for s, rc2, x2, it2 in ex.map(one, range(nseg)):
            r0, r1 = int(seg[s]), int(seg[s + 1])
            assert rc2 == 0
            assert abs(int(it[s]) - it2) <= 1, (s, it[s], it2)
            np.testing.assert_allclose(hx[r0:r1], x2, rtol=0,
                                       atol=1e-9 * max(1.0, np.abs(x2).max()), err_msg=str(s))


# ------------------------------------------------------------------ HPCG --
def test_hpcg_64_eight_rhs_matches_reference(cuda):
    """64^3 with three coarser levels (32^3, 16^3, 8^3), 27 colours, 8
    right-hand sides ~ N(0, 1) solved together, tolerance 1e-9: each against
    its own run of grb::algorithms::hpcg on the reference backend (the 8
    reference runs go in parallel)."""
    import torch
    from test_gpu_hpcg import Hpcg, reference
    h = Hpcg(64, 3, 27, 8)
    assert h.levels == 4
    rng = np.random.default_rng(6464)
    b = rng.standard_normal((h.n, 8))
    it, res, x = h.solve(torch.from_numpy(b.reshape(-1)).cuda(), 200, 1e-9)
    h.close()
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        refs = list(ex.map(lambda k: reference(64, 3, 27, 1, 1, 200, 1e-9, True, b[:, k]),
                           range(8)))
    for k, (ir, rr, xr) in enumerate(refs):
        assert it[k] == ir, (k, it[k], ir)
        np.testing.assert_allclose(x[:, k], xr, rtol=1e-9, atol=1e-9 * np.abs(xr).max())
        assert abs(res[k] - rr) <= 1e-6 * rr + 1e-300, (k, res[k], rr)


def test_hpcg_256_true_residuals(cuda):
    """The benchmark's HPCG (256^3, 3 coarser levels, 27 colours, 8 right-hand
    sides from the device generator, seed 31, tolerance 1e-9): for every
    right-hand side, ||b - A x|| / ||b|| from an independent alpb_mxv on the
    finest matrix is within the tolerance (the solver stops on its recurrence
    residual, which may drift from the true one by rounding)."""
    import torch
    from alp_b200 import _abi as abi
    from test_gpu_hpcg import Hpcg
    dev = _dev()
    sp = dev.stream_ptr()
    nrhs = 8
    h = Hpcg(256, 3, 27, nrhs)
    b = torch.empty(h.n * nrhs, dtype=torch.float64, device="cuda")
    abi.call("alpb_gen_normal", dev.ptr(b), h.n * nrhs, 31, 1, sp)
    x = torch.zeros_like(b)
    it = (C.c_int64 * nrhs)()
    res = (C.c_double * nrhs)()
    abi.call("alpb_hpcg_solve", h.h, dev.ptr(b), dev.ptr(x), 1, 1, 1, 500, 1e-9, it, res, sp)
    o, ix, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
    n, nnz = C.c_int64(), C.c_int64()
    abi.call("alpb_hpcg_matrix", h.h, 0, C.byref(o), C.byref(ix), C.byref(v), C.byref(n),
             C.byref(nnz))
    assert n.value == 256 ** 3
    B = b.view(h.n, nrhs)
    X = x.view(h.n, nrhs)
    for k in range(nrhs):
        xk = X[:, k].contiguous()
        ax = torch.zeros(h.n, dtype=torch.float64, device="cuda")
        abi.call("alpb_mxv", 0, 0, 2, h.n, h.n, nnz.value, o, ix, v, FP64,
                 dev.ptr(ax), None, None, None, None, 1, -1,
                 dev.ptr(xk), None, h.n, None, None, 1, -1, None, sp)
        bk = B[:, k]
        rel = float((bk - ax).norm() / bk.norm())
        assert it[k] < 500 and rel <= 1.5e-9, (k, it[k], rel)
    h.close()


# ------------------------------------------------- personalised PageRank --
def _ppr_handle(A, S):
    from alp_b200 import _abi as abi
    dev = _dev()
    hnd = C.c_void_p()
    abi.call("alpb_ppr_create", C.byref(hnd), A.n, A.nnz, dev.ptr(A.offsets), dev.ptr(A.indices),
             dev.ptr(A.values), S, dev.stream_ptr())
    return hnd


def _ppr_solve(hnd, seeds, S, x, conv, max_iter=1000, warm=False):
    from alp_b200 import _abi as abi
    dev = _dev()
    sd = np.ascontiguousarray(seeds, np.int64)
    it = (C.c_int64 * S)()
    res = (C.c_double * S)()
    abi.call("alpb_ppr_solve", hnd, sd.ctypes.data_as(C.c_void_p), 0.85, conv, max_iter,
             dev.ptr(x), int(warm), it, res, dev.stream_ptr())
    return np.array(it), np.array(res)


def _ppr_adjoint(hnd, S, g, lam, conv):
    from alp_b200 import _abi as abi
    dev = _dev()
    it = (C.c_int64 * S)()
    res = (C.c_double * S)()
    abi.call("alpb_ppr_adjoint", hnd, dev.ptr(g), dev.ptr(lam), conv, 1000, it, res,
             dev.stream_ptr())
    return np.array(it), np.array(res)


def test_ppr_rmat20_64_seeds_matches_restatement(cuda, oracle):
    """R-MAT scale 20 (edge factor 16, seed 42, U(0, 1) weights), 64 seeds
    (one repeated), conv 1e-9: the forward with the restatement's per-seed
    iteration counts, forward and adjoint iterates within 1e-11 relative (the
    adjoint's counts within three, see below); the gradient within 1e-9
    relative."""
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    S = 64
    A = dev.rmat(20, vtype=FP64, seed=42)
    n = A.n
    rng = np.random.default_rng(20)
    seeds = rng.integers(0, n, S)
    seeds[-1] = seeds[0]
    hnd = _ppr_handle(A, S)
    x = torch.empty(n * S, dtype=torch.float64, device="cuda")
    it, res = _ppr_solve(hnd, seeds, S, x, 1e-9)
    c = rng.standard_normal((n, S))
    g = torch.from_numpy(c.reshape(-1)).cuda()
    lam = torch.empty_like(x)
    ita, _ = _ppr_adjoint(hnd, S, g, lam, 1e-9)
    grad = torch.empty(A.nnz, dtype=torch.float64, device="cuda")
    abi.call("alpb_ppr_grad_weights", hnd, dev.ptr(x), dev.ptr(lam), dev.ptr(grad),
             dev.stream_ptr())
    torch.cuda.synchronize()
    abi.lib().alpb_ppr_destroy(hnd)
    o, i, w = A.to_host()
    xh, lh, gh = x.view(n, S).cpu().numpy(), lam.view(n, S).cpu().numpy(), grad.cpu().numpy()
    del x, lam, g, grad
    xo, ito, _ = oracle.ppr_forward(o, i, w, seeds, conv=1e-9)
    np.testing.assert_array_equal(it, ito)
    np.testing.assert_allclose(xh, xo, rtol=1e-11, atol=1e-11 * np.abs(xo).max())
    lo, itao, _ = oracle.ppr_adjoint(o, i, w, seeds, c, conv=1e-9)
    # the adjoint's L1 change sums 1 M entries of size ~1 (dL/dx ~ N(0, 1)):
    # conv = 1e-9 is near the FP64 floor of that sum, where the last
    # iterations change lambda by rounding noise alone, so the stopping
    # iteration may differ by a few; lambda itself agrees to 1e-11
    assert np.abs(ita - itao).max() <= 3, (ita, itao)
    np.testing.assert_allclose(lh, lo, rtol=1e-11, atol=1e-11 * np.abs(lo).max())
    go = oracle.ppr_grad(o, i, w, xo, lo)
    np.testing.assert_allclose(gh, go, rtol=1e-9, atol=1e-9 * np.abs(go).max())


def test_ppr_rmat24_64_seeds_mass_and_central_differences(cuda):
    """The benchmark's graph (R-MAT scale 24, seed 42, U(0, 1) weights) and
    seeds (64, rng seed 24).  At conv 1e-9 every seed's vector sums to one.
    Then, solved to 1e-12 with L = g . x (g ~ N(0, 1)), the 16 edges of
    largest |dL/dw| (weights above 1e-3) are perturbed by h = 1e-6 each way,
    re-solved from the converged x, and the central differences match the
    adjoint gradient within 1e-4 relative."""
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    sp = dev.stream_ptr()
    S = 64
    A = dev.rmat(24, vtype=FP64, seed=42)
    n = A.n
    seeds = np.random.default_rng(24).integers(0, n, S)
    hnd = _ppr_handle(A, S)
    x = torch.empty(n * S, dtype=torch.float64, device="cuda")
    it, _ = _ppr_solve(hnd, seeds, S, x, 1e-9)
    mass = x.view(n, S).sum(0)
    assert float((mass - 1).abs().max()) < 1e-9, mass
    assert (it < 1000).all()
    it, _ = _ppr_solve(hnd, seeds, S, x, 1e-12, warm=True)
    assert (it < 1000).all()
    g = torch.empty_like(x)
    abi.call("alpb_gen_normal", dev.ptr(g), n * S, 41, 1, sp)
    lam = torch.empty_like(x)
    ita, _ = _ppr_adjoint(hnd, S, g, lam, 1e-12)
    assert (ita < 1000).all()
    grad = torch.empty(A.nnz, dtype=torch.float64, device="cuda")
    abi.call("alpb_ppr_grad_weights", hnd, dev.ptr(x), dev.ptr(lam), dev.ptr(grad), sp)
    del lam
    score = torch.where(A.values > 1e-3, grad.abs(), torch.zeros_like(grad))
    picks = torch.topk(score, 16).indices.tolist()
    gh = grad.cpu().numpy()
    h = 1e-6
    xp = torch.empty_like(x)
    w = A.values.clone()              # held by the handle while it solves
    worst = 0.0
    for k in picks:
        Ls = []
        for sign in (1.0, -1.0):
            w[k] = A.values[k] + sign * h
            abi.call("alpb_ppr_set_weights", hnd, dev.ptr(w), sp)
            xp.copy_(x)
            itp, _ = _ppr_solve(hnd, seeds, S, xp, 1e-12, warm=True)
            assert (itp < 1000).all()
            Ls.append(float(torch.dot(g, xp)))
        w[k] = A.values[k]
        fd = (Ls[0] - Ls[1]) / (2 * h)
        worst = max(worst, abs(fd - gh[k]) / abs(gh[k]))
    abi.call("alpb_ppr_set_weights", hnd, dev.ptr(A.values), sp)
    torch.cuda.synchronize()
    abi.lib().alpb_ppr_destroy(hnd)
    assert worst < 1e-4, worst
