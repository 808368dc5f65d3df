"""GPU parity of the fused solvers (CG, PageRank) against the reference's
golden outputs and the C restatement.  Bars: the same iteration count as the
reference, the same converged residual within rounding, and solutions within
the stated tolerances."""
import ctypes as C

import numpy as np
import pytest

import golden_cases as G

pytestmark = pytest.mark.gpu
FP64 = 3


def _dev():
    from alp_b200 import device
    return device


def cg_device(A, b, x0, max_iter, tol, plan=None):
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    x = x0.clone()
    it = C.c_int64()
    res = C.c_double()
    rc = abi.lib().alpb_cg_solve(A.m, dev.ptr(A.offsets), dev.ptr(A.indices), dev.ptr(A.values),
                                 dev.ptr(b), dev.ptr(x), max_iter, tol, C.byref(it), C.byref(res),
                                 None, plan.h if plan else None, dev.stream_ptr())
    torch.cuda.synchronize()
    return rc, x, it.value, res.value


def test_cg_golden_27pt_16(cuda, oracle):
    import torch
    dev = _dev()
    g = G.load("cg_27pt_16.npz")["cg"]
    m = 16 ** 3
    rp, col, vals = oracle.coo_to_crs(m, g["I"], g["J"], g["V"], FP64)
    A = dev.from_host(m, m, rp, col, vals, FP64)
    b = torch.from_numpy(g["b"]).cuda()
    rc, x, it, res = cg_device(A, b, torch.zeros_like(b), 500, 1e-10)
    assert rc == 0
    assert it == int(g["iterations"])
    assert abs(res - float(g["residual"])) <= 1e-3 * float(g["residual"])
    np.testing.assert_allclose(x.cpu().numpy(), g["x"], rtol=0, atol=1e-12)


def test_cg_27pt_32_plain_config(cuda, oracle):
    """The plain-CG workload: 27-point 32^3, diag 26 / off -1, b = A 1,
    x0 = 0, tol 1e-10, max 500 (54 iterations on the reference)."""
    import torch
    dev = _dev()
    A = dev.stencil((32, 32, 32), 26.0, -1.0)
    ones = torch.ones(A.n, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(ones)
    dev.mxv(0, A, b, ones)
    rc, x, it, res = cg_device(A, b, torch.zeros_like(b), 500, 1e-10)
    assert rc == 0
    o, i, v = A.to_host()
    rc2, x2, it2, res2 = oracle.cg(o, i, v, b.cpu().numpy(), np.zeros(A.n), 500, 1e-10)
    assert it == it2 == 54
    assert abs(res - res2) <= 1e-3 * res2
    np.testing.assert_allclose(x.cpu().numpy(), np.ones(A.n), rtol=0, atol=1e-9)
    np.testing.assert_allclose(x.cpu().numpy(), x2, rtol=0, atol=1e-12)


def test_cg_not_converged_returns_failed(cuda):
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    A = dev.stencil((16, 16, 16), 26.0, -1.0)
    b = torch.ones(A.n, dtype=torch.float64, device="cuda")
    rc, x, it, res = cg_device(A, b, torch.zeros_like(b), 3, 1e-14)
    assert rc == abi.FAILED and it == 3


def test_cg_illegal_arguments(cuda):
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    A = dev.stencil((8, 8, 8))
    b = torch.ones(A.n, dtype=torch.float64, device="cuda")
    assert cg_device(A, b, torch.zeros_like(b), 0, 1e-8)[0] == abi.ILLEGAL
    assert cg_device(A, b, torch.zeros_like(b), 10, 0.0)[0] == abi.ILLEGAL


def pagerank_device(L, LT, alpha=0.85, conv=1e-9, max_iter=1000):
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    pr = torch.zeros(L.m, dtype=torch.float64, device="cuda")
    it = C.c_int64()
    res = C.c_double()
    rc = abi.lib().alpb_pagerank(L.m, dev.ptr(L.offsets), dev.ptr(L.indices), dev.ptr(L.values),
                                 dev.ptr(LT.offsets), dev.ptr(LT.indices), dev.ptr(LT.values),
                                 dev.ptr(pr), 0, alpha, conv, max_iter, C.byref(it), C.byref(res),
                                 dev.stream_ptr())
    torch.cuda.synchronize()
    return rc, pr.cpu().numpy(), it.value, res.value


def test_pagerank_golden_rmat_s10(cuda, oracle):
    dev = _dev()
    g = G.load("pagerank_rmat_s10.npz")["pr"]
    n = int(g["n"])
    rp, col, vals = oracle.coo_to_crs(n, g["I"], g["J"], g["V"], FP64)
    cp, row, tv = oracle.coo_to_crs(n, g["J"], g["I"], g["V"], FP64)
    L = dev.from_host(n, n, rp, col, vals, FP64)
    LT = dev.from_host(n, n, cp, row, tv, FP64)
    rc, pr, it, res = pagerank_device(L, LT)
    assert rc == 0
    assert it == int(g["iterations"])
    np.testing.assert_allclose(pr, g["pr"], rtol=1e-10, atol=1e-15)


@pytest.mark.parametrize("scale", [14, 18])
def test_pagerank_rmat_matches_restatement(cuda, oracle, scale):
    import torch
    dev = _dev()
    L = dev.rmat(scale, vtype=FP64, seed=5)
    L.values.fill_(1.0)
    LT = dev.transpose(L)
    rc, pr, it, res = pagerank_device(L, LT)
    o, i, v = L.to_host()
    to, ti, tv = LT.to_host()
    rc2, pr2, it2, res2 = oracle.pagerank(o, i[:L.nnz], v[:L.nnz], to, ti[:L.nnz], tv[:L.nnz])
    assert rc == rc2 == 0
    assert abs(it - it2) <= 1
    np.testing.assert_allclose(pr, pr2, rtol=1e-9, atol=1e-14)
    assert abs(pr.sum() - 1.0) < 1e-8


@pytest.mark.parametrize("scale", [14, 20])
def test_pagerank_planned_equals_plain(cuda, oracle, scale):
    """alpb_pagerank_planned with a caller-held plan of the CCS and scratch
    gives alpb_pagerank's result bit for bit (same tiles, same grid), on two
    solves in a row with the same plan; a plan of other offsets is refused.
    Scale 14 runs the single cooperative kernel, scale 20 (16 M nonzeroes)
    the per-step launches of large graphs, which are also checked against
    the restatement."""
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    L = dev.rmat(scale, vtype=FP64, seed=8)
    L.values.fill_(1.0)
    LT = dev.transpose(L)
    rc, pr, it, res = pagerank_device(L, LT)
    assert rc == 0
    if scale == 20:
        o, i, v = L.to_host()
        to, ti, tv = LT.to_host()
        rc2, pr2, it2, _ = oracle.pagerank(o, i, v, to, ti, tv)
        assert rc2 == 0 and it == it2
        np.testing.assert_allclose(pr, pr2, rtol=1e-10, atol=1e-10 * np.abs(pr2).max())
    plan = dev.Plan(LT, sched=abi.SCHED_AUTO)
    work = torch.empty(3 * L.m, dtype=torch.float64, device="cuda")
    for use_work in (True, False):
        p2 = torch.zeros(L.m, dtype=torch.float64, device="cuda")
        it2, res2 = C.c_int64(), C.c_double()
        rc2 = abi.lib().alpb_pagerank_planned(
            L.m, dev.ptr(L.offsets), dev.ptr(L.indices), dev.ptr(L.values), dev.ptr(LT.offsets),
            dev.ptr(LT.indices), dev.ptr(LT.values), dev.ptr(p2), 0, 0.85, 1e-9, 1000,
            C.byref(it2), C.byref(res2), dev.ptr(work) if use_work else None, plan.h,
            dev.stream_ptr())
        torch.cuda.synchronize()
        assert rc2 == 0 and it2.value == it and res2.value == res
        np.testing.assert_array_equal(p2.cpu().numpy(), pr)
    other = dev.Plan(L, sched=abi.SCHED_AUTO)
    it2, res2 = C.c_int64(), C.c_double()
    rc3 = abi.lib().alpb_pagerank_planned(
        L.m, dev.ptr(L.offsets), dev.ptr(L.indices), dev.ptr(L.values), dev.ptr(LT.offsets),
        dev.ptr(LT.indices), dev.ptr(LT.values), dev.ptr(work), 0, 0.85, 1e-9, 1000,
        C.byref(it2), C.byref(res2), None, other.h, dev.stream_ptr())
    assert rc3 == abi.MISMATCH
