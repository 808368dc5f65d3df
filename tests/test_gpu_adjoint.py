"""Adjoint gradients of the CG solve, through a torch.autograd.Function shim
over the C-ABI (test code only), against
  * gradients assembled from the reference algorithm: CG forward, CG on A^T,
    then -lambda_i x_j on the host (the C restatement of
    algorithms::conjugate_gradient), and
  * central finite differences with h = 1e-6: [L(theta+h) - L(theta-h)] / 2h.
    Subtracting two separately solved losses would lose every digit the
    solver leaves (~1e-14 relative, divided by 2h), so the difference is
    formed exactly instead: with x+ = x(theta+h), x- = x(theta-h),
        A(theta+h) (x+ - x-) = (A(theta-h) - A(theta+h)) x-
    whose right-hand side has two nonzeros of size 2h; solving it for
    d = x+ - x- keeps d to ~1e-14 RELATIVE, and
        L(theta+h) - L(theta-h) = 0.5 d . (2 (x- - x*) + d).

Gradients are per stored entry: dL/dA_ij = -lambda_i x_j.  A is symmetric
(a_ij = a_ji keyed by the pair), so a finite difference perturbs the pair
(i, j), (j, i) together -- keeping A SPD for CG -- and is compared with
dL/dA_ij + dL/dA_ji; a diagonal entry is perturbed alone.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
FP64 = 3
TOL = 1e-13       # forward/adjoint relative residual for the FD comparisons


def _dev():
    from alp_b200 import device
    return device


def sym_dd_matrix(sizes, seed=11):
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    A = dev.stencil(sizes, 1.0, 1.0, ref_order=False)
    abi.call("alpb_gen_sym_dd_values", dev.ptr(A.offsets), dev.ptr(A.indices), A.m, seed, 0.5, 1.5,
             1.05, dev.ptr(A.values), dev.stream_ptr())
    torch.cuda.synchronize()
    return A


def cg_solve(A, values, b, tol=TOL, to_floor=False):
    """x = A^{-1} b by the fused CG.  to_floor: iterate to the FP64 floor (the
    finite differences need the loss to ~1e-16 relative: FD noise is about
    solver error * |x|^2 / h); the solve then ends on its iteration budget."""
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    x = torch.zeros_like(b)
    it, res = C.c_int64(), C.c_double()
    rc = abi.lib().alpb_cg_solve(A.m, dev.ptr(A.offsets), dev.ptr(A.indices), dev.ptr(values),
                                 dev.ptr(b), dev.ptr(x), 400 if to_floor else 5000,
                                 1e-18 if to_floor else tol, C.byref(it), C.byref(res), None,
                                 None, dev.stream_ptr())
    assert rc == abi.SUCCESS or (to_floor and rc == abi.FAILED), abi.last_error()
    return x


class CGSolve:
    """x = A(values)^{-1} b as a differentiable function of (values, b)."""

    @staticmethod
    def make(A):
        import torch
        from alp_b200 import _abi as abi
        dev = _dev()

        class Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, values, b):
                x = cg_solve(A, values, b)
                ctx.save_for_backward(values, x)
                return x

            @staticmethod
            def backward(ctx, gx):
                values, x = ctx.saved_tensors
                T = dev.CRS(A.m, A.n, A.nnz, A.offsets, A.indices, values.contiguous(), abi.FP64)
                At = dev.transpose(T)
                lam = torch.empty_like(x)
                gv = torch.empty_like(values)
                it, res = C.c_int64(), C.c_double()
                abi.call("alpb_cg_adjoint", A.m, dev.ptr(A.offsets), dev.ptr(A.indices),
                         dev.ptr(values), dev.ptr(At.offsets), dev.ptr(At.indices),
                         dev.ptr(At.values), dev.ptr(x), dev.ptr(gx.contiguous()), dev.ptr(lam),
                         dev.ptr(gv), 5000, TOL, C.byref(it), C.byref(res), None, None,
                         dev.stream_ptr())
                return gv, lam
        return Fn.apply


def test_adjoint_matches_reference_assembled_gradients(cuda, oracle):
    import torch
    A = sym_dd_matrix((12, 12, 12))
    dev = _dev()
    b = torch.empty(A.m, dtype=torch.float64, device="cuda")
    xs = torch.empty_like(b)
    from alp_b200 import _abi as abi
    abi.call("alpb_gen_normal", dev.ptr(b), A.m, 5, 1, dev.stream_ptr())
    abi.call("alpb_gen_normal", dev.ptr(xs), A.m, 6, 1, dev.stream_ptr())
    values = A.values.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    solve = CGSolve.make(A)
    x = solve(values, bb)
    loss = 0.5 * ((x - xs) ** 2).sum()
    loss.backward()
    # reference algorithm on the host: forward CG, CG on A^T, -lambda_i x_j
    o, i, v = A.to_host()
    hb, hxs = b.cpu().numpy(), xs.cpu().numpy()
    rc, xr, _, _ = oracle.cg(o, i, v, hb, np.zeros(A.m), 5000, TOL)
    assert rc == 0
    cp, row, tv = oracle.transpose(A.m, A.n, o, i, v, FP64)
    rc, lam, _, _ = oracle.cg(cp, row, tv, xr - hxs, np.zeros(A.m), 5000, TOL)
    assert rc == 0
    rows = np.repeat(np.arange(A.m), np.diff(o))
    g_ref = -lam[rows] * xr[i]
    np.testing.assert_allclose(x.detach().cpu().numpy(), xr, rtol=0, atol=1e-12)
    np.testing.assert_allclose(bb.grad.cpu().numpy(), lam, rtol=0, atol=1e-11)
    np.testing.assert_allclose(values.grad.cpu().numpy(), g_ref, rtol=0,
                               atol=1e-11 * np.abs(g_ref).max())


def test_adjoint_matches_central_differences(cuda):
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    A = sym_dd_matrix((10, 10, 10), seed=17)
    b = torch.empty(A.m, dtype=torch.float64, device="cuda")
    xs = torch.empty_like(b)
    abi.call("alpb_gen_normal", dev.ptr(b), A.m, 7, 1, dev.stream_ptr())
    abi.call("alpb_gen_normal", dev.ptr(xs), A.m, 8, 1, dev.stream_ptr())
    values = A.values.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    x = CGSolve.make(A)(values, bb)
    (0.5 * ((x - xs) ** 2).sum()).backward()
    grad = values.grad.cpu().numpy()
    o, i, v = A.to_host()
    rows = np.repeat(np.arange(A.m), np.diff(o))
    # position of the transposed entry (j, i) of every stored (i, j)
    key = rows.astype(np.int64) * A.m + i
    order = np.argsort(key)
    tkey = i.astype(np.int64) * A.m + rows
    partner = order[np.searchsorted(key[order], tkey)]

    h = 1e-6
    rng = np.random.default_rng(0)
    picks = rng.choice(A.nnz, size=64, replace=False)
    base = A.values.clone()
    x_base = cg_solve(A, base, b, to_floor=True)

    def loss_diff(vp, vm, dvals):
        """L(vp) - L(vm) where A(vp) - A(vm) has the entries dvals (stored
        position, value)."""
        xm = cg_solve(A, vm, b, to_floor=True)
        rhs = torch.zeros_like(b)        # (A(vm) - A(vp)) xm
        for pos, dv in dvals:
            rhs[int(rows[pos])] -= dv * xm[int(i[pos])]
        d = cg_solve(A, vp, rhs, to_floor=True)
        return 0.5 * float((d * (2 * (xm - xs) + d)).sum())

    worst = 0.0
    for k in picks:
        p = int(partner[k])
        vp, vm = base.clone(), base.clone()
        vp[int(k)] += h
        vm[int(k)] -= h
        dvals = [(int(k), 2 * h)]
        if p != k:
            vp[p] += h
            vm[p] -= h
            dvals.append((p, 2 * h))
        fd = loss_diff(vp, vm, dvals) / (2 * h)
        an = grad[k] + (grad[p] if p != k else 0.0)
        err = abs(fd - an) / max(abs(an), 1e-3 * np.abs(grad).max())
        worst = max(worst, err)
    assert worst < 1e-5, worst
    # dL/db on a few entries: x(b + h e_j) - x(b - h e_j) = A^{-1} (2h e_j)
    gb = bb.grad.cpu().numpy()
    for j in rng.choice(A.m, size=8, replace=False):
        e = torch.zeros_like(b)
        e[int(j)] = 2 * h
        d = cg_solve(A, base, e, to_floor=True)
        xm = x_base - 0.5 * d
        fd = 0.5 * float((d * (2 * (xm - xs) + d)).sum()) / (2 * h)
        assert abs(fd - gb[j]) <= 1e-5 * max(abs(gb[j]), 1e-3 * np.abs(gb).max()), (j, fd, gb[j])


def test_cg_grad_entry_point(cuda):
    """alpb_cg_grad (forward + adjoint + SDDMM in one call) equals the shim."""
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    A = sym_dd_matrix((8, 9, 10), seed=23)
    At = dev.transpose(A)
    b = torch.empty(A.m, dtype=torch.float64, device="cuda")
    xs = torch.empty_like(b)
    abi.call("alpb_gen_normal", dev.ptr(b), A.m, 9, 1, dev.stream_ptr())
    abi.call("alpb_gen_normal", dev.ptr(xs), A.m, 10, 1, dev.stream_ptr())
    x = torch.empty_like(b)
    lam = torch.empty_like(b)
    gv = torch.empty_like(A.values)
    work = torch.empty(A.m + 1, dtype=torch.float64, device="cuda")
    L, itf, ita = C.c_double(), C.c_int64(), C.c_int64()
    abi.call("alpb_cg_grad", A.m, dev.ptr(A.offsets), dev.ptr(A.indices), dev.ptr(A.values),
             dev.ptr(At.offsets), dev.ptr(At.indices), dev.ptr(At.values), dev.ptr(b), dev.ptr(xs),
             dev.ptr(x), dev.ptr(lam), dev.ptr(gv), dev.ptr(work), 5000, TOL, C.byref(L),
             C.byref(itf), C.byref(ita), None, None, dev.stream_ptr())
    values = A.values.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    x2 = CGSolve.make(A)(values, bb)
    loss = 0.5 * ((x2 - xs) ** 2).sum()
    loss.backward()
    assert abs(L.value - float(loss)) <= 1e-12 * float(loss)
    torch.testing.assert_close(x, x2.detach(), rtol=0, atol=1e-12)
    torch.testing.assert_close(lam, bb.grad, rtol=0, atol=1e-12)
    torch.testing.assert_close(gv, values.grad, rtol=0, atol=1e-12)
    assert itf.value > 0 and ita.value > 0
