"""Batched CG (one persistent launch, per-instance convergence masks) against
the single-system solver and the C restatement, instance by instance."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_batch(sides, shifts, seed=7):
    """Block-diagonal batch of 2-D 5-point Poisson systems on the device, with
    right-hand sides ~ N(0, 1)."""
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    sides = np.asarray(sides, np.int64)
    rows = sides * sides
    nnzs = 5 * sides * sides - 4 * sides
    seg_rows = np.concatenate([[0], np.cumsum(rows)]).astype(np.int64)
    seg_nnz = np.concatenate([[0], np.cumsum(nnzs)]).astype(np.int64)
    n, nnz = int(seg_rows[-1]), int(seg_nnz[-1])
    d = torch.device("cuda")
    tL = torch.from_numpy(sides).to(d)
    tS = torch.from_numpy(np.asarray(shifts, np.float64)).to(d)
    tR = torch.from_numpy(seg_rows).to(d)
    tN = torch.from_numpy(seg_nnz).to(d)
    rp = torch.empty(n + 1, dtype=torch.int64, device=d)
    ci = torch.empty(nnz, dtype=torch.int32, device=d)
    va = torch.empty(nnz, dtype=torch.float64, device=d)
    abi.call("alpb_gen_poisson2d_batch", len(sides), dev.ptr(tL), dev.ptr(tS), dev.ptr(tR),
             dev.ptr(tN), n, dev.ptr(rp), dev.ptr(ci), dev.ptr(va), dev.stream_ptr())
    b = torch.empty(n, dtype=torch.float64, device=d)
    abi.call("alpb_gen_normal", dev.ptr(b), n, seed, 1, dev.stream_ptr())
    A = dev.CRS(n, n, nnz, rp, ci, va, abi.FP64)
    return A, b, tR, seg_rows


def batched_solve(A, b, tR, nseg, max_iter, tol, capture=False):
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    h = C.c_void_p()
    abi.call("alpb_batched_cg_create", C.byref(h), A.m, A.nnz, dev.ptr(A.offsets),
             dev.ptr(A.indices), dev.ptr(A.values), nseg, dev.ptr(tR), dev.stream_ptr())
    x = torch.zeros_like(b)
    if capture:
        abi.call("alpb_batched_cg_capture", h, dev.ptr(b), dev.ptr(x), max_iter, tol,
                 dev.stream_ptr())
        abi.call("alpb_batched_cg_replay", h, dev.stream_ptr())
    else:
        abi.call("alpb_batched_cg_solve", h, dev.ptr(b), dev.ptr(x), max_iter, tol,
                 dev.stream_ptr())
    it = np.zeros(nseg, np.int64)
    res = np.zeros(nseg)
    conv = np.zeros(nseg, np.int32)
    rc = abi.lib().alpb_batched_cg_results(h, it.ctypes.data_as(C.c_void_p),
                                           res.ctypes.data_as(C.c_void_p),
                                           conv.ctypes.data_as(C.c_void_p), dev.stream_ptr())
    torch.cuda.synchronize()
    abi.lib().alpb_batched_cg_destroy(h)
    return rc, x, it, res, conv


@pytest.mark.parametrize("capture", [False, True], ids=["launch", "graph"])
def test_batched_cg_matches_per_instance_solves(cuda, oracle, capture):
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    rng = np.random.default_rng(3)
    nseg = 24
    sides = np.round(np.exp(rng.uniform(np.log(8), np.log(96), nseg))).astype(np.int64)
    shifts = rng.uniform(0.01, 1.0, nseg)
    A, b, tR, seg_rows = make_batch(sides, shifts)
    rc, x, it, res, conv = batched_solve(A, b, tR, nseg, 2000, 1e-8, capture=capture)
    assert rc == 0 and conv.all()
    o, i, v = A.to_host()
    hb = b.cpu().numpy()
    hx = x.cpu().numpy()
    for s in range(nseg):
        r0, r1 = int(seg_rows[s]), int(seg_rows[s + 1])
        rp = o[r0:r1 + 1] - o[r0]
        col = (i[o[r0]:o[r1]].astype(np.int64) - r0).astype(np.uint32)
        val = v[o[r0]:o[r1]]
        rc2, x2, it2, res2 = oracle.cg(rp, col, val, hb[r0:r1], np.zeros(r1 - r0), 2000, 1e-8)
        assert rc2 == 0
        assert abs(int(it[s]) - it2) <= 1, (s, it[s], it2)
        np.testing.assert_allclose(hx[r0:r1], x2, rtol=0, atol=1e-9 * max(1.0, np.abs(x2).max()))
        # the single-system fused solver on the same instance
        Ai = dev.from_host(r1 - r0, r1 - r0, rp, col, val, abi.FP64)
        bi = b[r0:r1].contiguous()
        xi = torch.zeros_like(bi)
        it3, res3 = C.c_int64(), C.c_double()
        abi.call("alpb_cg_solve", Ai.m, dev.ptr(Ai.offsets), dev.ptr(Ai.indices),
                 dev.ptr(Ai.values), dev.ptr(bi), dev.ptr(xi), 2000, 1e-8, C.byref(it3),
                 C.byref(res3), None, None, dev.stream_ptr())
        assert it3.value == int(it[s])
        assert abs(res3.value - res[s]) <= 1e-6 * res3.value


def test_batched_cg_budget_masks_instances(cuda):
    """An instance that exhausts the iteration budget stops with its own count
    and the call reports FAILED; the others still converge."""
    from alp_b200 import _abi as abi
    sides = [16, 64, 16]
    shifts = [1.0, 0.001, 1.0]
    A, b, tR, _ = make_batch(sides, shifts)
    rc, x, it, res, conv = batched_solve(A, b, tR, 3, 40, 1e-8)
    assert rc == abi.FAILED
    assert conv[0] == 1 and conv[2] == 1 and conv[1] == 0
    assert it[1] == 40 and it[0] < 40


def host_block_diagonal(blocks):
    """Block-diagonal CRS from a list of dense SPD blocks (numpy)."""
    rp, col, val, seg = [0], [], [], [0]
    base = 0
    for Bk in blocks:
        m = Bk.shape[0]
        for r in range(m):
            nz = np.flatnonzero(Bk[r])
            col.extend((nz + base).tolist())
            val.extend(Bk[r, nz].tolist())
            rp.append(len(col))
        base += m
        seg.append(base)
    return (np.asarray(rp, np.int64), np.asarray(col, np.uint32), np.asarray(val),
            np.asarray(seg, np.int64))


def check_against_restatement(oracle, rp, col, val, seg, hb, hx, it, sample):
    for s in sample:
        r0, r1 = int(seg[s]), int(seg[s + 1])
        srp = rp[r0:r1 + 1] - rp[r0]
        scol = (col[rp[r0]:rp[r1]].astype(np.int64) - r0).astype(np.uint32)
        sval = val[rp[r0]:rp[r1]]
        rc2, x2, it2, _ = oracle.cg(srp, scol, sval, hb[r0:r1], np.zeros(r1 - r0), 2000, 1e-8)
        assert rc2 == 0
        assert abs(int(it[s]) - it2) <= 1, (s, it[s], it2)
        np.testing.assert_allclose(hx[r0:r1], x2, rtol=0, atol=1e-9 * max(1.0, np.abs(x2).max()))


def test_batched_cg_long_rows_merge_tiles(cuda, oracle):
    """Rows of more than 32 nonzeroes: the solver keeps the merge engine's warp
    tiles (rows crossing tiles, ordered waits) instead of the sliced storage."""
    import torch
    from alp_b200 import device as dev
    rng = np.random.default_rng(21)
    blocks = []
    for m in rng.integers(40, 220, 12):
        band = 24
        Bk = np.zeros((m, m))
        for r in range(m):
            for c in range(max(0, r - band), min(m, r + band + 1)):
                if c != r:
                    Bk[r, c] = -rng.uniform(0.1, 1.0) if c > r else 0.0
        Bk = Bk + Bk.T
        np.fill_diagonal(Bk, np.abs(Bk).sum(1) * 1.05 + rng.uniform(0.01, 0.5, m))
        blocks.append(Bk)
    rp, col, val, seg = host_block_diagonal(blocks)
    assert np.diff(rp).max() > 32
    A = dev.from_host(int(seg[-1]), int(seg[-1]), rp, col, val)
    hb = rng.standard_normal(int(seg[-1]))
    b = torch.from_numpy(hb).cuda()
    tR = torch.from_numpy(seg).cuda()
    rc, x, it, res, conv = batched_solve(A, b, tR, len(blocks), 2000, 1e-8)
    assert rc == 0 and conv.all()
    check_against_restatement(oracle, rp, col, val, seg, hb, x.cpu().numpy(), it,
                              range(len(blocks)))


def test_batched_cg_many_instances_tile_walk(cuda, oracle):
    """More instances than the active list holds (1024): the solver walks all
    tiles and skips converged instances."""
    rng = np.random.default_rng(5)
    nseg = 1100
    sides = rng.integers(3, 9, nseg)
    shifts = rng.uniform(0.05, 1.0, nseg)
    A, b, tR, seg_rows = make_batch(sides, shifts)
    rc, x, it, res, conv = batched_solve(A, b, tR, nseg, 2000, 1e-8)
    assert rc == 0 and conv.all()
    o, i, v = A.to_host()
    check_against_restatement(oracle, o, i, v, seg_rows, b.cpu().numpy(), x.cpu().numpy(), it,
                              list(range(0, nseg, 37)) + [nseg - 1])
