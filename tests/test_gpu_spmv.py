"""GPU parity of the SpMV engine, the generators and the device build against
the oracle (C restatement, pinned to the reference) and the golden fixtures
written by the unmodified reference.  Everything is called through the C-ABI.

Tolerances: bool and int32 semirings bit-exact; FP64 plus-times relative
1e-12 per entry (summation order differs from the reference's sequential
row sums)."""
import numpy as np
import pytest

import golden_cases as G

pytestmark = pytest.mark.gpu

FP64, INT32, BOOL, VOID = 3, 2, 1, 0
RTOL = 1e-12


def _dev():
    from alp_b200 import device
    return device


def _np(t):
    return t.cpu().numpy()


def assert_ring_equal(ring, got, want, where=None):
    if G.RING_TYPE[ring] == FP64:
        np.testing.assert_allclose(got, want, rtol=RTOL, atol=1e-300, err_msg=str(where))
    else:
        np.testing.assert_array_equal(got, want, err_msg=str(where))


# ------------------------------------------------------------- generators --
@pytest.mark.parametrize("vtype", [FP64, INT32, BOOL])
def test_rmat_generator_matches_oracle(cuda, oracle, vtype):
    dev = _dev()
    A = dev.rmat(12, vtype=vtype, seed=7)
    rp, col, vals = oracle.rmat(12, vtype=vtype, seed=7)
    o, i, v = A.to_host()
    np.testing.assert_array_equal(o, rp)
    np.testing.assert_array_equal(i[:A.nnz], col)
    np.testing.assert_array_equal(v[:A.nnz], vals)


def test_value_generator_matches_oracle(cuda, oracle):
    dev = _dev()
    for vtype in (FP64, INT32, BOOL):
        t = dev.gen_values(10000, vtype, seed=5, sid=3, lo=-7, hi=99, p=0.3)
        np.testing.assert_array_equal(_np(t), oracle.values(10000, vtype, 5, 3, -7, 99, 0.3))


@pytest.mark.parametrize("sizes", [(8, 9, 10), (16, 16, 16), (5, 7)])
def test_stencil_matches_reference_build(cuda, oracle, sizes):
    dev = _dev()
    A = dev.stencil(sizes, 26.0, -1.0, ref_order=True)
    I, J, V = oracle.stencil_coo(sizes, 26.0, -1.0)
    rp, col, vals = oracle.coo_to_crs(int(np.prod(sizes)), I, J, V, FP64)
    o, i, v = A.to_host()
    np.testing.assert_array_equal(o, rp)
    np.testing.assert_array_equal(i, col)
    np.testing.assert_array_equal(v, vals)


@pytest.mark.parametrize("L", [2, 3, 32, 100])
def test_poisson2d(cuda, L):
    dev = _dev()
    A = dev.poisson2d(L, 0.25)
    o, i, v = A.to_host()
    dense = np.zeros((L * L, L * L))
    for y in range(L):
        for x in range(L):
            r = y * L + x
            dense[r, r] = 4.25
            for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                if 0 <= x + dx < L and 0 <= y + dy < L:
                    dense[r, (y + dy) * L + x + dx] = -1.0
    got = np.zeros_like(dense)
    for r in range(L * L):
        cols = i[o[r]:o[r + 1]]
        assert np.all(np.diff(cols.astype(np.int64)) > 0)
        got[r, cols] = v[o[r]:o[r + 1]]
    np.testing.assert_array_equal(got, dense)
    assert A.nnz == 5 * L * L - 4 * L


def test_coo_to_crs_keeps_reference_row_order(cuda, oracle):
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    rng = np.random.default_rng(1)
    m, n, nnz = 300, 200, 5000
    keys = np.unique(rng.integers(0, m * n, size=nnz))
    rng.shuffle(keys)
    I = (keys // n).astype(np.uint32)
    J = (keys % n).astype(np.uint32)
    V = rng.random(len(keys))
    rp, col, vals = oracle.coo_to_crs(m, I, J, V, FP64)
    d = torch.device("cuda")
    tI = torch.from_numpy(I.view(np.int32)).to(d)
    tJ = torch.from_numpy(J.view(np.int32)).to(d)
    tV = torch.from_numpy(V).to(d)
    o = torch.empty(m + 1, dtype=torch.int64, device=d)
    c = torch.empty(len(I), dtype=torch.int32, device=d)
    w = torch.empty(len(I), dtype=torch.float64, device=d)
    abi.call("alpb_coo_to_crs", m, n, len(I), dev.ptr(tI), dev.ptr(tJ), dev.ptr(tV), FP64,
             dev.ptr(o), dev.ptr(c), dev.ptr(w), dev.stream_ptr())
    np.testing.assert_array_equal(_np(o), rp)
    np.testing.assert_array_equal(_np(c).view(np.uint32), col)
    np.testing.assert_array_equal(_np(w), vals)
    # out-of-range coordinate -> MISMATCH, outputs untouched semantics
    tI[0] = m
    with pytest.raises(abi.AlpError) as e:
        abi.call("alpb_coo_to_crs", m, n, len(I), dev.ptr(tI), dev.ptr(tJ), dev.ptr(tV), FP64,
                 dev.ptr(o), dev.ptr(c), dev.ptr(w), dev.stream_ptr())
    assert e.value.rc == abi.MISMATCH


def test_transpose_matches_oracle(cuda, oracle):
    dev = _dev()
    A = dev.rmat(11, vtype=FP64, seed=3)
    T = dev.transpose(A)
    rp, col, vals = A.to_host()
    cp, row, tv = oracle.transpose(A.m, A.n, rp, col[:A.nnz], vals[:A.nnz], FP64)
    o, i, v = T.to_host()
    np.testing.assert_array_equal(o, cp)
    np.testing.assert_array_equal(i[:A.nnz], row)
    np.testing.assert_array_equal(v[:A.nnz], tv)


# --------------------------------------------------------------------- mxv --
SCHEDS = [("merge", 1, 0), ("vector1", 2, 1), ("vector4", 2, 4), ("vector32", 2, 32)]


@pytest.mark.parametrize("ring", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("sched", SCHEDS, ids=[s[0] for s in SCHEDS])
@pytest.mark.parametrize("form", [2, 1], ids=["mxv", "vxm"])
def test_mxv_dense_parity(cuda, oracle, ring, sched, form):
    import torch
    dev = _dev()
    t = G.RING_TYPE[ring]
    vt = t
    A = dev.rmat(13, vtype=vt, seed=21 + ring, lo=1, hi=100)
    S = A if form == 2 else dev.transpose(A)
    x = dev.gen_values(A.n, t, seed=4, lo=0, hi=1000)
    u0 = dev.gen_values(A.m, t, seed=6, lo=0, hi=5000)
    if ring == 1:
        x = dev.gen_values(A.n, BOOL, seed=4, p=0.3)
        u0 = dev.gen_values(A.m, BOOL, seed=6, p=0.2)
    u = u0.clone()
    plan = dev.Plan(S, sched=sched[1], vector_width=sched[2])
    dev.mxv(ring, S, u, x, form=form, plan=plan)
    torch.cuda.synchronize()
    o, i, v = S.to_host()
    want = _np(u0).copy()
    rc, _ = oracle.mxv(ring, 0, form, S.m, S.n, o, i[:S.nnz], None if v is None else v[:S.nnz],
                       vt, want, v=_np(x))
    assert rc == 0
    assert_ring_equal(ring, _np(u), want)
    # a second product with the same plan (counters were reset)
    u2 = u0.clone()
    dev.mxv(ring, S, u2, x, form=form, plan=plan)
    assert torch.equal(u, u2), "merge path must be deterministic"


@pytest.mark.parametrize("ring", [5, 6, 7])
@pytest.mark.parametrize("sched", SCHEDS, ids=[s[0] for s in SCHEDS])
@pytest.mark.parametrize("form", [2, 1], ids=["mxv", "vxm"])
@pytest.mark.parametrize("pattern", [False, True], ids=["valued", "void"])
def test_mxv_pregel_and_switched_rings(cuda, oracle, ring, sched, form, pattern):
    """The Pregel degree ring (add, right_assign_if over size_t), its message
    ring under max (max, left_assign_if) and the switched (times, plus) ring on
    R-MAT scale 13, every schedule, valued and pattern matrices: bit-exact for
    the u64 rings, 1e-12 relative for the FP64 products (different order)."""
    import torch
    dev = _dev()
    t = G.RING_TYPE[ring]
    n, I, J, V, v, u0 = G.new_ring_case(oracle, ring, 13, 500 + ring)
    vt = VOID if pattern else t
    rp, col, vals = oracle.coo_to_crs(n, I, J, None if pattern else V, vt)
    if form == 1:
        rp, col, vals = oracle.transpose(n, n, rp, col, vals, vt)
    view = (lambda a: a.view(np.int64)) if t == G.INT64 else (lambda a: a)
    S = dev.from_host(n, n, rp, col, None if pattern else view(vals), vt)
    x = torch.from_numpy(view(v).copy()).cuda()
    u = torch.from_numpy(view(u0).copy()).cuda()
    plan = dev.Plan(S, sched=sched[1], vector_width=sched[2])
    dev.mxv(ring, S, u, x, form=form, plan=plan)
    torch.cuda.synchronize()
    want = u0.copy()
    rc, _ = oracle.mxv(ring, 0, form, n, n, rp, col, vals, vt, want, v=v)
    assert rc == 0
    got = _np(u).view(np.uint64) if t == G.INT64 else _np(u)
    assert_ring_equal(ring, got, want)


@pytest.mark.parametrize("name", sorted(G.mxv_cases()[1].keys()))
def test_mxv_golden_reference(cuda, oracle, name):
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    mats, cases = G.mxv_cases()
    c = cases[name]
    ring, descr, vxm_form = int(c["ring"]), int(c["descr"]), int(c["vxm_form"])
    mat = mats[f"mat{ring}"]
    n = int(mat["n"])
    t = G.RING_TYPE[ring]
    rp, col, vals, form, _ = G.gather_storage(oracle, mat, ring, vxm_form, descr)
    S = dev.from_host(n, n, rp, col, vals, t)
    u, ua, v, va, um, uma, umc, vm, vma, vmc, vc = G.vector_args(c, n)
    d = torch.device("cuda")
    T = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(d)
    tu, tua, tv, tva = T(u), T(ua), T(v), T(va)
    tnnz = None if ua is None else torch.tensor([int(ua.sum())], dtype=torch.int64, device=d)
    dev.mxv(ring, S, tu, tv, descr=descr & ~G.TRANSPOSE, form=form, u_assigned=tua, u_nnz=tnnz,
            u_mask=T(um), u_mask_assigned=T(uma), u_mask_type=abi.BOOL, u_mask_count=umc,
            v_assigned=tva, v_count=vc, v_mask=T(vm), v_mask_assigned=T(vma),
            v_mask_type=abi.BOOL, v_mask_count=vmc)
    torch.cuda.synchronize()
    ref_a = c["ua_out"].astype(bool)
    got_a = _np(tua).astype(bool) if tua is not None else np.ones(n, bool)
    np.testing.assert_array_equal(got_a, ref_a)
    if tnnz is not None:
        assert int(tnnz.item()) == int(ref_a.sum())
    assert_ring_equal(ring, _np(tu)[ref_a], c["u_out"][ref_a], name)


@pytest.mark.parametrize("xcase", ["half", "sparse", "none", "one_late"])
@pytest.mark.parametrize("valued", [False, True], ids=["void", "bool"])
@pytest.mark.parametrize("form", [2, 1], ids=["mxv", "vxm"])
def test_lor_land_early_exit_path(cuda, oracle, xcase, valued, form):
    """The lor/land dense path (row heads of 32 nonzeroes, chunks of 256 for
    the rest of long rows, early exit at the first true product, rows already
    true skipped) is bit-exact against the oracle's full gather: x half true,
    1% true (a BFS frontier), all false (no early exit anywhere), and one true
    entry at the column that only the last nonzero of the longest row reads;
    pattern and bool-valued matrices (30% false values); u 20% true."""
    import torch
    dev = _dev()
    A = dev.rmat(13, vtype=BOOL, seed=31)
    if valued:
        A.values.copy_(dev.gen_values(A.nnz, BOOL, seed=32, p=0.7))
    else:
        A = dev.CRS(A.m, A.n, A.nnz, A.offsets, A.indices, None, VOID)
    S = A if form == 2 else dev.transpose(A)
    o, i, v = S.to_host()
    if xcase == "half":
        x = dev.gen_values(S.n, BOOL, seed=4, p=0.5)
    elif xcase == "sparse":
        x = dev.gen_values(S.n, BOOL, seed=4, p=0.01)
    else:
        x = torch.zeros(S.n, dtype=torch.uint8, device="cuda")
        if xcase == "one_late":
            r = int(np.argmax(np.diff(o)))
            assert o[r + 1] - o[r] > 32 + 256, "the longest row must reach a tail chunk"
            x[int(i[o[r + 1] - 1])] = 1
    u0 = dev.gen_values(S.m, BOOL, seed=6, p=0.2)
    u = u0.clone()
    plan = dev.Plan(S, sched=1)
    dev.mxv(1, S, u, x, form=form, plan=plan)
    torch.cuda.synchronize()
    want = _np(u0).copy()
    rc, _ = oracle.mxv(1, 0, form, S.m, S.n, o, i[:S.nnz], None if v is None else v[:S.nnz],
                       BOOL if valued else VOID, want, v=_np(x))
    assert rc == 0
    np.testing.assert_array_equal(_np(u), want)
    if xcase == "one_late":
        assert int(_np(u)[r]) == 1


def test_mxv_error_codes(cuda):
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    A = dev.rmat(8, vtype=FP64)
    x = dev.gen_values(A.n, FP64, seed=1)
    with pytest.raises(abi.AlpError) as e:          # output aliases input
        dev.mxv(0, A, x, x)
    assert e.value.rc == abi.OVERLAP
    with pytest.raises(abi.AlpError) as e:          # semiring not instantiated
        dev.mxv(17, A, torch.zeros_like(x), x)
    assert e.value.rc == abi.UNSUPPORTED
    with pytest.raises(abi.AlpError) as e:          # value type vs ring
        dev.mxv(2, A, torch.zeros(A.m, dtype=torch.int32, device=x.device), x)
    assert e.value.rc == abi.UNSUPPORTED
    va = torch.ones(A.n, dtype=torch.uint8, device=x.device)
    va[0] = 0
    with pytest.raises(abi.AlpError) as e:          # dense descriptor on a sparse input
        dev.mxv(0, A, torch.zeros_like(x), x, descr=16, v_assigned=va)
    assert e.value.rc == abi.ILLEGAL
    B = dev.rmat(9, vtype=FP64)
    plan = dev.Plan(B)
    with pytest.raises(abi.AlpError) as e:          # plan of another matrix
        dev.mxv(0, A, torch.zeros_like(x), x, plan=plan)
    assert e.value.rc == abi.MISMATCH


def test_mxv_trivial_and_empty(cuda, oracle):
    """Empty input / empty matrix: output unchanged; explicit_zero assigns the
    identity (reference/blas2.hpp:1001-1037)."""
    import torch
    dev = _dev()
    A = dev.rmat(8, vtype=FP64)
    d = torch.device("cuda")
    u = torch.full((A.m,), 3.0, dtype=torch.float64, device=d)
    ua = torch.zeros(A.m, dtype=torch.uint8, device=d)
    ua[:10] = 1
    nnz = torch.tensor([10], dtype=torch.int64, device=d)
    x = torch.zeros(A.n, dtype=torch.float64, device=d)
    xa = torch.zeros(A.n, dtype=torch.uint8, device=d)
    dev.mxv(0, A, u, x, u_assigned=ua, u_nnz=nnz, v_assigned=xa, v_count=0)
    assert int(nnz.item()) == 10 and float(u[0]) == 3.0
    dev.mxv(0, A, u, x, descr=512, u_assigned=ua, u_nnz=nnz, v_assigned=xa, v_count=0)
    assert int(nnz.item()) == A.m and float(u[20]) == 0.0 and float(u[0]) == 3.0


@pytest.mark.parametrize("ring", [0, 1, 2])
def test_mxv_full_scale_rmat22(cuda, oracle, ring):
    """The bench workload itself (R-MAT scale 22, ~64M nonzeroes after
    merging duplicates): merge path against the C restatement on the same
    device-built storage."""
    import torch
    dev = _dev()
    t = G.RING_TYPE[ring]
    A = dev.rmat(22, vtype=t, seed=42, lo=1, hi=100)
    x = dev.gen_values(A.n, t, seed=9, lo=0, hi=1000) if ring != 1 else \
        dev.gen_values(A.n, BOOL, seed=9, p=0.5)
    if ring == 2:
        u = torch.full((A.m,), 2**31 - 1, dtype=torch.int32, device=x.device)
    else:
        u = torch.zeros(A.m, dtype=x.dtype, device=x.device)
    u0 = _np(u).copy()
    plan = dev.Plan(A, sched=1)
    dev.mxv(ring, A, u, x, plan=plan)
    torch.cuda.synchronize()
    o, i, v = A.to_host()
    oracle.mxv(ring, 0, 2, A.m, A.n, o, i, v, t, u0, v=_np(x))
    assert_ring_equal(ring, _np(u), u0)


# ------------------------------------------------------------------ BLAS1 --
def test_dot_and_reduce(cuda):
    import torch
    from alp_b200 import _abi as abi
    import ctypes as C
    dev = _dev()
    n = 1_000_003
    x = dev.gen_values(n, FP64, seed=1)
    y = dev.gen_values(n, FP64, seed=2)
    r = C.c_double(0.5)
    abi.call("alpb_dot_f64", C.byref(r), abi.OP_ADD, abi.OP_MUL, n, dev.ptr(x), None, dev.ptr(y),
             None, dev.stream_ptr())
    want = 0.5 + float(np.dot(_np(x), _np(y)))
    assert abs(r.value - want) <= 1e-12 * abs(want)
    r = C.c_double(0.0)
    abi.call("alpb_dot_f64", C.byref(r), abi.OP_ADD, abi.OP_ABS_DIFF, n, dev.ptr(x), None,
             dev.ptr(y), None, dev.stream_ptr())
    want = float(np.abs(_np(x) - _np(y)).sum())
    assert abs(r.value - want) <= 1e-12 * want
    xa = dev.gen_values(n, BOOL, seed=3, p=0.5)
    r = C.c_double(0.0)
    abi.call("alpb_reduce_f64", C.byref(r), abi.OP_ADD, n, dev.ptr(x), dev.ptr(xa),
             dev.stream_ptr())
    want = float(_np(x)[_np(xa) > 0].sum())
    assert abs(r.value - want) <= 1e-12 * want
    r = C.c_double(np.inf)
    abi.call("alpb_reduce_f64", C.byref(r), abi.OP_MIN, n, dev.ptr(x), None, dev.stream_ptr())
    assert r.value == float(_np(x).min())


def test_elementwise(cuda):
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    n = 12345
    a = dev.gen_values(n, FP64, seed=1)
    b = dev.gen_values(n, FP64, seed=2)
    out = torch.empty_like(a)
    abi.call("alpb_ewise_apply_f64", dev.ptr(out), abi.OP_MUL, n, dev.ptr(a), 0.0, dev.ptr(b), 0.0,
             dev.stream_ptr())
    assert torch.equal(out, a * b)
    z = a.clone()
    abi.call("alpb_ewise_muladd_f64", dev.ptr(z), abi.OP_ADD, abi.OP_MUL, n, None, 0.25,
             dev.ptr(b), 0.0, dev.stream_ptr())
    torch.testing.assert_close(z, a + 0.25 * b, rtol=1e-15, atol=0)
    abi.call("alpb_foldl_f64", dev.ptr(z), abi.OP_SUB, n, dev.ptr(b), 0.0, dev.stream_ptr())
    torch.testing.assert_close(z, a + 0.25 * b - b, rtol=1e-15, atol=0)
    abi.call("alpb_set_scalar", dev.ptr(z), FP64, n, 7.0, None, None, dev.stream_ptr())
    assert bool((z == 7.0).all())


@pytest.mark.parametrize("case", ["rmat18", "stencil64"])
def test_autotuner_picks_a_schedule_and_keeps_parity(cuda, oracle, case):
    """The schedule rule and the autotuner (alpb_spmv_autotune).  The rule
    (ALPB_SCHED_AUTO without timing): skewed rows (R-MAT scale 18) take the
    merge path; regular rows (27-point 64^3) take the vector schedule with
    about mean/6 lanes per row (4 for 27 nonzeroes).  The autotuner then times
    the candidates on the device: on R-MAT the vector schedules are several
    times slower, so it must keep the merge path; on the stencil either may
    win.  Whatever it keeps, the product through the tuned plan matches the
    restatement (1e-12 relative) on two calls in a row."""
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    if case == "rmat18":
        A = dev.rmat(18, vtype=FP64, seed=61)
    else:
        A = dev.stencil((64, 64, 64), 26.0, -1.0)
    x = dev.gen_values(A.n, FP64, seed=62)
    u0 = dev.gen_values(A.m, FP64, seed=63)
    plan = dev.Plan(A, sched=abi.SCHED_AUTO)
    sched, vw, _ = plan.info()
    if case == "rmat18":
        assert sched == abi.SCHED_MERGE_PATH
    else:
        assert sched == abi.SCHED_VECTOR and vw == 4, (sched, vw)
    scratch = torch.empty_like(u0)
    plan.autotune(0, x, scratch)
    sched2, vw2, _ = plan.info()
    if case == "rmat18":
        assert sched2 == abi.SCHED_MERGE_PATH
    else:
        assert sched2 in (abi.SCHED_MERGE_PATH, abi.SCHED_VECTOR)
    o, i, v = A.to_host()
    want = _np(u0).copy()
    rc, _ = oracle.mxv(0, 0, 2, A.m, A.n, o, i, v, FP64, want, v=_np(x))
    assert rc == 0
    # the stencil's rows cancel (26 x_i minus 26 neighbours), so the bar is
    # relative to the terms' size, not to the (small) row result
    scale = 1e-12 * 52 * float(np.abs(_np(x)).max()) + 1e-12 * float(np.abs(_np(u0)).max())
    for _ in range(2):
        u = u0.clone()
        dev.mxv(0, A, u, x, plan=plan)
        torch.cuda.synchronize()
        np.testing.assert_allclose(_np(u), want, rtol=1e-12, atol=scale)


def test_vec_engine_integer_domains(cuda):
    """alpb_vec_op_dom / alpb_vec_reduce_dom in the integer domains: int32
    products and sums wrap as 32-bit arithmetic, uint64 values above 2^53 keep
    every bit (numpy's wrapping arithmetic is the checker), and the folded
    result includes the scalar it starts from."""
    import ctypes as C
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    rng = np.random.default_rng(17)
    n = 100_003
    a = rng.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32)
    b = rng.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32)
    u = rng.integers(0, 2**63, n, dtype=np.int64).astype(np.uint64) * np.uint64(2) + np.uint64(1)
    v = rng.integers(0, 2**63, n, dtype=np.int64).astype(np.uint64)
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    tu, tv = torch.from_numpy(u.view(np.int64)).cuda(), torch.from_numpy(v.view(np.int64)).cuda()
    INT32, INT64, UINT64 = abi.INT32, 5, 8
    ADD, MUL, MAX = 0, 2, 5
    # z = a * b in int32 (wraps), computed in the signed 64-bit domain
    z = torch.empty_like(ta)
    abi.call("alpb_vec_op_dom", 3, MUL, 0, 0, 0, 0, INT64, n, dev.ptr(z), INT32, None, None,
             None, None, 0, 0, dev.ptr(ta), INT32, None, 0, dev.ptr(tb), INT32, None, 0,
             dev.stream_ptr())
    with np.errstate(over="ignore"):
        np.testing.assert_array_equal(z.cpu().numpy(), a * b)
    # dot over int32 with 32-bit wrap: fold into 5 in int64, truncate
    r = C.c_uint64(5)
    abi.call("alpb_vec_reduce_dom", C.byref(r), ADD, 0, MUL, 0, INT64, n, dev.ptr(ta), INT32, None,
             dev.ptr(tb), INT32, None, None, None, 0, 0, dev.stream_ptr())
    want = (5 + (a.astype(np.int64) * b.astype(np.int64)).sum()) & 0xffffffff
    assert (r.value & 0xffffffff) == int(want)
    # uint64: z = u + v (wraps mod 2^64), dot and max fold, every bit kept
    z64 = torch.empty_like(tu)
    abi.call("alpb_vec_op_dom", 3, ADD, 0, 0, 0, 0, UINT64, n, dev.ptr(z64), INT64, None, None,
             None, None, 0, 0, dev.ptr(tu), INT64, None, 0, dev.ptr(tv), INT64, None, 0,
             dev.stream_ptr())
    with np.errstate(over="ignore"):
        np.testing.assert_array_equal(z64.cpu().numpy().view(np.uint64), u + v)
    r = C.c_uint64(3)
    abi.call("alpb_vec_reduce_dom", C.byref(r), ADD, 0, MUL, 0, UINT64, n, dev.ptr(tu), INT64,
             None, dev.ptr(tv), INT64, None, None, None, 0, 0, dev.stream_ptr())
    want = 3
    for x, y in zip(u.tolist(), v.tolist()):
        want = (want + x * y) & (2**64 - 1)
    assert r.value == want
    r = C.c_uint64(0)
    abi.call("alpb_vec_reduce_dom", C.byref(r), MAX, 0, MUL, 0, UINT64, n, dev.ptr(tu), INT64,
             None, None, INT64, None, None, None, 0, 0, dev.stream_ptr())
    assert r.value == int(u.max())
    # the int32 domain wraps each operation at 32 bits: a min over wrapped
    # sums differs from a min over the exact sums
    MIN, INT32_DOM = 4, abi.INT32
    z = torch.empty_like(ta)
    abi.call("alpb_vec_op_dom", 3, ADD, 0, 0, 0, 0, INT32_DOM, n, dev.ptr(z), INT32, None, None,
             None, None, 0, 0, dev.ptr(ta), INT32, None, 0, dev.ptr(tb), INT32, None, 0,
             dev.stream_ptr())
    with np.errstate(over="ignore"):
        wrapped = a + b
    np.testing.assert_array_equal(z.cpu().numpy(), wrapped)
    ident = np.array([2**31 - 1], np.int32).view(np.uint32)[0]
    r = C.c_uint64(int(ident))
    abi.call("alpb_vec_reduce_dom", C.byref(r), MIN, int(ident), ADD, 0, INT32_DOM, n,
             dev.ptr(ta), INT32, None, dev.ptr(tb), INT32, None, None, None, 0, 0,
             dev.stream_ptr())
    got = np.array([r.value & 0xffffffff], np.uint32).view(np.int32)[0]
    assert got == wrapped.min() and wrapped.min() != (a.astype(np.int64) + b).min()


@pytest.mark.parametrize("slots", [4096, 16384])
@pytest.mark.parametrize("ring", [0, 1, 2, 5])
@pytest.mark.parametrize("form", [2, 1], ids=["mxv", "vxm"])
def test_hot_column_cache_bit_identical(cuda, oracle, ring, form, slots):
    """The merge path with the hot-column cache (alpb_spmv_plan_hot: the most
    frequent columns' x values in shared memory) gives the merge path's
    result bit for bit -- same products, same sums in the same order -- for
    FP64, boolean, int32 and u64 rings, on two calls in a row; removing the
    cache (0 slots) restores the plain path; too many slots are refused."""
    import ctypes as C
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    t = G.RING_TYPE[ring]
    if t == G.INT64:
        n, I, J, V, v, uh = G.new_ring_case(oracle, ring, 16, 900 + ring)
        rp, col, vals = oracle.coo_to_crs(n, I, J, V, t)
        A = dev.from_host(n, n, rp, col, vals.view(np.int64), t)
        x = torch.from_numpy(v.view(np.int64).copy()).cuda()
        u0 = torch.from_numpy(uh.view(np.int64).copy()).cuda()
    else:
        A = dev.rmat(16, vtype=VOID if ring == 1 else t, seed=70 + ring, lo=1, hi=100)
        if ring == 1:
            x = dev.gen_values(A.n, BOOL, seed=71, p=0.3)
            u0 = dev.gen_values(A.m, BOOL, seed=72, p=0.2)
        else:
            x = dev.gen_values(A.n, t, seed=71, lo=0, hi=1000)
            u0 = dev.gen_values(A.m, t, seed=72, lo=0, hi=1000)
    S = A if form == 2 else dev.transpose(A)
    plan = dev.Plan(S, sched=abi.SCHED_MERGE_PATH)
    want = u0.clone()
    dev.mxv(ring, S, want, x, form=form, plan=plan)
    abi.call("alpb_spmv_plan_hot", plan.h, ring, S.n, dev.ptr(S.indices), slots,
             dev.stream_ptr())
    nslots, cover = C.c_int64(), C.c_double()
    abi.call("alpb_spmv_plan_hot_info", plan.h, C.byref(nslots), C.byref(cover))
    assert nslots.value == slots and 0.1 < cover.value < 1.0, (nslots.value, cover.value)
    for _ in range(2):
        got = u0.clone()
        dev.mxv(ring, S, got, x, form=form, plan=plan)
        torch.cuda.synchronize()
        assert torch.equal(got, want)
    abi.call("alpb_spmv_plan_hot", plan.h, ring, S.n, dev.ptr(S.indices), 0, dev.stream_ptr())
    abi.call("alpb_spmv_plan_hot_info", plan.h, C.byref(nslots), C.byref(cover))
    assert nslots.value == 0
    got = u0.clone()
    dev.mxv(ring, S, got, x, form=form, plan=plan)
    torch.cuda.synchronize()
    assert torch.equal(got, want)
    rc = abi.lib().alpb_spmv_plan_hot(plan.h, ring, S.n, dev.ptr(S.indices), 1 << 20,
                                      dev.stream_ptr())
    assert rc == abi.ILLEGAL


@pytest.mark.parametrize("slots", [4096, 16384])
def test_hot_column_cache_matches_restatement_rmat22(cuda, oracle, slots):
    """The benchmark's product (R-MAT scale 22, FP64 plus-times) through a plan
    with the hot-column cache, against the restatement (1e-12 relative)."""
    import ctypes as C
    import torch
    from alp_b200 import _abi as abi
    dev = _dev()
    A = dev.rmat(22, vtype=FP64, seed=42)
    x = dev.gen_values(A.n, FP64, seed=49)
    u = torch.zeros(A.m, dtype=torch.float64, device="cuda")
    plan = dev.Plan(A, sched=abi.SCHED_MERGE_PATH)
    abi.call("alpb_spmv_plan_hot", plan.h, 0, A.n, dev.ptr(A.indices), slots, dev.stream_ptr())
    got, cover = C.c_int64(), C.c_double()
    abi.call("alpb_spmv_plan_hot_info", plan.h, C.byref(got), C.byref(cover))
    assert got.value == slots and cover.value > 0.15
    dev.mxv(0, A, u, x, plan=plan)
    torch.cuda.synchronize()
    o, i, v = A.to_host()
    want = np.zeros(A.m)
    rc, _ = oracle.mxv(0, 0, 2, A.m, A.n, o, i, v, FP64, want, v=_np(x))
    assert rc == 0
    np.testing.assert_allclose(_np(u), want, rtol=1e-12, atol=1e-300)
