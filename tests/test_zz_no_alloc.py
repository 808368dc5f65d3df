"""The allocation-free entry point, alpb_mxv_dense_noalloc.

It exists for callers that cannot allocate device memory at call time: a
program whose memory pool already owns the whole device, code that runs
inside an allocator or a stream callback, or a latency-critical thread that
must not meet cudaMalloc's implicit synchronisation.  It must give what the
regular entry point alpb_mxv gives on the same inputs, on two calls in a row
(its scratch array keeps the previous call's contents, so the second call
checks that whatever must start from zero is cleared).  The file is collected
last, so a run that stops at its first failure has run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOOL, INT32, FP64 = 1, 2, 3
RING_TYPE = {0: FP64, 1: BOOL, 2: INT32}


@pytest.mark.parametrize("ring", [0, 1, 2])
@pytest.mark.parametrize("form", [2, 1], ids=["mxv", "vxm"])
def test_noalloc_matches_alpb_mxv_on_two_calls(cuda, ring, form):
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    t = RING_TYPE[ring]
    A = dev.rmat(16, vtype=t, seed=31 + ring, lo=1, hi=100)
    S = A if form == 2 else dev.transpose(A)
    if ring == 1:
        x = dev.gen_values(S.n, BOOL, seed=2, p=0.3)
        u0 = dev.gen_values(S.m, BOOL, seed=3, p=0.2)
    else:
        x = dev.gen_values(S.n, t, seed=2, lo=0, hi=1000)
        u0 = dev.gen_values(S.m, t, seed=3, lo=0, hi=1000)
    want = u0.clone()
    dev.mxv(ring, S, want, x, form=form, plan=dev.Plan(S, sched=abi.SCHED_MERGE_PATH))
    torch.cuda.synchronize()
    for call in range(2):
        got = u0.clone()
        rc = abi.lib().alpb_mxv_dense_noalloc(ring, form, S.m, S.n, S.nnz, dev.ptr(S.offsets),
                                              dev.ptr(S.indices), dev.ptr(S.values), S.vtype,
                                              dev.ptr(got), dev.ptr(x), dev.stream_ptr())
        assert rc == abi.SUCCESS, abi.last_error()
        torch.cuda.synchronize()
        if t == FP64:
            np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=1e-12, atol=0,
                                       err_msg=f"call {call}")
        else:
            np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy(),
                                          err_msg=f"call {call}")


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    from alp_b200 import _abi as abi
    m = 1 << 30
    rc = abi.lib().alpb_mxv_dense_noalloc(0, 2, m, m, 1 << 30, None, None, None, FP64, None,
                                          None, None)
    assert rc == abi.ILLEGAL
    assert "scratch limit" in abi.last_error()


@pytest.mark.parametrize("case", ["void", "plus_pattern", "u64_degree", "u64_message",
                                  "tile_multiple"])
def test_noalloc_more_rings_and_shapes(cuda, oracle, case):
    """A pattern (void) matrix, the plus-pattern ring (PageRank's out-degree
    ring), both unsigned 64-bit Pregel rings, and a matrix whose merge list
    (rows + nonzeroes) is an exact multiple of the 2048-item tile, each on two
    calls in a row against alpb_mxv on the merge-path schedule."""
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    import golden_cases as G
    ring = {"void": 0, "plus_pattern": 3, "u64_degree": 5, "u64_message": 6,
            "tile_multiple": 0}[case]
    t = G.RING_TYPE[ring]
    if case == "tile_multiple":
        # rows + nonzeroes = 8 * 2048: a 1024-row band matrix with 15 per row
        m = 1024
        per = 15
        rp = np.arange(m + 1, dtype=np.int64) * per
        col = ((np.arange(m)[:, None] + np.arange(per)[None, :]) % m).astype(np.uint32).ravel()
        col.reshape(m, per).sort(axis=1)
        assert (m + len(col)) % 2048 == 0
        vals = oracle.values(len(col), FP64, 71)
        S = dev.from_host(m, m, rp, col, vals, FP64)
        x = dev.gen_values(m, FP64, seed=72)
        u0 = dev.gen_values(m, FP64, seed=73)
    elif t == G.INT64:
        n, I, J, V, v, uh = G.new_ring_case(oracle, ring, 12, 700 + ring)
        rp, col, vals = oracle.coo_to_crs(n, I, J, V, t)
        S = dev.from_host(n, n, rp, col, vals.view(np.int64), t)
        x = torch.from_numpy(v.view(np.int64).copy()).cuda()
        u0 = torch.from_numpy(uh.view(np.int64).copy()).cuda()
    else:
        A = dev.rmat(14, vtype=FP64, seed=81)
        vt = abi.VOID if case == "void" else FP64
        S = A if vt == FP64 else dev.CRS(A.m, A.n, A.nnz, A.offsets, A.indices, None, abi.VOID)
        x = dev.gen_values(S.n, FP64, seed=82)
        u0 = dev.gen_values(S.m, FP64, seed=83)
    want = u0.clone()
    dev.mxv(ring, S, want, x, plan=dev.Plan(S, sched=abi.SCHED_MERGE_PATH))
    torch.cuda.synchronize()
    for call in range(2):
        got = u0.clone()
        rc = abi.lib().alpb_mxv_dense_noalloc(ring, 2, S.m, S.n, S.nnz, dev.ptr(S.offsets),
                                              dev.ptr(S.indices), dev.ptr(S.values), S.vtype,
                                              dev.ptr(got), dev.ptr(x), dev.stream_ptr())
        assert rc == abi.SUCCESS, abi.last_error()
        torch.cuda.synchronize()
        if t == FP64:
            np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=1e-12, atol=0,
                                       err_msg=f"call {call}")
        else:
            np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy(),
                                          err_msg=f"call {call}")


def test_noalloc_rejects_partly_overlapping_vectors(cuda):
    """u and v sharing only some bytes is an overlap too."""
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    A = dev.rmat(10, vtype=FP64, seed=5)
    buf = torch.zeros(A.m + A.n, dtype=torch.float64, device="cuda")
    u = buf[: A.m]
    v = buf[A.m // 2: A.m // 2 + A.n]
    rc = abi.lib().alpb_mxv_dense_noalloc(0, 2, A.m, A.n, A.nnz, dev.ptr(A.offsets),
                                          dev.ptr(A.indices), dev.ptr(A.values), FP64,
                                          dev.ptr(u), dev.ptr(v), dev.stream_ptr())
    assert rc == abi.OVERLAP
