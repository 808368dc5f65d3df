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
