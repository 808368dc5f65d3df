"""Fused level-1 chains (alpb_vec_chain, and the C++ backend's lazy recording
of set / foldl / foldr / eWiseMul / eWiseMulAdd steps on dense vectors): one
device pass must give, bit for bit, what the steps give one by one through
alpb_vec_op_dom followed by alpb_vec_reduce_dom -- every element-wise step is
the same arithmetic, and the closing reduction runs on the same grid in the
same order.  ALP's own GMRES smoke program must print the same results with
the fusion on and off (ALPB_FUSE=0), and fuse steps when on."""
import ctypes as C
import re
import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64, INT64 = 3, 5
ADD, SUB, MUL, DIV, MIN, MAX = 0, 1, 2, 3, 4, 5


def _bits(v, dom):
    if dom == FP64:
        return struct.unpack("<Q", struct.pack("<d", v))[0]
    return int(v) & 0xFFFFFFFFFFFFFFFF


def _steps(dom):
    """A chain over slots z, w, v (outputs) and x, y (inputs), closed by a dot:
    z += alpha x; w (+)= z; w = x - w; v = w; v += w * y; v = max(v, beta);
    dot(v, w)."""
    from alp_b200 import _abi as abi
    a, b = (0.375, -1.5) if dom == FP64 else (3, -7)
    Z, W, V, X, Y = range(5)
    S = abi.VecStep
    return [
        S(kind=abi.VEC_MULADD, op=ADD, mul_op=MUL, z=Z, x=-1, y=X, alpha=_bits(a, dom)),
        S(kind=abi.VEC_FOLDL, op=ADD, z=W, x=Z, y=-1),
        S(kind=abi.VEC_FOLDR, op=SUB, z=W, x=X, y=-1),
        S(kind=abi.VEC_SET, op=ADD, z=V, x=W, y=-1),
        S(kind=abi.VEC_MULADD, op=ADD, mul_op=MUL, z=V, x=W, y=Y),
        S(kind=abi.VEC_FOLDL, op=MAX, z=V, x=-1, y=-1, alpha=_bits(b, dom)),
        S(kind=abi.VEC_REDUCE, op=ADD, mul_op=MUL, z=0, x=V, y=W, identity=_bits(0, dom)),
    ]


def _vectors(dom, n, seed):
    import torch
    g = torch.Generator().manual_seed(seed)
    if dom == FP64:
        mk = lambda: torch.randn(n, generator=g, dtype=torch.float64)
    else:  # values near 2^61: the products and sums wrap around in int64
        mk = lambda: torch.randint(-(1 << 61), 1 << 61, (n,), generator=g, dtype=torch.int64)
    return [mk().cuda() for _ in range(5)]


def _one_by_one(dom, vecs, steps, init):
    """The same steps through the unfused entry points."""
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    lib = abi.lib()
    n = vecs[0].numel()
    ptr = [dev.ptr(t) for t in vecs]
    for s in steps[:-1]:
        x = ptr[s.x] if s.x >= 0 else None
        y = ptr[s.y] if s.kind == abi.VEC_MULADD and s.y >= 0 else None
        rc = lib.alpb_vec_op_dom(s.kind, s.op, 0, 0, s.mul_op, s.descr, dom, n, ptr[s.z], dom,
                                 None, None, None, None, 0, 0, x, dom, None, s.alpha, y, dom,
                                 None, s.beta, dev.stream_ptr())
        assert rc == abi.SUCCESS, abi.last_error()
    r = steps[-1]
    res = C.c_uint64(init)
    rc = lib.alpb_vec_reduce_dom(C.byref(res), r.op, r.identity, r.mul_op, 0, dom, n, ptr[r.x],
                                 dom, None, ptr[r.y], dom, None, None, None, 0, 0,
                                 dev.stream_ptr())
    assert rc == abi.SUCCESS, abi.last_error()
    return res.value


@pytest.mark.parametrize("dom", [FP64, INT64], ids=["fp64", "int64"])
@pytest.mark.parametrize("n", [1, 1000, 1_000_003])
def test_chain_matches_steps_one_by_one(cuda, dom, n):
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    steps = _steps(dom)
    init = _bits(0.25 if dom == FP64 else 11, dom)
    ref = _vectors(dom, n, 5)
    fused = [t.clone() for t in ref]
    want = _one_by_one(dom, ref, steps, init)
    arr = (abi.VecStep * len(steps))(*steps)
    vals = (C.c_void_p * 5)(*[dev.ptr(t) for t in fused])
    types = (C.c_int * 5)(*([dom] * 5))
    got = C.c_uint64(init)
    rc = abi.lib().alpb_vec_chain(dom, n, 5, vals, types, len(steps), arr, C.byref(got),
                                  dev.stream_ptr())
    assert rc == abi.SUCCESS, abi.last_error()
    torch.cuda.synchronize()
    for k, (a, b) in enumerate(zip(fused, ref)):
        assert torch.equal(a, b), f"slot {k}"
    assert got.value == want


def test_chain_without_reduction_and_errors(cuda):
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    lib = abi.lib()
    n = 4097
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    z = torch.randn(n, dtype=torch.float64, device="cuda")
    z0, x0 = z.clone(), x.clone()
    vals = (C.c_void_p * 2)(dev.ptr(z), dev.ptr(x))
    types = (C.c_int * 2)(FP64, FP64)
    S = abi.VecStep
    steps = (S * 2)(S(kind=abi.VEC_FOLDL, op=MUL, z=0, x=1, y=-1),
                    S(kind=abi.VEC_SET, op=ADD, descr=64, z=1, x=-1, y=-1))  # use_index
    assert lib.alpb_vec_chain(FP64, n, 2, vals, types, 2, steps, None,
                              dev.stream_ptr()) == abi.SUCCESS
    torch.cuda.synchronize()
    assert torch.equal(z, z0 * x0)   # z (*)= x, then x = index: z saw the old x
    np.testing.assert_array_equal(x.cpu().numpy(), np.arange(n, dtype=np.float64))
    # left_assign_if may leave entries unassigned: refused
    bad = (S * 1)(S(kind=abi.VEC_FOLDL, op=11, z=0, x=1, y=-1))
    assert lib.alpb_vec_chain(FP64, n, 2, vals, types, 1, bad, None,
                              dev.stream_ptr()) == abi.UNSUPPORTED
    # a reduction must be the last step
    red = (S * 2)(S(kind=abi.VEC_REDUCE, op=ADD, mul_op=MUL, z=0, x=0, y=1),
                  S(kind=abi.VEC_FOLDL, op=ADD, z=0, x=1, y=-1))
    got = C.c_uint64(0)
    assert lib.alpb_vec_chain(FP64, n, 2, vals, types, 2, red, C.byref(got),
                              dev.stream_ptr()) == abi.ILLEGAL
    # every vector in the domain's own type
    types_bad = (C.c_int * 2)(FP64, 2)
    assert lib.alpb_vec_chain(FP64, n, 2, vals, types_bad, 2, steps, None,
                              dev.stream_ptr()) == abi.UNSUPPORTED


def _smoke(name, *args, fuse):
    import os
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    exe = root / "_build" / "cpp" / f"smoke_{name}_b200"
    if not exe.exists():
        pytest.fail(f"{exe} is not built (build() compiles it where the ALP sources exist)")
    env = dict(os.environ, ALPB_TRACE="1", ALPB_FUSE="1" if fuse else "0")
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=900,
                       env=env)
    out = r.stdout + r.stderr
    assert r.returncode == 0 and "Test OK" in out, out[-3000:]
    # one line per grb::finalize (the program may initialise more than once):
    # the counters are cumulative, so the last line has the totals
    m = re.findall(r"fused level-1 passes (\d+) for (\d+) steps, kernel launches (\d+)", out)
    assert m, out[-2000:]
    results = [l for l in out.splitlines()
               if re.search(r"iterations|residual|x\[\d+\]|converge", l) and "time" not in l]
    return results, int(m[-1][0]), int(m[-1][1]), int(m[-1][2])


@pytest.mark.parametrize("prog,args", [("gmres", ("--n", 256))], ids=["gmres"])
def test_alp_programs_same_with_and_without_fusion(cuda, prog, args):
    """ALP's GMRES smoke program, unchanged: the printed iteration counts and
    residuals are identical with the fusion on and off; with it on, chains of
    several steps run as single passes and fewer kernels are launched."""
    on, runs, steps, launches_on = _smoke(prog, *args, fuse=True)
    off, runs0, steps0, launches_off = _smoke(prog, *args, fuse=False)
    assert on == off and on
    assert runs0 == 0 and steps0 == 0
    assert runs > 0 and steps > runs, (runs, steps)
    assert launches_on < launches_off, (launches_on, launches_off)
