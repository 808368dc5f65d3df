"""Device HPCG (alpb_hpcg_*) against grb::algorithms::hpcg run unchanged on ALP's
reference backend (tests/cpp/hpcg_driver.cpp, built into oracle/_ref/cpp by
__graft_entry__.build()), on the systems build_hpcg_system makes.

Parity bar: the same iteration count, and x within a relative 1e-9 of the
reference solution (FP64; the sums differ only in rounding).  The known answer
of ALP's HPCG smoke test (16^3, b = A 1, 56 iterations, ||x - 1|| < 4e-14) is
checked too."""
import ctypes as C
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
CHECKER = ROOT / "oracle" / "_ref" / "cpp" / "hpcg_driver_ref"


def reference(nx, levels, colors, pre, post, max_iter, tol, precondition, b=None):
    if not CHECKER.exists():
        pytest.fail(f"{CHECKER} is not built (build() compiles it where the ALP sources exist)")
    with tempfile.TemporaryDirectory() as d:
        rhs = "-"
        if b is not None:
            rhs = str(Path(d) / "b.bin")
            np.asarray(b, np.float64).tofile(rhs)
        xo = Path(d) / "x.bin"
        r = subprocess.run([str(CHECKER), *map(str, (nx, nx, nx, levels, colors, pre, post,
                                                      max_iter, tol, int(precondition))),
                            rhs, str(xo)], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        out = dict(line.split() for line in r.stdout.splitlines() if len(line.split()) == 2)
        return int(out["iterations"]), float(out["residual"]), np.fromfile(xo)


class Hpcg:
    def __init__(self, nx, levels, colors, nrhs):
        from alp_b200 import _abi as abi
        from alp_b200 import device as dev
        self.h = C.c_void_p()
        abi.call("alpb_hpcg_create", C.byref(self.h), nx, nx, nx, 26.0, -1.0, colors, 4, levels,
                 nrhs, dev.stream_ptr())
        self.nrhs = nrhs
        lv, n, nnz, fused = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int()
        abi.call("alpb_hpcg_info", self.h, C.byref(lv), C.byref(n), C.byref(nnz), C.byref(fused))
        self.levels, self.n, self.nnz, self.fused = lv.value, n.value, nnz.value, fused.value

    def ones_rhs(self):
        """b = A 1 on the device, for every right-hand side."""
        import torch
        from alp_b200 import _abi as abi
        from alp_b200 import device as dev
        o, i, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
        n, nnz = C.c_int64(), C.c_int64()
        abi.call("alpb_hpcg_matrix", self.h, 0, C.byref(o), C.byref(i), C.byref(v), C.byref(n),
                 C.byref(nnz))
        ones = torch.ones(self.n, dtype=torch.float64, device="cuda")
        b = torch.zeros(self.n, dtype=torch.float64, device="cuda")
        abi.call("alpb_mxv", 0, 0, 2, self.n, self.n, nnz.value, o, i, v, 3,
                 dev.ptr(b), None, None, None, None, 1, -1,
                 dev.ptr(ones), None, self.n, None, None, 1, -1, None, dev.stream_ptr())
        return b.repeat_interleave(self.nrhs)

    def solve(self, b, max_iter, tol, precondition=True, pre=1, post=1):
        import torch
        from alp_b200 import _abi as abi
        from alp_b200 import device as dev
        x = torch.zeros(self.n * self.nrhs, dtype=torch.float64, device="cuda")
        it = (C.c_int64 * self.nrhs)()
        res = (C.c_double * self.nrhs)()
        abi.call("alpb_hpcg_solve", self.h, dev.ptr(b), dev.ptr(x), int(precondition), pre, post,
                 max_iter, tol, it, res, dev.stream_ptr())
        torch.cuda.synchronize()
        return list(it), list(res), x.view(self.n, self.nrhs).cpu().numpy()

    def close(self):
        from alp_b200 import _abi as abi
        abi.lib().alpb_hpcg_destroy(self.h)


def test_hpcg_smoke_known_answer(cuda):
    """16^3, two levels, 27 colours, b = A 1, x0 = 0, 56 iterations, tolerance 0."""
    h = Hpcg(16, 1, 27, 1)
    assert h.levels == 2 and h.n == 4096
    it, res, x = h.solve(h.ones_rhs(), 56, 0.0)
    ir, rr, xr = reference(16, 1, 27, 1, 1, 56, 0.0, True)
    h.close()
    assert it[0] == ir == 56
    assert np.abs(x[:, 0] - 1).max() < 4e-14
    np.testing.assert_allclose(x[:, 0], xr, rtol=0, atol=1e-14)


@pytest.mark.parametrize("nx,levels", [(16, 1), (32, 2)])
def test_hpcg_eight_rhs_match_reference(cuda, oracle, nx, levels):
    """8 random right-hand sides (N(0,1)) solved together; each against its
    own reference run."""
    import torch
    h = Hpcg(nx, levels, 27, 8)
    rng = np.random.default_rng(nx)
    b = rng.standard_normal((h.n, 8))
    it, res, x = h.solve(torch.from_numpy(b.reshape(-1)).cuda(), 200, 1e-9)
    h.close()
    for k in range(8):
        ir, rr, xr = reference(nx, levels, 27, 1, 1, 200, 1e-9, True, b[:, k])
        assert it[k] == ir, (k, it[k], ir)
        np.testing.assert_allclose(x[:, k], xr, rtol=1e-9, atol=1e-9 * np.abs(xr).max())
        assert abs(res[k] - rr) <= 1e-6 * rr + 1e-300, (k, res[k], rr)


def test_hpcg_rhs_counts_agree(cuda):
    """The same system and right-hand side with 1, 2, 4 and 8 columns."""
    import torch
    rng = np.random.default_rng(5)
    b1 = rng.standard_normal(16 ** 3)
    sols = {}
    for nrhs in (1, 2, 4, 8):
        h = Hpcg(16, 1, 27, nrhs)
        b = torch.from_numpy(np.repeat(b1, nrhs)).cuda()
        it, _, x = h.solve(b, 100, 1e-10)
        h.close()
        assert len(set(it)) == 1
        for k in range(nrhs):
            np.testing.assert_allclose(x[:, k], x[:, 0], rtol=0, atol=0)
        sols[nrhs] = (it[0], x[:, 0])
    for nrhs in (2, 4, 8):
        assert sols[nrhs][0] == sols[1][0]
        np.testing.assert_allclose(sols[nrhs][1], sols[1][1], rtol=1e-11,
                                   atol=1e-11 * np.abs(sols[1][1]).max())


def test_hpcg_conflicting_colours_two_pass(cuda):
    """16 colours on a 16^3 grid put y-neighbours in one colour: the smoother
    must store each colour's products before updating (Jacobi within a
    colour, as the masked mxv of the reference does)."""
    import torch
    h = Hpcg(16, 1, 16, 2)
    assert h.fused == 0
    rng = np.random.default_rng(9)
    b = rng.standard_normal((h.n, 2))
    it, res, x = h.solve(torch.from_numpy(b.reshape(-1)).cuda(), 200, 1e-9)
    h.close()
    for k in range(2):
        ir, rr, xr = reference(16, 1, 16, 1, 1, 200, 1e-9, True, b[:, k])
        assert it[k] == ir
        np.testing.assert_allclose(x[:, k], xr, rtol=1e-9, atol=1e-9 * np.abs(xr).max())


def test_hpcg_without_preconditioning(cuda):
    import torch
    h = Hpcg(16, 1, 27, 1)
    rng = np.random.default_rng(3)
    b = rng.standard_normal(h.n)
    it, res, x = h.solve(torch.from_numpy(b).cuda(), 300, 1e-9, precondition=False)
    h.close()
    ir, rr, xr = reference(16, 1, 27, 1, 1, 300, 1e-9, False, b)
    assert it[0] == ir
    np.testing.assert_allclose(x[:, 0], xr, rtol=1e-9, atol=1e-9 * np.abs(xr).max())


B200_DRIVER = ROOT / "_build" / "cpp" / "hpcg_driver_b200"


@pytest.mark.parametrize("nx,levels,colors", [(16, 1, 27), (32, 2, 27), (16, 1, 16)])
def test_alp_hpcg_call_takes_the_fused_path(cuda, nx, levels, colors):
    """grb::algorithms::hpcg called unchanged on a b200 system that
    build_hpcg_system made (tests/cpp/hpcg_driver.cpp compiled for b200): the
    overload recognises the system on the device and runs the fused device
    HPCG (ALPB_TRACE line), with the reference build's iteration count and x
    within 1e-9 relative; 16 colours exercise the two-pass colour step."""
    import os
    if not B200_DRIVER.exists():
        pytest.fail(f"{B200_DRIVER} is not built")
    rng = np.random.default_rng(100 + nx)
    b = rng.standard_normal(nx ** 3)
    with tempfile.TemporaryDirectory() as d:
        rhs = str(Path(d) / "b.bin")
        b.tofile(rhs)
        xo = Path(d) / "x.bin"
        r = subprocess.run([str(B200_DRIVER), *map(str, (nx, nx, nx, levels, colors, 1, 1, 200,
                                                         1e-9, 1)), rhs, str(xo)],
                           capture_output=True, text=True, timeout=600,
                           env=dict(os.environ, ALPB_TRACE="1"))
        assert r.returncode == 0, r.stdout + r.stderr
        assert "grb::b200: fused hpcg" in r.stderr, r.stderr
        out = dict(line.split() for line in r.stdout.splitlines() if len(line.split()) == 2)
        x = np.fromfile(xo)
    ir, rr, xr = reference(nx, levels, colors, 1, 1, 200, 1e-9, True, b)
    assert int(out["iterations"]) == ir
    np.testing.assert_allclose(x, xr, rtol=1e-9, atol=1e-9 * np.abs(xr).max())
    assert abs(float(out["residual"]) - rr) <= 1e-6 * rr
