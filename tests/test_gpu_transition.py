"""ALP's transition CG API (include/transition/solver.h) on the b200 backend:
ALP's own src/transition/solver.cpp compiled unchanged for b200
(_build/cpp/libalp_b200_solver.so) against the same source on the reference
backend (oracle/_ref/cpp/libalp_ref_solver.so), both driven from C by
tests/cpp/transition_driver.c.  Same return codes, iteration counts within 1,
solutions within 1e-10."""
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
B200 = ROOT / "_build" / "cpp" / "transition_driver_b200"
REF = ROOT / "oracle" / "_ref" / "cpp" / "transition_driver_ref"


def drive(exe, variant, pre, nx, tol, max_iter):
    if not exe.exists():
        pytest.fail(f"{exe} is not built (build() compiles it where the ALP sources exist)")
    with tempfile.TemporaryDirectory() as d:
        xo = Path(d) / "x.bin"
        r = subprocess.run([str(exe), variant, str(pre), str(nx), str(tol), str(max_iter), str(xo)],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        out = dict(line.split() for line in r.stdout.splitlines())
        return out, np.fromfile(xo)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["dii", "diz", "dzz"])
@pytest.mark.parametrize("pre", [0, 1], ids=["plain", "jacobi"])
@pytest.mark.parametrize("nx", [16, 32])
def test_transition_cg_matches_reference(cuda, variant, pre, nx):
    ob, xb = drive(B200, variant, pre, nx, 1e-10, 500)
    orf, xr = drive(REF, variant, pre, nx, 1e-10, 500)
    for k in ("rc_init", "rc_tol", "rc_max", "rc_pre", "rc_solve", "rc_iter", "rc_res",
              "rc_destroy"):
        assert ob[k] == orf[k] == "0", (k, ob[k], orf[k])
    assert abs(int(ob["iterations"]) - int(orf["iterations"])) <= 1
    np.testing.assert_allclose(xb, xr, rtol=0, atol=1e-10)
    assert np.abs(xb - 1).max() < 1e-8


def test_solver_library_exports_the_transition_api():
    """Symbols of the d-variants (no device work: loading only)."""
    import ctypes as C
    so = ROOT / "_build" / "cpp" / "libalp_b200_solver.so"
    if not so.exists():
        pytest.skip("libalp_b200_solver.so is built where the ALP sources exist")
    lib = C.CDLL(str(so))
    for v in ("dii", "diz", "dzz"):
        for f in ("init", "solve", "destroy", "get_residual", "get_iter_count", "set_tolerance",
                  "set_max_iter_count", "set_preconditioner", "get_preconditioner", "get_size",
                  "get_tolerance"):
            assert hasattr(lib, f"sparse_cg_{f}_{v}"), f"sparse_cg_{f}_{v}"
