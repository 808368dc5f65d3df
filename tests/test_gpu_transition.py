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


SB_B200 = ROOT / "_build" / "cpp" / "sparseblas_driver_b200"
SB_REF = ROOT / "oracle" / "_ref" / "cpp" / "sparseblas_driver_ref"


def drive_sparseblas(exe, m, n, seed):
    if not exe.exists():
        pytest.fail(f"{exe} is not built (build() compiles it where the ALP sources exist)")
    with tempfile.TemporaryDirectory() as d:
        yo = Path(d) / "y.bin"
        r = subprocess.run([str(exe), str(m), str(n), str(seed), str(yo)], capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        out = dict(line.split() for line in r.stdout.splitlines() if len(line.split()) == 2)
        y = np.fromfile(yo)
        return out, y[:m], y[m:2 * m], y[2 * m:2 * m + n]


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,seed", [(300, 200, 7), (1000, 1500, 3)])
def test_sparse_blas_dusmv_matches_reference(cuda, m, n, seed):
    """Matrix assembly by entries and by rows, y = alpha A x + y and
    y = alpha A^T z + w (alpha 1 and 2.5) through BLAS_dusmv.  The reference
    pre- and post-scales a transposed product's y over the row count; the
    driver's y buffer has room for that, so both builds see the same data."""
    ob, *yb = drive_sparseblas(SB_B200, m, n, seed)
    orf, *yr = drive_sparseblas(SB_REF, m, n, seed)
    for k in ("rc_insert", "rc_end", "rc_nz", "rc_mv1", "rc_mv2", "rc_mv3", "rc_destroy"):
        assert ob[k] == orf[k] == "0", (k, ob[k], orf[k])
    assert ob["stored"] == orf["stored"] == ob["nnz"]
    for a, b in zip(yb, yr):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-14)
