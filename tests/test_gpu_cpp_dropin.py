"""The C++ drop-in: ALP programs compiled unchanged against the b200 backend.

* ALP's own self-contained unit tests (tests/unit/*.cpp of the ALP tree),
  compiled against b200 by tests/cpp/Makefile, must print "Test OK".
* tests/cpp/alp_driver.cpp is compiled twice -- against ALP's reference
  backend (the checker, oracle/_ref/cpp) and against b200 (_build/cpp) -- and
  both run the same case files: mxv / vxm over three semirings with masks and
  descriptors, the BLAS1 primitives, conjugate_gradient and simple_pagerank.
  Their printed results must agree: bool and int exactly, FP64 within
  relative 1e-12 for single primitives and 1e-9 for the solvers, with equal
  iteration counts.

The binaries are built by __graft_entry__.build() (they need the ALP sources
and are not rebuilt on the GPU host); a missing binary fails the test.
"""
import os
import struct
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
B200_BIN = ROOT / "_build" / "cpp"
REF_BIN = ROOT / "oracle" / "_ref" / "cpp"
UNIT = ["masked_mxv", "sparse_mxv", "masked_vxm", "dot", "set", "eWiseMul", "muladd",
        "masked_muladd", "eWiseLambda", "ewiseapply", "adapterIterator", "add15d", "add15m",
        "buildVector", "clearMatrix", "copyAndAssignVectorIterator", "copyVector",
        "doubleAssign", "emptyVector", "equals", "id", "iteratorFilter", "moveMatrix",
        "moveVector", "mul15i", "mul15m", "stdMatrix", "stdVector", "swapVector",
        "vectorFromListConstructor", "vectorToMatrix", "vmx", "vmxa", "wait", "copyVoidMatrices",
        "eWiseMatrix"]


def _run(exe: Path, *args, timeout=300, env=None):
    if not exe.exists():
        pytest.fail(f"{exe} is not built (build() compiles it where the ALP sources exist)")
    env = dict(os.environ, OMP_NUM_THREADS="1", **(env or {}))
    return subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True,
                          timeout=timeout, env=env)


@pytest.mark.parametrize("name", UNIT)
def test_alp_unit_test_passes_on_b200(cuda, name):
    r = _run(B200_BIN / f"unit_{name}_b200")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Test OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]


def _ok(r):
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-3000:]
    assert "Test OK" in r.stdout and "Test FAILED" not in r.stdout, out[-3000:]


def write_unsymmetric_mtx(path, n=497, nnz=1727, seed=497):
    """A seeded n x n unsymmetric real matrix with the shape of the west0497
    file ALP's unit tests read (497 rows, about 1.7 k nonzeroes).  Values are
    positive, so the sums RBGaussSeidel checks to a few ULPs do not cancel."""
    rng = np.random.default_rng(seed)
    k = np.unique(rng.integers(0, n, nnz) * n + rng.integers(0, n, nnz))
    I, J = k // n, k % n
    V = rng.uniform(0.1, 1, len(k)).round(6)
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real general\n{n} {n} {len(k)}\n")
        f.writelines(f"{a + 1} {b + 1} {float(v)!r}\n" for a, b, v in zip(I, J, V))


@pytest.fixture(scope="module")
def west_like(tmp_path_factory):
    p = tmp_path_factory.mktemp("alp_unit") / "w497.mtx"
    write_unsymmetric_mtx(p)
    return p


def test_alp_build_matrix_unique_unit_test(cuda):
    """ALP's buildMatrixUnique: sequential and parallel ingestion of band and
    random matrices, checked nonzero by nonzero through the matrix iterator."""
    _ok(_run(B200_BIN / "unitu_buildMatrixUnique_b200", timeout=900))


def test_alp_matrix_iterator_unit_test(cuda):
    """ALP's matrixIterator: copy, move and i()/j()/v() of the matrix
    iterators of valued and pattern matrices against the input triples."""
    _ok(_run(B200_BIN / "unitu_matrixIterator_b200"))


@pytest.mark.parametrize("n", [10, 1000])
@pytest.mark.parametrize("case", [1, 2, 3, 4])
def test_alp_sparse_vxm_unit_test(cuda, n, case):
    """ALP's sparse_vxm as its unit-test script runs it (sizes 10 and 1000,
    test cases 1-4, one inner and one outer repetition)."""
    _ok(_run(B200_BIN / "unit_sparse_vxm_b200", n, case, 1, 1))


@pytest.mark.parametrize("case", [1, 2, 3, 4])
def test_alp_dense_spmv_unit_test(cuda, west_like, case):
    """ALP's dense_spmv cases Ax, A^T x, xA, xA^T on a matrix of west0497's shape."""
    _ok(_run(B200_BIN / "unit_dense_spmv_b200", west_like, "direct", case, 1, 1))


def test_alp_red_black_gauss_seidel_unit_test(cuda, west_like):
    """ALP's RBGaussSeidel: double-masked mxv / vxm with safe_overlap."""
    _ok(_run(B200_BIN / "unit_RBGaussSeidel_b200", west_like))


# ------------------------------------------------------------ differential --
def write_case(path, op, ring, descr, m, n, I, J, V, u=None, v=None, um=None, vm=None):
    with open(path, "wb") as f:
        f.write(struct.pack("<6q", op, ring, descr, m, n, len(I)))
        f.write(np.asarray(I, np.uint32).tobytes())
        f.write(np.asarray(J, np.uint32).tobytes())
        f.write(np.asarray(V, np.float64).tobytes())
        for arr in (u, v, um, vm):
            if arr is None:
                f.write(struct.pack("<q", 0))
                continue
            vals, flags = arr
            f.write(struct.pack("<q", len(vals)))
            f.write(np.asarray(vals, np.float64).tobytes())
            f.write(np.asarray(flags, np.uint8).tobytes())


def _value(text: str):
    """A printed result: a number compares with tolerance, anything else as text."""
    try:
        return float(text)
    except ValueError:
        return text


def parse(out: str) -> dict:
    res = {}
    for line in out.splitlines():
        parts = line.split()
        if len(parts) == 3 and parts[1] != "nnz":
            res[(parts[0], int(parts[1]))] = float(parts[2])
        elif len(parts) >= 2:
            res[(parts[0], parts[1] if len(parts) == 3 else None)] = _value(parts[-1])
    return res


def compare(case_file, rtol):
    a = _run(REF_BIN / "alp_driver_ref", case_file)
    b = _run(B200_BIN / "alp_driver_b200", case_file)
    assert a.returncode == 0, a.stdout[-1000:] + a.stderr[-1000:]
    assert b.returncode == 0, b.stdout[-1000:] + b.stderr[-1000:]
    ra, rb = parse(a.stdout), parse(b.stdout)
    assert set(ra) == set(rb), (sorted(set(ra) ^ set(rb))[:10], a.stdout[:500], b.stdout[:500])
    for k, va in ra.items():
        vb = rb[k]
        if isinstance(va, float) and isinstance(vb, float):
            assert abs(va - vb) <= rtol * max(abs(va), abs(vb), 1e-300) or va == vb, (k, va, vb)
        else:
            assert va == vb, (k, va, vb)


def _vec(R, n, seed, p_assigned, lo=0, hi=100, vtype=3):
    vals = R.values(n, vtype, seed, 1, lo, hi).astype(np.float64)
    flags = R.values(n, 1, seed + 1, 2, p=p_assigned) if p_assigned < 1 else np.ones(n, np.uint8)
    return vals, flags


@pytest.mark.parametrize("ring", [0, 1, 2])
@pytest.mark.parametrize("op", [0, 1], ids=["mxv", "vxm"])
@pytest.mark.parametrize("descr", range(8),
                         ids=["plain", "invert", "structural", "structinv", "addidentity",
                              "explicitzero", "transpose", "dense"])
@pytest.mark.parametrize("sparse", [False, True], ids=["dense", "sparse"])
def test_driver_spmv_matches_reference(cuda, oracle, ring, op, descr, sparse):
    from oracle.oracle import crs_to_coo
    if descr == 7 and sparse:
        pytest.skip("dense descriptor on sparse inputs is ILLEGAL on both (covered in the ABI tests)")
    t = {0: 3, 1: 1, 2: 2}[ring]
    rp, col, vals = oracle.rmat(8, edge_factor=6, seed=40 + ring, vtype=t, lo=1, hi=100)
    n = len(rp) - 1
    I, J = crs_to_coo(rp, col)
    perm = np.random.default_rng(ring).permutation(len(I))
    I, J, V = I[perm], J[perm], vals[perm].astype(np.float64)
    if ring == 1:
        u = (oracle.values(n, 1, 3, 1, p=0.3).astype(float), np.ones(n, np.uint8))
        v = (oracle.values(n, 1, 4, 1, p=0.5).astype(float), np.ones(n, np.uint8))
    else:
        u = _vec(oracle, n, 3, 1.0, 0, 5000, t)
        v = _vec(oracle, n, 5, 1.0, 0, 1000, t)
    um = (oracle.values(n, 1, 7, 1, p=0.5).astype(float), np.ones(n, np.uint8))
    vm = None
    if sparse:
        u = (u[0], oracle.values(n, 1, 9, 3, p=0.3))
        v = (v[0], oracle.values(n, 1, 10, 3, p=0.6))
        um = (um[0], oracle.values(n, 1, 11, 3, p=0.8))
        vm = (oracle.values(n, 1, 12, 1, p=0.5).astype(float), oracle.values(n, 1, 13, 3, p=0.8))
    with tempfile.TemporaryDirectory() as d:
        f = Path(d) / "case.bin"
        write_case(f, op, ring, descr, n, n, I, J, V, u, v, um, vm)
        compare(f, 1e-12)


@pytest.mark.parametrize("sparse", [False, True])
def test_driver_blas1_matches_reference(cuda, oracle, sparse):
    n = 5000
    u = _vec(oracle, n, 21, 0.6 if sparse else 1.0)
    v = _vec(oracle, n, 23, 0.5 if sparse else 1.0)
    m = (oracle.values(n, 1, 25, 1, p=0.5).astype(float),
         oracle.values(n, 1, 26, 2, p=0.7) if sparse else np.ones(n, np.uint8))
    with tempfile.TemporaryDirectory() as d:
        f = Path(d) / "case.bin"
        write_case(f, 4, 0, 0, 0, 0, [], [], [], u, v, m, None)
        compare(f, 1e-12)


def test_driver_cg_matches_reference(cuda, oracle):
    I, J, V = oracle.stencil_coo((12, 12, 12), 26.0, -1.0)
    m = 12 ** 3
    rp, col, vals = oracle.coo_to_crs(m, I, J, V, 3)
    b = np.zeros(m)
    oracle.mxv(0, 0, 2, m, m, rp, col, vals, 3, b, v=np.ones(m))
    with tempfile.TemporaryDirectory() as d:
        f = Path(d) / "case.bin"
        write_case(f, 2, 0, 0, m, m, I, J, V, (np.zeros(m), np.ones(m, np.uint8)),
                   (b, np.ones(m, np.uint8)))
        compare(f, 1e-9)


def test_driver_pagerank_matches_reference(cuda, oracle):
    from oracle.oracle import crs_to_coo
    rp, col, _ = oracle.rmat(11, edge_factor=8, seed=77, vtype=3)
    I, J = crs_to_coo(rp, col)
    n = len(rp) - 1
    with tempfile.TemporaryDirectory() as d:
        f = Path(d) / "case.bin"
        write_case(f, 3, 0, 0, n, n, I, J, np.ones(len(I)))
        compare(f, 1e-9)


def test_driver_matrix_set_capacity_matches_reference(cuda, oracle):
    """Matrix-to-matrix set under ALP's capacity contract, against the
    reference build: the default capacity is max(rows, columns); a source
    with more nonzeroes than the target's capacity returns ILLEGAL and clears
    the target (reference/io.hpp set_copy); the RESIZE phase reserves and
    the EXECUTE phase then copies; an empty source clears the target."""
    from oracle.oracle import crs_to_coo
    rp, col, vals = oracle.rmat(7, edge_factor=6, seed=91, vtype=3)
    I, J = crs_to_coo(rp, col)
    n = len(rp) - 1
    with tempfile.TemporaryDirectory() as d:
        f = Path(d) / "case.bin"
        write_case(f, 5, 0, 0, n, n, I, J, vals)
        compare(f, 0.0)
        r = _run(B200_BIN / "alp_driver_b200", f)
    out = parse(r.stdout)
    assert out[("rc_set_small", None)] == 7          # ILLEGAL
    assert out[("nnz_C_small", None)] == 0
    assert out[("rc_set", None)] == 0 and out[("C", "nnz")] == len(I)
    assert out[("nnz_C_empty", None)] == 0


# ------------------------------------------------------------------ HPCG --
def _hpcg_result(out: str):
    import re
    it = re.search(r"took (\d+) iterations to converge with residual ([0-9.eE+-]+)", out)
    norm = re.search(r"Residual norm: ([0-9.eE+-]+)", out)
    assert it and norm, out[-2000:]
    return int(it.group(1)), float(it.group(2)), float(norm.group(1))


@pytest.mark.parametrize("n", [50, 5000])
def test_driver_integer_blas1_bit_exact(cuda, n):
    """Integer level-1 primitives against the reference build, bit for bit:
    size_t values above 2^53 (dot over the (+, *) ring, folds under add, max
    and min, eWiseApply, foldl, eWiseMul, set of a value near 2^64) and int
    values near the ends of their range, whose sums and products overflow and
    must wrap as the reference's 32-bit arithmetic does (dot, fold,
    eWiseApply, eWiseMulAdd over the min-plus ring)."""
    with tempfile.TemporaryDirectory() as d:
        f = Path(d) / "case.bin"
        write_case(f, 6, 0, 0, n, 0, [], [], [])
        compare(f, 0.0)


def test_driver_solvers_take_the_fused_path(cuda, oracle):
    """ALP's conjugate_gradient and simple_pagerank, called unchanged on b200
    containers, run the fused device solvers (one launch per solve), as the
    ALPB_TRACE line shows; the results were compared above."""
    from oracle.oracle import crs_to_coo
    I, J, V = oracle.stencil_coo((10, 10, 10), 26.0, -1.0)
    m = 1000
    rp, col, vals = oracle.coo_to_crs(m, I, J, V, 3)
    b = np.zeros(m)
    oracle.mxv(0, 0, 2, m, m, rp, col, vals, 3, b, v=np.ones(m))
    rp2, col2, _ = oracle.rmat(9, edge_factor=8, seed=78, vtype=3)
    I2, J2 = crs_to_coo(rp2, col2)
    n2 = len(rp2) - 1
    env = dict(os.environ, ALPB_TRACE="1")
    with tempfile.TemporaryDirectory() as d:
        f = Path(d) / "cg.bin"
        write_case(f, 2, 0, 0, m, m, I, J, V, (np.zeros(m), np.ones(m, np.uint8)),
                   (b, np.ones(m, np.uint8)))
        r = subprocess.run([str(B200_BIN / "alp_driver_b200"), str(f)], capture_output=True,
                           text=True, timeout=300, env=env)
        assert r.returncode == 0 and "grb::b200: fused conjugate_gradient" in r.stderr, r.stderr
        f2 = Path(d) / "pr.bin"
        write_case(f2, 3, 0, 0, n2, n2, I2, J2, np.ones(len(I2)))
        r = subprocess.run([str(B200_BIN / "alp_driver_b200"), str(f2)], capture_output=True,
                           text=True, timeout=300, env=env)
        assert r.returncode == 0 and "grb::b200: fused simple_pagerank" in r.stderr, r.stderr


def test_hpcg_smoke_matches_reference(cuda):
    """ALP's HPCG smoke test (tests/smoke/hpcg.cpp: 16^3, multigrid V-cycle with
    red-black Gauss-Seidel smoothing, CG outer loop), compiled unchanged on
    b200 and on the reference backend: both print "Test OK", converge in the
    same number of iterations (within one), and reach ||x - 1|| < 4e-14."""
    args = ("--test-rep", 1, "--init-iter", 1)
    a = _run(REF_BIN / "smoke_hpcg_ref", *args)
    b = _run(B200_BIN / "smoke_hpcg_b200", *args)
    assert a.returncode == 0 and "Test OK" in a.stdout, a.stdout[-2000:] + a.stderr[-2000:]
    assert b.returncode == 0 and "Test OK" in b.stdout, b.stdout[-2000:] + b.stderr[-2000:]
    ia, _, na = _hpcg_result(a.stdout)
    ib, _, nb = _hpcg_result(b.stdout)
    assert abs(ia - ib) <= 1, (ia, ib)
    assert nb < 4e-14, nb
    # the unchanged program's hpcg call ran the fused device solver
    b = _run(B200_BIN / "smoke_hpcg_b200", *args, env={"ALPB_TRACE": "1"})
    assert "grb::b200: fused hpcg" in b.stderr, b.stderr[-2000:]
