"""MatrixMarket ingest straight to the device (alpb_mm_read and the C++
extension buildMatrixUniqueFromFile) against ALP's own reader.

* alpb_mm_read returns the triples in the order ALP's iterator yields them
  (file order, 0-based, each off-diagonal entry of a symmetric file followed
  by its mirror; pattern entries 1), checked against a numpy reading of the
  same text, including a file large enough to be parsed by several threads;
  malformed and unsupported files are refused with their codes.
* tests/cpp/mm_driver.cpp, built for b200 and for the reference backend, reads
  general, symmetric, pattern and integer files through ALP's
  MatrixFileReader + buildMatrixUnique and, on b200, also through
  buildMatrixUniqueFromFile: every build yields the same matrix, entry for
  entry, and the same product y = A x (1e-12 relative).
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
B200 = ROOT / "_build" / "cpp" / "mm_driver_b200"
REF = ROOT / "oracle" / "_ref" / "cpp" / "mm_driver_ref"


def write_mtx(path, kind, symmetric, m, n, nz, seed):
    rng = np.random.default_rng(seed)
    k = np.unique(rng.integers(0, m, nz) * n + rng.integers(0, n, nz))
    I, J = k // n, k % n
    if symmetric:
        keep = I >= J
        I, J = I[keep], J[keep]
    perm = rng.permutation(len(I))
    I, J = I[perm], J[perm]
    V = rng.uniform(-1, 1, len(I)).round(8)
    if kind == "integer":
        V = np.round(V * 100)
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {kind} "
                f"{'symmetric' if symmetric else 'general'}\n% generated\n{m} {n} {len(I)}\n")
        for a, b, v in zip(I.tolist(), J.tolist(), V.tolist()):
            if kind == "pattern":
                f.write(f"{a + 1} {b + 1}\n")
            elif kind == "integer":
                f.write(f"{a + 1} {b + 1} {int(v)}\n")
            else:
                f.write(f"{a + 1} {b + 1} {v!r}\n")
    return I, J, (np.ones(len(I)) if kind == "pattern" else V)


def expected(I, J, V, symmetric):
    """ALP's iterator order: each entry, then its mirror if off-diagonal."""
    ei, ej, ev = [], [], []
    for a, b, v in zip(I.tolist(), J.tolist(), V.tolist()):
        ei.append(a), ej.append(b), ev.append(v)
        if symmetric and a != b:
            ei.append(b), ej.append(a), ev.append(v)
    return np.array(ei), np.array(ej), np.array(ev)


def mm_read(path, vtype):
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    m, n, nnz = C.c_int64(), C.c_int64(), C.c_int64()
    I, J, V = C.c_void_p(), C.c_void_p(), C.c_void_p()
    rc = abi.lib().alpb_mm_read(str(path).encode(), vtype, C.byref(m), C.byref(n), C.byref(nnz),
                                C.byref(I), C.byref(J), C.byref(V), dev.stream_ptr())
    if rc != 0:
        return rc, None
    k = nnz.value
    hi = np.empty(k, np.uint32)
    hj = np.empty(k, np.uint32)
    abi.call("alpb_memcpy_d2h", hi.ctypes.data_as(C.c_void_p), I, 4 * k, dev.stream_ptr())
    abi.call("alpb_memcpy_d2h", hj.ctypes.data_as(C.c_void_p), J, 4 * k, dev.stream_ptr())
    hv = None
    if V.value:
        dt = {3: np.float64, 2: np.int32, 1: np.uint8}[vtype]
        hv = np.empty(k, dt)
        abi.call("alpb_memcpy_d2h", hv.ctypes.data_as(C.c_void_p), V, hv.nbytes, dev.stream_ptr())
    torch.cuda.synchronize()
    for p in (I, J, V):
        abi.lib().alpb_free(p)
    return 0, (m.value, n.value, hi, hj, hv)


@pytest.mark.parametrize("kind,symmetric,vtype", [
    ("real", False, 3), ("real", True, 3), ("pattern", False, 3), ("pattern", True, 0),
    ("integer", True, 2), ("real", False, 1)])
def test_mm_read_order_and_values(cuda, tmp_path, kind, symmetric, vtype):
    f = tmp_path / "a.mtx"
    I, J, V = write_mtx(f, kind, symmetric, 500, 400 if not symmetric else 500, 4000, 11)
    rc, out = mm_read(f, vtype)
    assert rc == 0
    m, n, hi, hj, hv = out
    ei, ej, ev = expected(I, J, V, symmetric)
    assert (m, n) == (500, 400 if not symmetric else 500)
    np.testing.assert_array_equal(hi, ei)
    np.testing.assert_array_equal(hj, ej)
    if vtype == 0:
        assert hv is None
    elif vtype == 1:
        np.testing.assert_array_equal(hv, (ev != 0).astype(np.uint8))
    elif vtype == 2:
        np.testing.assert_array_equal(hv, ev.astype(np.int32))
    else:
        np.testing.assert_array_equal(hv, ev)


def test_mm_read_large_file_parsed_by_threads(cuda, tmp_path):
    """About 8 MB of text: split over every host thread, concatenated in order."""
    f = tmp_path / "big.mtx"
    I, J, V = write_mtx(f, "real", True, 60000, 60000, 600000, 12)
    assert f.stat().st_size > (1 << 22)
    rc, out = mm_read(f, 3)
    assert rc == 0
    _, _, hi, hj, hv = out
    ei, ej, ev = expected(I, J, V, True)
    np.testing.assert_array_equal(hi, ei)
    np.testing.assert_array_equal(hj, ej)
    np.testing.assert_array_equal(hv, ev)


def test_mm_read_refuses_bad_files(cuda, tmp_path):
    from alp_b200 import _abi as abi
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 0.5\n4 1 1.0\n")
    assert mm_read(bad, 3)[0] == abi.ILLEGAL                     # row index beyond m
    short = tmp_path / "short.mtx"
    short.write_text("%%MatrixMarket matrix coordinate real general\n3 3 3\n1 1 0.5\n")
    assert mm_read(short, 3)[0] == abi.ILLEGAL                   # fewer entries than announced
    cplx = tmp_path / "c.mtx"
    cplx.write_text("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n")
    assert mm_read(cplx, 3)[0] == abi.UNSUPPORTED
    assert mm_read(tmp_path / "missing.mtx", 3)[0] == abi.ILLEGAL


def parse(text):
    out = {}
    for line in text.splitlines():
        p = line.split()
        if len(p) == 3 and p[1] != "nnz":
            out[(p[0], int(p[1]))] = float(p[2])
        elif len(p) >= 2 and not line.startswith("Info"):
            out[(p[0], p[1] if len(p) == 3 else None)] = float(p[-1])
    return out


def same(a, b, rtol=1e-12):
    assert set(a) == set(b), sorted(set(a) ^ set(b))[:10]
    for k, va in a.items():
        vb = b[k]
        assert abs(va - vb) <= rtol * max(abs(va), abs(vb), 1e-300) or va == vb, (k, va, vb)


@pytest.mark.parametrize("kind,symmetric", [("real", False), ("real", True), ("pattern", False),
                                            ("integer", True)])
def test_file_ingest_matches_alp_reader(cuda, tmp_path, kind, symmetric):
    for exe in (B200, REF):
        if not exe.exists():
            pytest.fail(f"{exe} is not built (build() compiles it where the ALP sources exist)")
    f = tmp_path / "a.mtx"
    write_mtx(f, kind, symmetric, 700, 700, 6000, 13)
    env = dict(os.environ, OMP_NUM_THREADS="1")
    a = subprocess.run([str(REF), str(f), "0"], capture_output=True, text=True, timeout=300,
                       env=env)
    b = subprocess.run([str(B200), str(f), "1" if kind == "pattern" else "0"],
                       capture_output=True, text=True, timeout=300, env=env)
    assert a.returncode == 0, a.stderr[-2000:]
    assert b.returncode == 0, b.stderr[-2000:]
    ref = parse(a.stdout)
    assert ref[("A", "nnz")] > 0 and ref[("rc_reader", None)] == 0
    # ALP's reader on b200, and the device ingest on b200, each against the reference
    same(ref, parse(b.stdout))
    dev_out = {k: v for k, v in parse(b.stderr).items()
               if k[0] not in ("rc_file", "pattern_rc", "pattern_nnz")}
    assert parse(b.stderr)[("rc_file", None)] == 0
    same(ref, dev_out)
    if kind == "pattern":
        pb = parse(b.stderr)
        assert pb[("pattern_rc", None)] == 0 and pb[("pattern_nnz", None)] == ref[("A", "nnz")]
