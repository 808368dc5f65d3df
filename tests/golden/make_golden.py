"""Generate the golden fixtures of tests/golden/ by running the UNMODIFIED ALP
reference (oracle/_ref/libalp_ref_{omp,seq}.so, compiled from the reference
sources by oracle/Makefile) on small seeded inputs.

    OMP_NUM_THREADS=4 python tests/golden/make_golden.py

Inputs come from the seeded generators of oracle/alp_oracle.c (the same
integer hash as the device generators); outputs are what grb::mxv / grb::vxm,
grb::algorithms::conjugate_gradient and grb::algorithms::simple_pagerank
return for them.  Each fixture stores inputs and outputs, so the tests need
neither the reference nor the generator to replay it.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle.oracle import BOOL, FP64, INT32, NP, RING_TYPE, Reference, Restatement, crs_to_coo  # noqa: E402

INVERT, TRANSPOSE, STRUCTURAL, DENSE = 1, 2, 8, 16
ADD_IDENTITY, USE_INDEX, EXPLICIT_ZERO = 32, 64, 512


def mxv_cases():
    """(name, ring, descr, vxm_form, sparse_u, sparse_v, u_mask, v_mask)"""
    cases = []
    for ring in (0, 1, 2, 3, 4):
        cases.append((f"r{ring}_dense_mxv", ring, 0, 0, False, False, False, False))
        cases.append((f"r{ring}_dense_vxm", ring, 0, 1, False, False, False, False))
    for ring in (0, 1, 2):
        for d, dn in ((0, "plain"), (INVERT, "invert"), (STRUCTURAL, "structural"),
                      (STRUCTURAL | INVERT, "structinv"), (EXPLICIT_ZERO, "explicitzero"),
                      (ADD_IDENTITY, "addidentity"), (TRANSPOSE, "transpose")):
            cases.append((f"r{ring}_{dn}_umask_sparse", ring, d, 0, True, True, True, False))
            cases.append((f"r{ring}_{dn}_vmask_sparse", ring, d, 1, True, True, False, True))
        cases.append((f"r{ring}_useindex", ring, USE_INDEX, 0, False, False, False, False))
        cases.append((f"r{ring}_dense_desc", ring, DENSE, 0, False, False, True, False))
    return cases


def make_mxv(R: Restatement, ref: Reference, omp: Reference, out: dict):
    """Outputs from the sequential reference backend.  `omp_differs` records
    where the OpenMP backend returns something else: its loop choice weighs
    the sequential scatter loop by the thread count
    (reference/blas2.hpp:1120-1129), so it takes the gather where the
    sequential backend scatters, and the two loops differ observably."""
    scale = 8
    for name, ring, descr, vxm_form, su, sv, um, vm in mxv_cases():
        t = RING_TYPE[ring]
        vt = FP64 if t == FP64 else t
        rp, col, vals = R.rmat(scale, edge_factor=6, seed=11 + ring, vtype=vt, lo=1, hi=100)
        n = len(rp) - 1
        I, J = crs_to_coo(rp, col)
        # shuffle the input order so the reference's in-row reversal matters
        perm = np.random.default_rng(5).permutation(len(I))
        I, J, V = I[perm], J[perm], vals[perm]
        v = R.values(n, t, 21, sid=1, lo=0, hi=1000)
        va = R.values(n, BOOL, 22, sid=2, p=0.6) if sv else None
        if t == INT32:
            u = R.values(n, INT32, 23, sid=3, lo=0, hi=5000)
        else:
            u = R.values(n, t, 23, sid=3, lo=0, hi=1)
        ua = R.values(n, BOOL, 24, sid=4, p=0.3) if su else None
        umask = R.values(n, BOOL, 25, sid=5, p=0.5) if um else None
        umask_a = R.values(n, BOOL, 26, sid=6, p=0.8) if um and su else None
        vmask = R.values(n, BOOL, 27, sid=7, p=0.5) if vm else None
        vmask_a = R.values(n, BOOL, 28, sid=8, p=0.8) if vm and sv else None
        uo = u.copy()
        uao = (ua.copy() if ua is not None else np.ones(n, np.uint8))
        rc, _ = ref.mxv(ring, descr, vxm_form, n, n, I, J, V, uo, uao, v, va, umask, umask_a,
                        vmask, vmask_a)
        if rc != 0:
            raise RuntimeError(f"reference returned {rc} for {name}")
        us = u.copy()
        uas = (ua.copy() if ua is not None else np.ones(n, np.uint8))
        omp.mxv(ring, descr, vxm_form, n, n, I, J, V, us, uas, v, va, umask, umask_a,
                vmask, vmask_a)
        omp_differs = int(not (np.array_equal(uas, uao) and
                               np.allclose(us[uas > 0], uo[uao > 0], rtol=1e-12)))
        out.setdefault(f"mat{ring}", dict(n=n, I=I, J=J, V=V))
        out[name] = dict(ring=ring, descr=descr, vxm_form=vxm_form, v=v,
                         va=va, u=u, ua=ua, umask=umask, umask_a=umask_a, vmask=vmask,
                         vmask_a=vmask_a, u_out=uo, ua_out=uao, omp_differs=omp_differs)


def save(cases: dict, path: Path):
    flat = {}
    for name, d in cases.items():
        for k, v in d.items():
            if v is None:
                continue
            flat[f"{name}/{k}"] = np.asarray(v)
    np.savez_compressed(path, **flat)


def main():
    R = Restatement()
    ref = Reference()
    omp = Reference(omp=True)
    mx = {}
    make_mxv(R, ref, omp, mx)
    print(f"cases where reference_omp ({omp.threads()} threads) differs:",
          [k for k, v in mx.items() if v.get("omp_differs")])
    save(mx, HERE / "mxv_rmat_s8.npz")

    # CG on the 27-point 16^3 stencil, b = A*1, x0 = 0, tol 1e-10 (the
    # configuration of the plain-CG workload at a smaller grid)
    I, J, V = R.stencil_coo((16, 16, 16), 26.0, -1.0)
    m = 16 ** 3
    rp, col, vv = R.coo_to_crs(m, I, J, V, FP64)
    b = np.zeros(m)
    R.mxv(0, 0, 0, m, m, rp, col, vv, FP64, b, v=np.ones(m))
    rc, x, it, res, _ = ref.cg(m, I, J, V, b, np.zeros(m), 500, 1e-10)
    assert rc == 0
    save({"cg": dict(I=I, J=J, V=V, b=b, x=x, iterations=it, residual=res)},
         HERE / "cg_27pt_16.npz")

    # simple_pagerank on an R-MAT scale-10 pattern with unit values
    rp, col, _ = R.rmat(10, edge_factor=8, seed=3, vtype=FP64)
    I, J = crs_to_coo(rp, col)
    V = np.ones(len(I))
    n = len(rp) - 1
    rc, pr, it, _ = ref.pagerank(n, I, J, V, 0.85, 1e-9, 1000)
    assert rc == 0, rc
    save({"pr": dict(I=I, J=J, V=V, n=n, pr=pr, iterations=it)}, HERE / "pagerank_rmat_s10.npz")
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
