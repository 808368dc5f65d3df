"""TEST INFRASTRUCTURE ONLY: Python access to the checkers.

* ``Restatement`` -- the plain-C restatement (alp_oracle.c, _build/liboracle.so)
* ``Reference``   -- the compiled, unmodified ALP reference behind ref_shim.cpp
                     (_ref/libalp_ref_seq.so or _ref/libalp_ref_omp.so)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SEQ_SO = HERE / "_ref" / "libalp_ref_seq.so"
REF_OMP_SO = HERE / "_ref" / "libalp_ref_omp.so"

VOID, BOOL, INT32, FP64 = 0, 1, 2, 3
INT64 = 5  # holds the unsigned 64-bit values of rings 5 and 6
NP = {FP64: np.float64, INT32: np.int32, BOOL: np.uint8, INT64: np.uint64}
RING_TYPE = {0: FP64, 1: BOOL, 2: INT32, 3: FP64, 4: INT32, 5: INT64, 6: INT64, 7: FP64}
P = C.c_void_p


def _p(a):
    return None if a is None else a.ctypes.data_as(P)


def build():
    """Compile the restatement (and the reference shims when the reference
    sources are present) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", str(HERE), "-j8"], check=True)


class Restatement:
    def __init__(self):
        if not ORACLE_SO.exists():
            build()
        L = C.CDLL(str(ORACLE_SO))
        I64, U64, D, I32 = C.c_int64, C.c_uint64, C.c_double, C.c_int
        L.alpo_hash3.restype = U64
        L.alpo_hash3.argtypes = [U64, U64, U64]
        L.alpo_gen_values.argtypes = [P, I32, I64, U64, U64, C.c_int32, C.c_int32, D]
        L.alpo_rmat_keys.argtypes = [P, I64, I32, D, D, D, U64]
        L.alpo_sort_unique.restype = I64
        L.alpo_sort_unique.argtypes = [P, I64]
        L.alpo_crs_from_sorted_keys.argtypes = [P, I64, I64, P, P]
        L.alpo_edge_values.argtypes = [P, I32, P, P, I64, U64, C.c_int32, C.c_int32]
        L.alpo_stencil_coo.restype = I64
        L.alpo_stencil_coo.argtypes = [I32, P, D, D, P, P, P]
        L.alpo_coo_to_crs.argtypes = [I64, I64, P, P, P, I32, P, P, P]
        L.alpo_crs_transpose.argtypes = [I64, I64, P, P, P, I32, P, P, P]
        L.alpo_mxv.argtypes = [I32, C.c_uint32, I32, I64, I64, I64, P, P, P, I32,
                               P, P, P, P, P, I32, I64, P, P, I64, P, P, I32, I64]
        L.alpo_cg.argtypes = [I64, P, P, P, P, P, I64, D, P, P]
        L.alpo_pagerank.argtypes = [I64, P, P, P, P, P, P, P, I32, D, D, I64, P, P]
        L.alpo_ppr_forward.argtypes = [I64, P, P, P, I64, P, D, D, I64, I32, P, P, P]
        L.alpo_ppr_adjoint.argtypes = [I64, P, P, P, I64, P, P, D, D, I64, P, P, P]
        L.alpo_ppr_grad.argtypes = [I64, P, P, P, I64, P, P, D, P]
        self.L = L

    # --- generators (bit-identical to the device ones) ---
    def values(self, n, vtype, seed, sid=0, lo=0, hi=1000, p=0.5):
        out = np.empty(n, dtype=NP[vtype])
        self.L.alpo_gen_values(_p(out), vtype, n, seed, sid, lo, hi, p)
        return out

    def rmat(self, scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=42, vtype=FP64, lo=1,
             hi=100, value_seed=None):
        n = 1 << scale
        keys = np.empty(edge_factor * n, dtype=np.uint64)
        self.L.alpo_rmat_keys(_p(keys), keys.size, scale, a, b, c, seed)
        nnz = self.L.alpo_sort_unique(_p(keys), keys.size)
        rp = np.empty(n + 1, dtype=np.int64)
        col = np.empty(nnz, dtype=np.uint32)
        self.L.alpo_crs_from_sorted_keys(_p(keys), nnz, n, _p(rp), _p(col))
        vals = None
        if vtype != VOID:
            vals = np.empty(nnz, dtype=NP[vtype])
            self.L.alpo_edge_values(_p(vals), vtype, _p(rp), _p(col), n,
                                    seed + 1 if value_seed is None else value_seed, lo, hi)
        return rp, col, vals

    def stencil_coo(self, sizes, diag=26.0, off=-1.0):
        sz = np.asarray(list(sizes) + [0] * (4 - len(sizes)), dtype=np.int64)
        nnz = self.L.alpo_stencil_coo(len(sizes), _p(sz), diag, off, None, None, None)
        I = np.empty(nnz, dtype=np.uint32)
        J = np.empty(nnz, dtype=np.uint32)
        V = np.empty(nnz, dtype=np.float64)
        self.L.alpo_stencil_coo(len(sizes), _p(sz), diag, off, _p(I), _p(J), _p(V))
        return I, J, V

    def coo_to_crs(self, m, I, J, V, vtype):
        rp = np.empty(m + 1, dtype=np.int64)
        col = np.empty(len(I), dtype=np.uint32)
        vals = None if vtype == VOID else np.empty(len(I), dtype=NP[vtype])
        self.L.alpo_coo_to_crs(m, len(I), _p(np.ascontiguousarray(I, np.uint32)),
                               _p(np.ascontiguousarray(J, np.uint32)),
                               _p(None if V is None else np.ascontiguousarray(V, NP[vtype])),
                               vtype, _p(rp), _p(col), _p(vals))
        return rp, col, vals

    def transpose(self, m, n, rp, col, vals, vtype):
        cp = np.empty(n + 1, dtype=np.int64)
        row = np.empty(len(col), dtype=np.uint32)
        tv = None if vals is None else np.empty_like(vals)
        self.L.alpo_crs_transpose(m, n, _p(rp), _p(col), _p(vals), vtype, _p(cp), _p(row), _p(tv))
        return cp, row, tv

    # --- semantics ---
    def mxv(self, ring, descr, form, m_out, n_in, rp, col, vals, vtype, u, u_assigned=None,
            u_mask=None, u_mask_assigned=None, u_mask_type=BOOL, u_mask_count=-1,
            v=None, v_assigned=None, v_count=None, v_mask=None, v_mask_assigned=None,
            v_mask_type=BOOL, v_mask_count=-1):
        """In place on u / u_assigned; returns (rc, nnz(u))."""
        u_nnz = np.array([int(u_assigned.sum()) if u_assigned is not None else m_out],
                         dtype=np.int64)
        if v_count is None:
            v_count = n_in if v_assigned is None else int(v_assigned.sum())
        rc = self.L.alpo_mxv(ring, descr, form, m_out, n_in, len(col), _p(rp), _p(col), _p(vals),
                             vtype, _p(u), _p(u_assigned), _p(u_nnz), _p(u_mask),
                             _p(u_mask_assigned), u_mask_type, u_mask_count, _p(v), _p(v_assigned),
                             v_count, _p(v_mask), _p(v_mask_assigned), v_mask_type, v_mask_count)
        return rc, int(u_nnz[0])

    def cg(self, rp, col, vals, b, x0, max_iter, tol):
        n = len(rp) - 1
        x = np.array(x0, dtype=np.float64, copy=True)
        it = np.zeros(1, np.int64)
        res = np.zeros(1, np.float64)
        rc = self.L.alpo_cg(n, _p(rp), _p(col), _p(vals), _p(np.ascontiguousarray(b)), _p(x),
                            max_iter, tol, _p(it), _p(res))
        return rc, x, int(it[0]), float(res[0])

    def pagerank(self, rp, col, vals, cp, row, tvals, alpha=0.85, conv=1e-9, max_iter=1000,
                 pr0=None):
        n = len(rp) - 1
        pr = np.zeros(n) if pr0 is None else np.array(pr0, dtype=np.float64, copy=True)
        it = np.zeros(1, np.int64)
        res = np.zeros(1, np.float64)
        rc = self.L.alpo_pagerank(n, _p(rp), _p(col), _p(vals), _p(cp), _p(row), _p(tvals), _p(pr),
                                  int(pr0 is not None), alpha, conv, max_iter, _p(it), _p(res))
        return rc, pr, int(it[0]), float(res[0])

    # --- personalised PageRank (ppr_oracle.c: oracle/ppr.py in C, OpenMP) ---
    @staticmethod
    def _crs(rp, col, w):
        return (np.ascontiguousarray(rp, np.int64), np.ascontiguousarray(col, np.uint32),
                np.ascontiguousarray(w, np.float64))

    def ppr_forward(self, rp, col, w, seeds, alpha=0.85, conv=1e-9, max_iter=1000, x0=None):
        """Same contract as oracle.ppr.forward: (x [n, S], iterations, residuals)."""
        rp, col, w = self._crs(rp, col, w)
        n = len(rp) - 1
        seeds = np.ascontiguousarray(seeds, np.int64)
        S = len(seeds)
        x = np.empty((n, S)) if x0 is None else np.array(x0, np.float64, copy=True, order="C")
        it = np.zeros(S, np.int64)
        res = np.zeros(S)
        rc = self.L.alpo_ppr_forward(n, _p(rp), _p(col), _p(w), S, _p(seeds), alpha, conv,
                                     max_iter, int(x0 is not None), _p(x), _p(it), _p(res))
        assert rc == 0, rc
        return x, it, res

    def ppr_adjoint(self, rp, col, w, seeds, g, alpha=0.85, conv=1e-9, max_iter=1000):
        """Same contract as oracle.ppr.adjoint: (lambda [n, S], iterations, residuals)."""
        rp, col, w = self._crs(rp, col, w)
        n = len(rp) - 1
        seeds = np.ascontiguousarray(seeds, np.int64)
        S = len(seeds)
        g = np.ascontiguousarray(g, np.float64).reshape(n, S)
        lam = np.empty((n, S))
        it = np.zeros(S, np.int64)
        res = np.zeros(S)
        rc = self.L.alpo_ppr_adjoint(n, _p(rp), _p(col), _p(w), S, _p(seeds), _p(g), alpha, conv,
                                     max_iter, _p(lam), _p(it), _p(res))
        assert rc == 0, rc
        return lam, it, res

    def ppr_grad(self, rp, col, w, x, lam, alpha=0.85):
        """Same contract as oracle.ppr.grad_weights."""
        rp, col, w = self._crs(rp, col, w)
        n = len(rp) - 1
        x = np.ascontiguousarray(x, np.float64)
        lam = np.ascontiguousarray(lam, np.float64)
        S = x.shape[1]
        grad = np.empty(len(col))
        rc = self.L.alpo_ppr_grad(n, _p(rp), _p(col), _p(w), S, _p(x), _p(lam), alpha, _p(grad))
        assert rc == 0, rc
        return grad


class Reference:
    """The unmodified ALP reference (sequential or OpenMP backend)."""

    def __init__(self, omp: bool = False):
        so = REF_OMP_SO if omp else REF_SEQ_SO
        if not so.exists():
            raise FileNotFoundError(f"{so} is not built (needs the reference sources)")
        L = C.CDLL(str(so))
        I64, D, I32 = C.c_int64, C.c_double, C.c_int
        L.refw_threads.restype = I32
        L.refw_mxv.argtypes = [I32, C.c_uint32, I32, I64, I64, I64, P, P, P, P, P, P, P, I32, P, P,
                               P, P, I32, I32, P]
        L.refw_cg.argtypes = [I64, I64, P, P, P, P, P, I64, D, P, P, P]
        L.refw_pagerank.argtypes = [I64, I64, P, P, P, P, D, D, I64, P, P]
        L.refw_hpcg.argtypes = [I64, I64, I64, I64, I64, P, P, I64, D, P, P, P, P]
        self.L = L
        self.omp = omp

    def threads(self):
        return self.L.refw_threads()

    def mxv(self, ring, descr, vxm_form, m, n, I, J, V, u, u_assigned, v, v_assigned=None,
            u_mask=None, u_mask_assigned=None, v_mask=None, v_mask_assigned=None, reps=1):
        """u, u_assigned updated in place; returns (rc, ms per call)."""
        ms = np.zeros(1)
        ua = u_assigned if u_assigned is not None else np.ones(len(u), np.uint8)
        rc = self.L.refw_mxv(ring, descr, vxm_form, m, n, len(I),
                             _p(np.ascontiguousarray(I, np.uint32)),
                             _p(np.ascontiguousarray(J, np.uint32)), _p(V), _p(u), _p(ua),
                             _p(u_mask), _p(u_mask_assigned), int(u_mask is not None or
                                                                  u_mask_assigned is not None),
                             _p(v), _p(v_assigned), _p(v_mask), _p(v_mask_assigned),
                             int(v_mask is not None or v_mask_assigned is not None), reps, _p(ms))
        return rc, float(ms[0])

    def cg(self, n, I, J, V, b, x0, max_iter, tol):
        x = np.array(x0, dtype=np.float64, copy=True)
        it = np.zeros(1, np.int64)
        res = np.zeros(1)
        ms = np.zeros(1)
        rc = self.L.refw_cg(n, len(I), _p(np.ascontiguousarray(I, np.uint32)),
                            _p(np.ascontiguousarray(J, np.uint32)),
                            _p(np.ascontiguousarray(V, np.float64)), _p(np.ascontiguousarray(b)),
                            _p(x), max_iter, tol, _p(it), _p(res), _p(ms))
        return rc, x, int(it[0]), float(res[0]), float(ms[0])

    def pagerank(self, n, I, J, V, alpha=0.85, conv=1e-9, max_iter=1000):
        pr = np.zeros(n)
        it = np.zeros(1, np.int64)
        ms = np.zeros(1)
        rc = self.L.refw_pagerank(n, len(I), _p(np.ascontiguousarray(I, np.uint32)),
                                  _p(np.ascontiguousarray(J, np.uint32)),
                                  _p(np.ascontiguousarray(V, np.float64)), _p(pr), alpha, conv,
                                  max_iter, _p(it), _p(ms))
        return rc, pr, int(it[0]), float(ms[0])

    def hpcg(self, nx, levels, colors=27, b=None, max_iter=200, tol=1e-9):
        """grb::algorithms::hpcg on the nx^3 system; returns (rc, x, iterations,
        residual, ms of the solve, ms of the system build)."""
        n = nx ** 3
        x = np.zeros(n)
        it = np.zeros(1, np.int64)
        res = np.zeros(1)
        ms = np.zeros(1)
        bms = np.zeros(1)
        bb = None if b is None else np.ascontiguousarray(b, np.float64)
        rc = self.L.refw_hpcg(nx, nx, nx, levels, colors, _p(bb), _p(x), max_iter, tol, _p(it),
                              _p(res), _p(ms), _p(bms))
        return rc, x, int(it[0]), float(res[0]), float(ms[0]), float(bms[0])


def crs_to_coo(rp, col):
    """Row indices of each stored nonzero (CRS storage order)."""
    counts = np.diff(rp)
    return np.repeat(np.arange(len(rp) - 1, dtype=np.uint32), counts), np.asarray(col, np.uint32)
