"""Loading and replaying the golden fixtures of tests/golden/.

A golden mxv case holds the reference's inputs (COO in input order, vectors
with assigned flags, masks) and the reference's output.  `replay` rebuilds
the gather storage the way the reference does (counting sort, reverse input
order inside a row) and runs any implementation with the alpb_mxv signature.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
TRANSPOSE = 2
FP64, INT32, BOOL, INT64 = 3, 2, 1, 5
# ring code -> value type (include/alp_b200.h enum alpb_ring); the two
# unsigned 64-bit rings hold ALPB_INT64 storage
RING_TYPE = {0: FP64, 1: BOOL, 2: INT32, 3: FP64, 4: INT32, 5: INT64, 6: INT64, 7: FP64}


def load(name: str) -> dict:
    z = np.load(GOLDEN / name)
    out: dict = {}
    for key in z.files:
        case, field = key.split("/", 1)
        out.setdefault(case, {})[field] = z[key]
    return out


def mxv_cases() -> tuple[dict, dict]:
    allc = load("mxv_rmat_s8.npz")
    mats = {k: v for k, v in allc.items() if k.startswith("mat")}
    cases = {k: v for k, v in allc.items() if not k.startswith("mat")}
    return mats, cases


def gather_storage(R, mat: dict, ring: int, vxm_form: int, descr: int):
    """(offsets, indices, values, form, transposed) of the storage the
    reference gathers over for this call form; form bit 1 = vector on the
    left, bit 2 = the storage is the matrix's CRS."""
    n = int(mat["n"])
    t = RING_TYPE[ring]
    rp, col, vals = R.coo_to_crs(n, mat["I"], mat["J"], mat["V"], t)
    transposed = bool(vxm_form) ^ bool(descr & TRANSPOSE)
    if transposed:
        # CCS with the reference's in-column order: counting sort by column
        rp, col, vals = R.coo_to_crs(n, mat["J"], mat["I"], mat["V"], t)
    form = (1 if vxm_form else 0) | (0 if transposed else 2)
    return rp, col, vals, form, transposed


def vector_args(c: dict, n: int):
    u = c["u"].copy()
    ua = c["ua"].copy() if "ua" in c else None
    v = c["v"]
    va = c.get("va")
    um = c.get("umask")
    uma = c.get("umask_a")
    vm = c.get("vmask")
    vma = c.get("vmask_a")
    u_mask_count = -1 if um is None else (int(uma.sum()) if uma is not None else n)
    v_mask_count = -1 if vm is None else (int(vma.sum()) if vma is not None else n)
    v_count = int(va.sum()) if va is not None else n
    return u, ua, v, va, um, uma, u_mask_count, vm, vma, v_mask_count, v_count


def new_ring_case(R, ring: int, scale: int, seed: int):
    """R-MAT pattern with values of the ring's type: u64 values in {0, 1, 2}
    (a zero is a false condition of right_assign_if / left_assign_if), FP64
    values near 1 for the (times, plus) ring, whose row products must stay
    finite."""
    from oracle.oracle import VOID, crs_to_coo
    rp, col, _ = R.rmat(scale, edge_factor=8, seed=seed, vtype=VOID)
    n = len(rp) - 1
    I, J = crs_to_coo(rp, col)
    rng = np.random.default_rng(seed)
    if RING_TYPE[ring] == INT64:
        V = rng.integers(0, 3, len(I)).astype(np.uint64)
        v = rng.integers(0, 1000, n).astype(np.uint64)
        # small presets, so that the max ring's mxv form (products are A_ij) moves u too
        u0 = rng.integers(0, 1000 if ring == 5 else 2, n).astype(np.uint64)
    else:
        V = rng.uniform(-0.01, 0.01, len(I))
        v = rng.uniform(0.99, 1.01, n)
        u0 = rng.uniform(0.5, 1.5, n)
    return n, I, J, V, v, u0
