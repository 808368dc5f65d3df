"""Device containers and synthetic inputs for tests and benchmarks.

torch supplies the device memory and the stream; every computation goes
through the C-ABI (``_abi``).  ``CRS`` mirrors a compressed storage of
include/graphblas/reference/compressed_storage.hpp: int64 offsets, uint32
indices (held in int32 tensors; all sizes here are < 2^31), optional values.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi as abi

TORCH_DTYPE = {abi.FP64: torch.float64, abi.INT32: torch.int32, abi.BOOL: torch.uint8,
               abi.INT64: torch.int64}
NP_DTYPE = {abi.FP64: np.float64, abi.INT32: np.int32, abi.BOOL: np.uint8, abi.INT64: np.int64}


def stream_ptr(stream: torch.cuda.Stream | None = None) -> C.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def ptr(t: torch.Tensor | None) -> C.c_void_p:
    return C.c_void_p(t.data_ptr() if t is not None else None)


@dataclass
class CRS:
    m: int
    n: int
    nnz: int
    offsets: torch.Tensor          # int64 [m+1]
    indices: torch.Tensor          # int32 [nnz] (uint32 semantics)
    values: torch.Tensor | None    # [nnz] of vtype, or None (pattern)
    vtype: int

    def p(self):
        return ptr(self.offsets), ptr(self.indices), ptr(self.values)

    def to_host(self):
        return (self.offsets.cpu().numpy(), self.indices.cpu().numpy().view(np.uint32),
                None if self.values is None else self.values.cpu().numpy())

    def nbytes(self) -> int:
        vs = 0 if self.values is None else self.values.element_size()
        return self.nnz * (4 + vs) + (self.m + 1) * 8


def _dev():
    return torch.device("cuda", torch.cuda.current_device())


def rmat(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 42,
         vtype: int = abi.FP64, lo: int = 1, hi: int = 100, value_seed: int | None = None) -> CRS:
    """Seeded R-MAT graph, duplicates merged (self loops kept), values keyed
    by (row, col): FP64 U[0,1), INT32 U{lo..hi}, BOOL all true, VOID none."""
    n = 1 << scale
    draws = edge_factor * n
    dev = _dev()
    keys = torch.empty(draws, dtype=torch.int64, device=dev)
    s = stream_ptr()
    abi.call("alpb_gen_rmat_keys", ptr(keys), draws, scale, a, b, c, seed, s)
    nu = C.c_int64(0)
    abi.call("alpb_keys_sort_unique", ptr(keys), draws, C.byref(nu), s)
    nnz = nu.value
    offsets = torch.empty(n + 1, dtype=torch.int64, device=dev)
    indices = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
    abi.call("alpb_crs_from_sorted_keys", ptr(keys), nnz, n, ptr(offsets), ptr(indices), s)
    del keys
    values = None
    if vtype != abi.VOID:
        values = torch.empty(max(nnz, 1), dtype=TORCH_DTYPE[vtype], device=dev)
        abi.call("alpb_gen_edge_values", ptr(values), vtype, ptr(offsets), ptr(indices), n, nnz,
                 seed + 1 if value_seed is None else value_seed, lo, hi, s)
    return CRS(n, n, nnz, offsets, indices, values, vtype)


def stencil(sizes, diag: float = 26.0, off: float = -1.0, ref_order: bool = True) -> CRS:
    """Box stencil of halo 1 (27-point in 3-D) with the reference builder's
    row order (ref_order: columns decreasing inside a row)."""
    dims = len(sizes)
    m = int(np.prod(sizes))
    dev = _dev()
    offsets = torch.empty(m + 1, dtype=torch.int64, device=dev)
    sz = (C.c_int64 * 4)(*sizes)
    nnz = C.c_int64(0)
    s = stream_ptr()
    abi.call("alpb_gen_stencil_crs", dims, sz, diag, off, int(ref_order), ptr(offsets), None, None,
             C.byref(nnz), s)
    indices = torch.empty(nnz.value, dtype=torch.int32, device=dev)
    values = torch.empty(nnz.value, dtype=torch.float64, device=dev)
    abi.call("alpb_gen_stencil_crs", dims, sz, diag, off, int(ref_order), ptr(offsets), ptr(indices),
             ptr(values), C.byref(nnz), s)
    return CRS(m, m, nnz.value, offsets, indices, values, abi.FP64)


def poisson2d(L: int, shift: float) -> CRS:
    m = L * L
    nnz = 5 * L * L - 4 * L
    dev = _dev()
    offsets = torch.empty(m + 1, dtype=torch.int64, device=dev)
    indices = torch.empty(nnz, dtype=torch.int32, device=dev)
    values = torch.empty(nnz, dtype=torch.float64, device=dev)
    abi.call("alpb_gen_poisson2d_crs", L, shift, ptr(offsets), ptr(indices), ptr(values), stream_ptr())
    return CRS(m, m, nnz, offsets, indices, values, abi.FP64)


def from_host(m: int, n: int, offsets, indices, values=None, vtype: int = abi.FP64) -> CRS:
    dev = _dev()
    o = torch.from_numpy(np.ascontiguousarray(offsets, dtype=np.int64)).to(dev)
    i = torch.from_numpy(np.ascontiguousarray(indices).astype(np.uint32).view(np.int32)).to(dev)
    v = None
    if values is not None and vtype != abi.VOID:
        v = torch.from_numpy(np.ascontiguousarray(values, dtype=NP_DTYPE[vtype])).to(dev)
    return CRS(m, n, int(len(indices)), o, i, v, vtype)


def transpose(A: CRS) -> CRS:
    dev = _dev()
    cp = torch.empty(A.n + 1, dtype=torch.int64, device=dev)
    ri = torch.empty(max(A.nnz, 1), dtype=torch.int32, device=dev)
    tv = None if A.values is None else torch.empty_like(A.values)
    abi.call("alpb_crs_transpose", A.m, A.n, A.nnz, ptr(A.offsets), ptr(A.indices), ptr(A.values),
             A.vtype, ptr(cp), ptr(ri), ptr(tv), stream_ptr())
    return CRS(A.n, A.m, A.nnz, cp, ri, tv, A.vtype)


def gen_values(n: int, vtype: int, seed: int, sid: int = 0, lo: int = 0, hi: int = 1000,
               p: float = 0.5) -> torch.Tensor:
    t = torch.empty(max(n, 1), dtype=TORCH_DTYPE[vtype], device=_dev())[:n]
    abi.call("alpb_gen_values", ptr(t), vtype, n, seed, sid, lo, hi, p, stream_ptr())
    return t


class Plan:
    """SpMV plan (schedule + merge-path tile table) for one storage."""

    def __init__(self, A: CRS, sched: int = abi.SCHED_AUTO, vector_width: int = 0):
        h = C.c_void_p()
        abi.call("alpb_spmv_plan_create", C.byref(h), A.m, A.nnz, ptr(A.offsets), sched,
                 vector_width, stream_ptr())
        self.h = h
        self.A = A

    def info(self):
        s, w, t = C.c_int(), C.c_int(), C.c_int64()
        abi.call("alpb_spmv_plan_info", self.h, C.byref(s), C.byref(w), C.byref(t))
        return s.value, w.value, t.value

    def autotune(self, ring: int, x: torch.Tensor, y_scratch: torch.Tensor):
        A = self.A
        abi.call("alpb_spmv_autotune", self.h, ring, A.n, ptr(A.indices), ptr(A.values), A.vtype,
                 ptr(x), ptr(y_scratch), stream_ptr())

    def close(self):
        if self.h:
            abi.lib().alpb_spmv_plan_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mxv(ring: int, A: CRS, u: torch.Tensor, v: torch.Tensor, *, descr: int = 0, form: int = 2,
        u_assigned: torch.Tensor | None = None, u_nnz: torch.Tensor | None = None,
        u_mask=None, u_mask_assigned=None, u_mask_type: int = abi.BOOL, u_mask_count: int = -1,
        v_assigned: torch.Tensor | None = None, v_count: int | None = None,
        v_mask=None, v_mask_assigned=None, v_mask_type: int = abi.BOOL, v_mask_count: int = -1,
        plan: Plan | None = None, stream=None) -> None:
    """u (+)= A (x) v through alpb_mxv (A is the gather storage; form bit 1 =
    vector on the left, bit 2 = A is the matrix's CRS)."""
    if v_count is None:
        v_count = A.n if v_assigned is None else int(v_assigned.sum().item())
    abi.call("alpb_mxv", ring, descr, form, A.m, A.n, A.nnz, ptr(A.offsets), ptr(A.indices),
             ptr(A.values), A.vtype,
             ptr(u), ptr(u_assigned), ptr(u_nnz),
             ptr(u_mask), ptr(u_mask_assigned), u_mask_type, u_mask_count,
             ptr(v), ptr(v_assigned), v_count,
             ptr(v_mask), ptr(v_mask_assigned), v_mask_type, v_mask_count,
             plan.h if plan is not None else None, stream_ptr(stream))
