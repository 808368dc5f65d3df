"""ctypes binding of include/alp_b200.h (the C-ABI of libalp_b200.so).

This is how Python reaches the CUDA kernels: plain pointers and sizes, the
same entry points a C or C++ caller binds.  Loading fails loudly when the
shared object is missing -- there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("ALPB_LIB", _HERE / "libalp_b200.so"))

# status codes (grb::RC numbering)
SUCCESS, PANIC, OUTOFMEM, MISMATCH, OVERLAP, OVERFLW, UNSUPPORTED, ILLEGAL, FAILED = range(9)
RC_NAMES = ["SUCCESS", "PANIC", "OUTOFMEM", "MISMATCH", "OVERLAP", "OVERFLW",
            "UNSUPPORTED", "ILLEGAL", "FAILED"]

# descriptors (grb::descriptors)
DESC_NONE, DESC_INVERT_MASK, DESC_TRANSPOSE_MATRIX = 0, 1, 2
DESC_STRUCTURAL, DESC_DENSE, DESC_ADD_IDENTITY, DESC_USE_INDEX = 8, 16, 32, 64
DESC_EXPLICIT_ZERO, DESC_SAFE_OVERLAP = 512, 1024

# types
VOID, BOOL, INT32, FP64, UINT32, INT64 = range(6)
# rings
RING_PLUS_TIMES_F64, RING_LOR_LAND_BOOL, RING_MIN_PLUS_I32 = 0, 1, 2
RING_PLUS_PATTERN_F64, RING_PLUS_TIMES_I32 = 3, 4
RING_PLUS_RIGHT_IF_U64, RING_MAX_LEFT_IF_U64, RING_TIMES_PLUS_F64 = 5, 6, 7
RING_TYPE = {0: FP64, 1: BOOL, 2: INT32, 3: FP64, 4: INT32, 5: INT64, 6: INT64, 7: FP64}
# schedules
SCHED_AUTO, SCHED_MERGE_PATH, SCHED_VECTOR = 0, 1, 2
# ops
OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_MIN, OP_MAX, OP_ABS_DIFF = range(7)
OP_LEFT_ASSIGN, OP_RIGHT_ASSIGN, OP_LOR, OP_LAND = 7, 8, 9, 10

P = C.c_void_p
I32 = C.c_int
I64 = C.c_int64
U64 = C.c_uint64
U32 = C.c_uint32
D = C.c_double
PI64 = C.POINTER(C.c_int64)
PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)

# name -> argtypes (all return int unless listed in _RESTYPE)
PROTOS: dict[str, list] = {
    "alpb_init": [I32],
    "alpb_finalize": [],
    "alpb_last_error": [],
    "alpb_version": [],
    "alpb_launch_count": [],
    "alpb_malloc": [C.POINTER(P), C.c_size_t],
    "alpb_free": [P],
    "alpb_malloc_managed": [C.POINTER(P), C.c_size_t],
    "alpb_prefetch": [P, C.c_size_t, I32, P],
    "alpb_memcpy_h2d": [P, P, C.c_size_t, P],
    "alpb_memcpy_d2h": [P, P, C.c_size_t, P],
    "alpb_memcpy_d2d": [P, P, C.c_size_t, P],
    "alpb_memset": [P, I32, C.c_size_t, P],
    "alpb_stream_sync": [P],
    "alpb_gen_hash_u64": [P, I64, U64, U64, P],
    "alpb_gen_values": [P, I32, I64, U64, U64, C.c_int32, C.c_int32, D, P],
    "alpb_gen_rmat_keys": [P, I64, I32, D, D, D, U64, P],
    "alpb_gen_edge_values": [P, I32, P, P, I64, I64, U64, C.c_int32, C.c_int32, P],
    "alpb_keys_sort_unique": [P, I64, PI64, P],
    "alpb_crs_from_sorted_keys": [P, I64, I64, P, P, P],
    "alpb_mm_read": [C.c_char_p, I32, PI64, PI64, PI64, C.POINTER(P), C.POINTER(P), C.POINTER(P), P],
    "alpb_coo_to_crs": [I64, I64, I64, P, P, P, I32, P, P, P, P],
    "alpb_crs_transpose": [I64, I64, I64, P, P, P, I32, P, P, P, P],
    "alpb_gen_stencil_crs": [I32, PI64, D, D, I32, P, P, P, PI64, P],
    "alpb_gen_poisson2d_crs": [I64, D, P, P, P, P],
    "alpb_gen_poisson2d_batch": [I64, P, P, P, P, I64, P, P, P, P],
    "alpb_gen_normal": [P, I64, U64, U64, P],
    "alpb_gen_sym_dd_values": [P, P, I64, U64, D, D, D, P, P],
    "alpb_spmv_plan_create": [C.POINTER(P), I64, I64, P, I32, I32, P],
    "alpb_spmv_plan_destroy": [P],
    "alpb_spmv_plan_hot": [P, I32, I64, P, I64, P],
    "alpb_spmv_plan_hot_info": [P, PI64, PD],
    "alpb_spmv_autotune": [P, I32, I64, P, P, I32, P, P, P],
    "alpb_spmv_plan_info": [P, PI, PI, PI64],
    "alpb_mxv": [I32, U32, I32, I64, I64, I64, P, P, P, I32,
                 P, P, P,
                 P, P, I32, I64,
                 P, P, I64,
                 P, P, I32, I64,
                 P, P],
    "alpb_mxv_dense_noalloc": [I32, I32, I64, I64, I64, P, P, P, I32, P, P, P],
    "alpb_hpcg_create": [C.POINTER(P), I64, I64, I64, D, D, I64, I64, I64, I32, P],
    "alpb_hpcg_destroy": [P],
    "alpb_hpcg_info": [P, PI64, PI64, PI64, PI],
    "alpb_hpcg_matrix": [P, I64, C.POINTER(P), C.POINTER(P), C.POINTER(P), PI64, PI64],
    "alpb_hpcg_solve": [P, P, P, I32, I64, I64, I64, D, P, P, P],
    "alpb_hpcg_match_level": [P, I64, I64, I64, P, P, P, P, P, I64, P, P, I64, P, P, P, P, P],
    "alpb_ppr_create": [C.POINTER(P), I64, I64, P, P, P, I32, P],
    "alpb_ppr_destroy": [P],
    "alpb_ppr_set_weights": [P, P, P],
    "alpb_ppr_solve": [P, P, D, D, I64, P, I32, P, P, P],
    "alpb_ppr_adjoint": [P, P, P, D, I64, P, P, P],
    "alpb_ppr_grad_weights": [P, P, P, P, P],
    "alpb_ppr_info": [P, PI64, PI64, PI64, PI64],
    "alpb_dot_f64": [PD, I32, I32, I64, P, P, P, P, P],
    "alpb_dot_f64_device": [P, I32, I32, I64, P, P, P],
    "alpb_set_scalar": [P, I32, I64, D, P, P, P],
    "alpb_ewise_apply_f64": [P, I32, I64, P, D, P, D, P],
    "alpb_ewise_muladd_f64": [P, I32, I32, I64, P, D, P, D, P],
    "alpb_foldl_f64": [P, I32, I64, P, D, P],
    "alpb_reduce_f64": [PD, I32, I64, P, P, P],
    "alpb_vec_op": [I32, I32, I32, D, I32, U32, I64, P, I32, P, P, P, P, I32, I32,
                    P, I32, P, D, P, I32, P, D, P],
    "alpb_vec_op_dom": [I32, I32, I32, U64, I32, U32, I32, I64, P, I32, P, P, P, P, I32, I32,
                        P, I32, P, U64, P, I32, P, U64, P],
    "alpb_vec_reduce_dom": [P, I32, U64, I32, U32, I32, I64, P, I32, P, P, I32, P, P, P, I32,
                            I32, P],
    "alpb_count_assigned": [P, I64, PI64, P],
    "alpb_vec_chain": [I32, I64, I32, P, P, I32, P, P, P],
    "alpb_vec_reduce": [PD, I32, D, I32, U32, I64, P, I32, P, P, I32, P, P, P, I32, I32, P],
    "alpb_cg_solve": [I64, P, P, P, P, P, I64, D, PI64, PD, P, P, P],
    "alpb_pagerank": [I64, P, P, P, P, P, P, P, I32, D, D, I64, PI64, PD, P],
    "alpb_pagerank_planned": [I64, P, P, P, P, P, P, P, I32, D, D, I64, PI64, PD, P, P, P],
    "alpb_sddmm": [P, I64, I64, P, P, P, P, D, P, P],
    "alpb_cg_adjoint": [I64, P, P, P, P, P, P, P, P, P, P, I64, D, PI64, PD, P, P, P],
    "alpb_cg_grad": [I64, P, P, P, P, P, P, P, P, P, P, P, P, I64, D, PD, PI64, PI64, P, P, P],
    "alpb_batched_cg_create": [C.POINTER(P), I64, I64, P, P, P, I64, P, P],
    "alpb_batched_cg_destroy": [P],
    "alpb_batched_cg_solve": [P, P, P, I64, D, P],
    "alpb_batched_cg_capture": [P, P, P, I64, D, P],
    "alpb_batched_cg_replay": [P, P],
    "alpb_batched_cg_results": [P, P, P, P, P],
}
_RESTYPE = {"alpb_last_error": C.c_char_p, "alpb_launch_count": C.c_int64}

VEC_SET, VEC_FOLDL, VEC_FOLDR, VEC_APPLY, VEC_MULADD, VEC_REDUCE = 0, 1, 2, 3, 4, 5


class VecStep(C.Structure):
    """struct alpb_vec_step of alp_b200.h (one step of alpb_vec_chain)."""
    _fields_ = [("kind", C.c_int32), ("op", C.c_int32), ("mul_op", C.c_int32),
                ("descr", C.c_uint32), ("z", C.c_int32), ("x", C.c_int32), ("y", C.c_int32),
                ("reserved", C.c_int32), ("alpha", C.c_uint64), ("beta", C.c_uint64),
                ("identity", C.c_uint64)]

_lib = None


class AlpError(RuntimeError):
    def __init__(self, rc: int, where: str, msg: str):
        self.rc = rc
        name = RC_NAMES[rc] if 0 <= rc < len(RC_NAMES) else str(rc)
        super().__init__(f"{where}: {name}: {msg}")


def lib() -> C.CDLL:
    """The loaded libalp_b200.so with every prototype of alp_b200.h set."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m alp_b200.build` "
                "(there is no CPU fallback)")
        h = C.CDLL(str(LIB_PATH), mode=C.RTLD_GLOBAL)
        for name, argtypes in PROTOS.items():
            fn = getattr(h, name, None)
            if fn is None:
                continue  # symbol presence is checked by the ABI test
            fn.argtypes = argtypes
            fn.restype = _RESTYPE.get(name, C.c_int)
        _lib = h
    return _lib


def last_error() -> str:
    m = lib().alpb_last_error()
    return m.decode() if m else ""


def check(rc: int, where: str = "alpb") -> int:
    """Raise AlpError for a non-SUCCESS status."""
    if rc != SUCCESS:
        raise AlpError(rc, where, last_error())
    return rc


def call(name: str, *args) -> None:
    """Call an entry point and raise on a non-SUCCESS status."""
    check(getattr(lib(), name)(*args), name)


def launches() -> int:
    return int(lib().alpb_launch_count())
