/*
 * alp_b200.h -- C-ABI of the B200 backend for the ALP/GraphBLAS hot path.
 *
 * Every entry point takes plain device pointers, sizes, small integer codes
 * and a cudaStream_t passed as `void *` (NULL = legacy default stream).  No
 * C++ or torch type appears in a signature, so C, C++ (the grb::b200
 * template backend under include/graphblas/b200/), ctypes and any other FFI
 * bind it the same way.
 *
 * Status: every function returns an `int` whose values are numerically equal
 * to grb::RC (reference: include/graphblas/rc.hpp:47-155), so the C++ backend
 * returns them unchanged.  On a non-SUCCESS return the output containers are
 * unchanged, except for ALPB_PANIC (the grb::RC contract of
 * include/graphblas/base/blas2.hpp:208-223).  alpb_last_error() returns a
 * thread-local human-readable message for the last failing call.
 *
 * Storage conventions (mirroring internal::Compressed_Storage,
 * include/graphblas/reference/compressed_storage.hpp:48-797):
 *   - offsets   int64[m+1]   (NonzeroIndexType = size_t in the reference)
 *   - indices   uint32[nnz]  (RowIndexType = ColIndexType = unsigned int,
 *                             include/graphblas/base/config.hpp:436-475)
 *   - values    D[nnz] or NULL for a pattern (void) matrix.
 *   A CCS is passed through the same arguments: (col_start, row_index, values)
 *   of the transposed orientation, exactly as the reference stores both.
 *
 * Vector conventions (mirroring Vector<D,reference> + Coordinates,
 * include/graphblas/reference/vector.hpp:280-289, coordinates.hpp:61-1500):
 *   - values    D[n]
 *   - assigned  uint8[n] (1 = entry present) or NULL for a dense vector
 *   - nnz       int64 device counter of assigned entries, updated by kernels
 *               that assign new entries (may be NULL iff assigned is NULL).
 */
#ifndef ALP_B200_H
#define ALP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALPB_API __attribute__((visibility("default")))

/* ---- status codes: identical numbering to grb::RC (rc.hpp:47-155) ---- */
enum alpb_status {
	ALPB_SUCCESS = 0,
	ALPB_PANIC = 1,
	ALPB_OUTOFMEM = 2,
	ALPB_MISMATCH = 3,
	ALPB_OVERLAP = 4,
	ALPB_OVERFLW = 5,
	ALPB_UNSUPPORTED = 6,
	ALPB_ILLEGAL = 7,
	ALPB_FAILED = 8
};

/* ---- descriptor bits: identical to grb::descriptors (descriptors.hpp:63-267) ---- */
#define ALPB_DESC_NONE             0u
#define ALPB_DESC_INVERT_MASK      1u
#define ALPB_DESC_TRANSPOSE_MATRIX 2u
#define ALPB_DESC_NO_DUPLICATES    4u
#define ALPB_DESC_STRUCTURAL       8u
#define ALPB_DESC_DENSE           16u
#define ALPB_DESC_ADD_IDENTITY    32u
#define ALPB_DESC_USE_INDEX       64u
#define ALPB_DESC_NO_CASTING     256u
#define ALPB_DESC_EXPLICIT_ZERO  512u
#define ALPB_DESC_SAFE_OVERLAP  1024u

/* ---- element type codes ---- */
enum alpb_type {
	ALPB_VOID = 0,   /* pattern: no value array                      */
	ALPB_BOOL = 1,   /* uint8 holding 0 or 1                          */
	ALPB_INT32 = 2,
	ALPB_FP64 = 3,
	ALPB_UINT32 = 4,
	ALPB_INT64 = 5,
	ALPB_UINT8 = 6,  /* unsigned char                                */
	ALPB_INT8 = 7,   /* char / signed char                           */
	ALPB_UINT64 = 8  /* size_t; also the unsigned 64-bit compute domain of
	                    alpb_vec_op_dom / alpb_vec_reduce_dom            */
};

/*
 * ---- semirings instantiated on the device ----
 * Each is an ALP grb::Semiring< add, mul, zero-identity, one-identity >:
 *   PLUS_TIMES_F64   <operators::add<double>, operators::mul<double>,
 *                     identities::zero, identities::one>       (ops.hpp:175,208)
 *   LOR_LAND_BOOL    <operators::logical_or<bool>, operators::logical_and<bool>,
 *                     identities::logical_false, identities::logical_true>
 *                                                             (ops.hpp:462,490)
 *   MIN_PLUS_I32     <operators::min<int>, operators::add<int>,
 *                     identities::infinity, identities::zero>  (ops.hpp:274,175)
 *   PLUS_PATTERN_F64 <operators::add<double>,
 *                     operators::left_assign_if<double,bool,double>,
 *                     identities::zero, identities::logical_true>
 *                     -- the out-degree ring of simple_pagerank.hpp:224-237
 *   PLUS_TIMES_I32   <operators::add<int>, operators::mul<int>, zero, one>
 *   PLUS_RIGHT_IF_U64 <operators::add<size_t>,
 *                     operators::right_assign_if<bool,size_t,size_t>,
 *                     identities::zero, identities::logical_true>
 *                     -- the degree ring of interfaces/pregel.hpp:381-386
 *   MAX_LEFT_IF_U64  <operators::max<size_t>,
 *                     operators::left_assign_if<size_t,bool,size_t>,
 *                     identities::negative_infinity, identities::logical_true>
 *                     -- the message ring of the Pregel interface
 *                     (pregel.hpp:714-720) under connected components
 *                     (pregel_connected_components.hpp:148-151)
 * The two U64 rings hold values as ALPB_INT64 storage, compared unsigned.
 *   TIMES_PLUS_F64   <operators::mul<double>, operators::add<double>,
 *                     identities::one, identities::zero> -- the switched ring
 *                     of ALP's tests/unit/vmxa.cpp
 * Any other semiring is not instantiated and returns ALPB_UNSUPPORTED.
 */
enum alpb_ring {
	ALPB_RING_PLUS_TIMES_F64 = 0,
	ALPB_RING_LOR_LAND_BOOL = 1,
	ALPB_RING_MIN_PLUS_I32 = 2,
	ALPB_RING_PLUS_PATTERN_F64 = 3,
	ALPB_RING_PLUS_TIMES_I32 = 4,
	ALPB_RING_PLUS_RIGHT_IF_U64 = 5,
	ALPB_RING_MAX_LEFT_IF_U64 = 6,
	ALPB_RING_TIMES_PLUS_F64 = 7
};

/* SpMV schedules (the autotuner chooses among them per sparsity profile) */
enum alpb_schedule {
	ALPB_SCHED_AUTO = 0,
	ALPB_SCHED_MERGE_PATH = 1,   /* nnz+rows balanced tiles, deterministic carries */
	ALPB_SCHED_VECTOR = 2        /* W lanes per row, W in {1,2,4,8,16,32}      */
};

typedef struct alpb_spmv_plan_s *alpb_spmv_plan;

/* ======================================================================
 * Runtime (replaces grb::init / grb::finalize,
 * src/graphblas/reference/init.cpp:45-113, include/graphblas/base/init.hpp)
 * ====================================================================== */
/* Makes `device` current and its context ready; the device's default
 * memory pool then keeps the stream-ordered scratch that entry points free
 * (its release threshold is raised), so that repeated calls reuse it. */
ALPB_API int alpb_init(int device);
ALPB_API int alpb_finalize(void);
ALPB_API const char *alpb_last_error(void);
ALPB_API int alpb_version(void);
/* Number of kernels this library has launched since load (all entry points). */
ALPB_API int64_t alpb_launch_count(void);

/* device memory for the container classes (reference: utils::AutoDeleter /
 * reference/alloc.hpp allocation modes); bytes are rounded up to 256 B. */
ALPB_API int alpb_malloc(void **ptr, size_t bytes);
ALPB_API int alpb_free(void *ptr);
/* managed (unified) memory for containers whose values the host also reads
 * (grb::Vector of the C++ backend: raw(), operator[], iterators); prefetch
 * moves the pages to the device (to_device != 0) or the host. */
ALPB_API int alpb_malloc_managed(void **ptr, size_t bytes);
ALPB_API int alpb_prefetch(const void *ptr, size_t bytes, int to_device, void *stream);
ALPB_API int alpb_memcpy_h2d(void *dst, const void *src, size_t bytes, void *stream);
ALPB_API int alpb_memcpy_d2h(void *dst, const void *src, size_t bytes, void *stream);
ALPB_API int alpb_memcpy_d2d(void *dst, const void *src, size_t bytes, void *stream);
ALPB_API int alpb_memset(void *dst, int byte, size_t bytes, void *stream);
ALPB_API int alpb_stream_sync(void *stream);

/* ======================================================================
 * Synthetic generators, seeded counter-based (same integer hash as the
 * oracle, so CPU and GPU produce identical inputs).
 * ====================================================================== */
/* 64-bit mix used by every generator: out[k] = hash(seed, stream, k). */
ALPB_API int alpb_gen_hash_u64(uint64_t *out, int64_t count, uint64_t seed,
	uint64_t stream_id, void *stream);
/* fill a value array from the hash: FP64 -> U[0,1); INT32 -> lo + h % (hi-lo+1);
 * BOOL -> 1 with probability p (p only used for BOOL). */
ALPB_API int alpb_gen_values(void *out, int type, int64_t count, uint64_t seed,
	uint64_t stream_id, int32_t lo, int32_t hi, double p, void *stream);
/* R-MAT edge keys ((uint64)row << 32 | col), 2^scale vertices, quadrant
 * probabilities a, b, c (d = 1-a-b-c); no deduplication. */
ALPB_API int alpb_gen_rmat_keys(uint64_t *keys, int64_t n_draws, int scale,
	double a, double b, double c, uint64_t seed, void *stream);
/* edge values keyed by (row, col): identical for the same edge whatever its
 * position; FP64 -> U[0,1), INT32 -> lo + h % (hi-lo+1). */
ALPB_API int alpb_gen_edge_values(void *values, int type, const int64_t *row_ptr,
	const uint32_t *col_idx, int64_t m, int64_t nnz, uint64_t seed,
	int32_t lo, int32_t hi, void *stream);

/* ======================================================================
 * Matrix construction (replaces Matrix<D,reference>::buildMatrixUnique,
 * include/graphblas/reference/matrix.hpp:1820-2030, on the device)
 * ====================================================================== */
/* Sort keys ascending and remove duplicates in place; *n_unique receives the
 * count (synchronises `stream`). */
ALPB_API int alpb_keys_sort_unique(uint64_t *keys, int64_t n, int64_t *n_unique,
	void *stream);
/* Row offsets and column indices from sorted unique keys. */
ALPB_API int alpb_crs_from_sorted_keys(const uint64_t *keys, int64_t nnz, int64_t m,
	int64_t *row_ptr, uint32_t *col_idx, void *stream);
/* General COO -> CRS with the reference's in-row order (reverse of input
 * order, matrix.hpp:1921-1930).  I, J uint32[nnz]; values of `type` or NULL. */
ALPB_API int alpb_coo_to_crs(int64_t m, int64_t n, int64_t nnz, const uint32_t *I,
	const uint32_t *J, const void *values, int type, int64_t *row_ptr,
	uint32_t *col_idx, void *out_values, void *stream);
/* A MatrixMarket coordinate file (real, integer or pattern; general or
 * symmetric) straight to the device, for buildMatrixUnique-style ingest
 * (replaces ALP's host-side grb::utils::MatrixFileReader and its nonzero
 * iterator, include/graphblas/utils/parser/matrixFileIterator.hpp, and
 * src/graphblas/utils/hpparser.c).  The text is parsed on the host by all
 * cores at once; *rows, *cols (uint32[*nnz]) and *values (*nnz values of
 * value_type: FP64, INT32, BOOL (nonzero = true), or VOID for none) are new
 * device allocations the caller releases with alpb_free.  Triples come in the
 * order ALP's iterator yields them: file order, 0-based, a symmetric file's
 * off-diagonal entries each followed by its mirror; a pattern file's values
 * are 1.  ALPB_ILLEGAL for a malformed file, ALPB_UNSUPPORTED for complex or
 * skew/Hermitian files. */
ALPB_API int alpb_mm_read(const char *path, int value_type, int64_t *m, int64_t *n,
	int64_t *nnz, uint32_t **rows, uint32_t **cols, void **values, void *stream);
/* CCS (= CRS of the transpose) from CRS; stable, so within a column entries
 * appear in increasing row order. */
ALPB_API int alpb_crs_transpose(int64_t m, int64_t n, int64_t nnz,
	const int64_t *row_ptr, const uint32_t *col_idx, const void *values, int type,
	int64_t *col_ptr, uint32_t *row_idx, void *t_values, void *stream);
/* n-dimensional box stencil of halo 1 (hpcg/ndim_matrix_builders.hpp:198-394,
 * build_ndims_system_matrix, hpcg/matrix_building_utils.hpp:61-110): rows in
 * natural order, dimension 0 fastest; diag value on i==j else off value.  With
 * ref_order != 0 the in-row order is that of the reference build (decreasing
 * column); else increasing.  Call with row_ptr only (col_idx = NULL) to get
 * *nnz first. */
ALPB_API int alpb_gen_stencil_crs(int dims, const int64_t *sizes, double diag,
	double off, int ref_order, int64_t *row_ptr, uint32_t *col_idx, double *values,
	int64_t *nnz, void *stream);
/* 2-D 5-point Poisson on an L x L grid (Dirichlet), diag 4+shift, off -1;
 * columns ascending in each row. */
ALPB_API int alpb_gen_poisson2d_crs(int64_t L, double shift, int64_t *row_ptr,
	uint32_t *col_idx, double *values, void *stream);
/* nseg such systems as one block-diagonal CRS: instance i has side L[i] and
 * shift shift[i] (device arrays), rows [seg_rows[i], seg_rows[i+1]) and
 * nonzeroes from seg_nnz[i] (device arrays the caller fills: prefix sums of
 * L^2 and 5L^2-4L).  row_ptr has seg_rows[nseg]+1 entries. */
ALPB_API int alpb_gen_poisson2d_batch(int64_t nseg, const int64_t *L, const double *shift,
	const int64_t *seg_rows, const int64_t *seg_nnz, int64_t total_rows, int64_t *row_ptr,
	uint32_t *col_idx, double *values, void *stream);
/* Symmetric strictly diagonally dominant values on a symmetric CRS pattern:
 * a_ij = a_ji = -U(lo, hi) keyed by the pair {i, j}, a_ii = factor * sum |a_ij|. */
ALPB_API int alpb_gen_sym_dd_values(const int64_t *row_ptr, const uint32_t *col_idx, int64_t m,
	uint64_t seed, double lo, double hi, double diag_factor, double *values, void *stream);
/* standard normal samples (Box-Muller on two hash draws per sample) */
ALPB_API int alpb_gen_normal(double *out, int64_t count, uint64_t seed, uint64_t stream_id,
	void *stream);

/* ======================================================================
 * SpMV (replaces internal::vxm_generic + vxm_inner_kernel_gather,
 * include/graphblas/reference/blas2.hpp:283-551, 835-1528, and the public
 * grb::mxv / grb::vxm overloads, blas2.hpp:1532-2230)
 * ====================================================================== */
/* Analyse a compressed storage (row lengths: mean, max, CV), choose a
 * schedule (sched = ALPB_SCHED_AUTO) and precompute its tile table. */
ALPB_API int alpb_spmv_plan_create(alpb_spmv_plan *plan, int64_t m, int64_t nnz,
	const int64_t *offsets, int sched, int vector_width, void *stream);
ALPB_API int alpb_spmv_plan_destroy(alpb_spmv_plan plan);
/* Time the candidate schedules on this matrix/ring and keep the fastest; on
 * the merge path of a large skewed matrix also try the hot-column cache at
 * two sizes (alpb_spmv_plan_hot) and keep it when it is faster. */
ALPB_API int alpb_spmv_autotune(alpb_spmv_plan plan, int ring, int64_t n,
	const uint32_t *indices, const void *values, int value_type, const void *x,
	void *y_scratch, void *stream);
/* The hot-column cache of the merge path, for power-law matrices (the
 * autotuner sets it up when it pays; this call sets it up by hand, or removes
 * it with slots = 0).  The `slots` most frequent columns of `indices` (the
 * storage's column indices, n columns, n < 2^31) get shared-memory slots:
 * each dense product gathers x at those columns once, one block per SM
 * copies them into shared memory, and their nonzeroes read x from there
 * (random 8-byte shared loads cost a few L1 wavefronts per warp instead of
 * one per lane).  Results are bit-identical to the merge path without it.
 * The plan keeps a marked copy of `indices` (4 bytes per nonzero) and uses
 * the cache only for products given that same index array.  slots <= a
 * per-ring maximum (shared memory: 8,192 for 8-byte types); ALPB_ILLEGAL
 * beyond it. */
ALPB_API int alpb_spmv_plan_hot(alpb_spmv_plan plan, int ring, int64_t n,
	const uint32_t *indices, int64_t slots, void *stream);
/* slots in use (0: no cache) and the share of the nonzeroes they cover. */
ALPB_API int alpb_spmv_plan_hot_info(alpb_spmv_plan plan, int64_t *slots, double *cover);
/* chosen schedule and vector width (for reporting). */
ALPB_API int alpb_spmv_plan_info(alpb_spmv_plan plan, int *sched, int *vector_width,
	int64_t *tiles);

/* `form` bits of alpb_mxv */
#define ALPB_FORM_LEFT 1  /* vector on the left: mul(v_i, A_ij) (vxm)            */
#define ALPB_FORM_ROWS 2  /* the gather storage is the matrix's CRS              */

/*
 * u = u (+) A (x) v over `ring`, gathering over the compressed storage
 * (offsets, indices, values) whose outer dimension is the output:
 *   mxv(u, A, v)          : pass A's CRS, form = ROWS         (mul(A_ij, v_j))
 *   vxm(u, v, A)          : pass A's CCS, form = LEFT         (mul(v_i, A_ij))
 *   mxv<transpose_matrix> : pass A's CCS, form = 0
 *   vxm<transpose_matrix> : pass A's CRS, form = LEFT | ROWS
 * m_out = length of u, n_in = length of v.  Masks: u_mask on the output,
 * v_mask on the input, evaluated as utils::interpretMask (utils.hpp:318-341)
 * under `descr` (structural / invert_mask).  mask values of mask_type
 * (BOOL/INT32/FP64/VOID).  Descriptor bits honoured: invert_mask, structural,
 * dense, add_identity, use_index, explicit_zero, safe_overlap.  The
 * transpose_matrix bit must already be resolved by the caller (choice of
 * storage and form), as the reference does at blas2.hpp:1848.
 * The reference's observable semantics depend on which loop it runs, and
 * alpb_mxv applies the same choice (the sequential backend's rule,
 * blas2.hpp:1108-1132, 1311-1334): when the scatter over the input's
 * nonzeroes is the shorter loop, add_identity reaches every processed input
 * index whatever the output mask and explicit_zero writes nothing
 * (blas2.hpp:617-745); on the CRS gather (form & ROWS) a non-inverted output
 * mask is read by structure, not by value (blas2.hpp:1256-1301).
 * Host-side entry counts (the Coordinates::nonzeroes() the reference reads on
 * the host) drive the trivial cases (blas2.hpp:1001-1037) and the dense
 * checks (blas2.hpp:950-971): v_count = nnz(v); u_mask_count = nnz(u_mask)
 * or -1 for "no output mask"; v_mask_count likewise for the input mask.
 * `plan` may be NULL (vector schedule, no scratch).
 */
ALPB_API int alpb_mxv(int ring, uint32_t descr, int form,
	int64_t m_out, int64_t n_in, int64_t nnz,
	const int64_t *offsets, const uint32_t *indices, const void *values,
	int value_type,
	void *u, uint8_t *u_assigned, int64_t *u_nnz,
	const void *u_mask, const uint8_t *u_mask_assigned, int u_mask_type,
	int64_t u_mask_count,
	const void *v, const uint8_t *v_assigned, int64_t v_count,
	const void *v_mask, const uint8_t *v_mask_assigned, int v_mask_type,
	int64_t v_mask_count,
	alpb_spmv_plan plan, void *stream);

/*
 * Allocation-free dense SpMV.  No counterpart exists in the reference.  It is
 * for callers that cannot allocate device memory at call time: a memory pool
 * that already owns the whole device, code running inside an allocator or a
 * stream callback, or a thread that must not meet cudaMalloc's implicit
 * device synchronisation.  It computes u = u (+) A (x) v for dense u and v,
 * without masks, under descriptor `none` -- the result alpb_mxv gives on the
 * merge-path schedule, with the same `ring`, `form` and storage conventions.
 * Its merge-path tables live in one fixed 7 MiB device array inside the
 * library (held by every GPU that loads it, until the process exits), so the
 * caller passes no plan and no scratch.  Limit: m_out + nnz <= 268,435,456
 * (131,072 tiles of 2048 merge items); larger inputs return ALPB_ILLEGAL with
 * an error message.  u and v may not share any byte (ALPB_OVERLAP).  The
 * first call on a device resolves the array's address (cudaGetSymbolAddress),
 * and so does the first call in a new context of that device (after
 * cudaDeviceReset), so make that first call before any stream capture.
 * Every call, from any thread or stream, shares the one array: calls that
 * overlap in time on one device race and give wrong results; serialise them.
 */
ALPB_API int alpb_mxv_dense_noalloc(int ring, int form, int64_t m_out, int64_t n_in,
	int64_t nnz, const int64_t *offsets, const uint32_t *indices, const void *values,
	int value_type, void *u, const void *v, void *stream);

/* ======================================================================
 * BLAS1 (replaces reference/blas1.hpp: dot 9262-9681, eWiseMul 8610-9172,
 * eWiseMulAdd 6347-6770, foldl/foldr 1069-2897, eWiseApply 2966-5343, set in
 * reference/io.hpp).  FP64 unless stated; dense vectors unless an assigned
 * array is passed.
 * ====================================================================== */
enum alpb_op {
	ALPB_OP_ADD = 0, ALPB_OP_SUB = 1, ALPB_OP_MUL = 2, ALPB_OP_DIV = 3,
	ALPB_OP_MIN = 4, ALPB_OP_MAX = 5, ALPB_OP_ABS_DIFF = 6,
	ALPB_OP_LEFT_ASSIGN = 7, ALPB_OP_RIGHT_ASSIGN = 8,
	ALPB_OP_LOR = 9, ALPB_OP_LAND = 10,
	/* operators::left_assign_if (base/internalops.hpp:485-570): a where b is
	 * true; where b is false the output is left as it was, so the term is
	 * skipped (dot, fold) or nothing is written (element-wise kinds). */
	ALPB_OP_LEFT_ASSIGN_IF = 11,
	/* operators::equal / not_equal (ops.hpp:375-430): 1 where a == b
	 * (a != b), else 0 */
	ALPB_OP_EQUAL = 12, ALPB_OP_NOT_EQUAL = 13,
	/* operators::less_than / leq / greater_than / geq (ops.hpp:707-820):
	 * 1 where a < b (a <= b, a > b, a >= b), else 0 */
	ALPB_OP_LESS = 14, ALPB_OP_LEQ = 15, ALPB_OP_GREATER = 16, ALPB_OP_GEQ = 17
};
/* *result = *result (+) sum_i x_i (*) y_i with (+) = add_op, (*) = mul_op,
 * over entries assigned in both; result is a HOST double (synchronises). */
ALPB_API int alpb_dot_f64(double *result, int add_op, int mul_op, int64_t n,
	const double *x, const uint8_t *x_assigned, const double *y,
	const uint8_t *y_assigned, void *stream);
/* same, result left on the device (no synchronisation). */
ALPB_API int alpb_dot_f64_device(double *d_result, int add_op, int mul_op, int64_t n,
	const double *x, const double *y, void *stream);
/* x[i] = value for all i (dense result); if assigned != NULL it is set to 1
 * and *nnz = n. */
ALPB_API int alpb_set_scalar(void *x, int type, int64_t n, double value,
	uint8_t *assigned, int64_t *nnz, void *stream);
/* z = alpha (*) x (+) y style elementwise: out[i] = op(a[i], b[i]) for dense
 * FP64 vectors; a or b may be NULL to use the scalar sa / sb instead. */
ALPB_API int alpb_ewise_apply_f64(double *out, int op, int64_t n, const double *a,
	double sa, const double *b, double sb, void *stream);
/* out[i] = out[i] (+) (a[i] (*) b[i]) (eWiseMulAdd / eWiseMul in-place accumulate);
 * a or b NULL -> scalar. */
ALPB_API int alpb_ewise_muladd_f64(double *out, int add_op, int mul_op, int64_t n,
	const double *a, double sa, const double *b, double sb, void *stream);
/* foldl: x[i] = x[i] op y[i] (y NULL -> scalar sy); foldr: y[i] = x op y[i]. */
ALPB_API int alpb_foldl_f64(double *x, int op, int64_t n, const double *y, double sy,
	void *stream);
/* Generic element-wise primitive with ALP's sparse semantics (the device side
 * of grb::set, the vector forms of grb::foldl / grb::foldr, grb::eWiseApply
 * and grb::eWiseMul / eWiseMulAdd; reference/blas1.hpp, reference/io.hpp).
 * Operands: z (in/out), x, y as (values, type, assigned flags or NULL when
 * dense); x == NULL or y == NULL means the scalar alpha or beta.  An optional
 * mask (masked != 0) restricts the indices, as utils::interpretMask reads it
 * under descr.  Kinds:
 *   SET    z_i = x_i wherever x_i exists (z_i = i under the use_index bit of
 *          descr, as reference/io.hpp setIndexOrValue)
 *   FOLDL  z_i = z_i op x_i where both exist; a monoid also folds into absent
 *          z_i from its identity
 *   FOLDR  z_i = x_i op z_i, likewise
 *   APPLY  z = x op y: an operator on the intersection, a monoid on the union
 *          (absent operand = identity); z's old entries are dropped
 *   MULADD z_i = z_i (op) (x_i (mul_op) y_i) where x_i and y_i exist
 * Values are computed in double and cast to the output type. */
#define ALPB_VEC_SET 0
#define ALPB_VEC_FOLDL 1
#define ALPB_VEC_FOLDR 2
#define ALPB_VEC_APPLY 3
#define ALPB_VEC_MULADD 4
ALPB_API int alpb_vec_op(int kind, int op, int monoid, double identity, int mul_op,
	uint32_t descr, int64_t n, void *z, int z_type, uint8_t *z_assigned, int64_t *z_nnz,
	const void *mask, const uint8_t *mask_assigned, int mask_type, int masked,
	const void *x, int x_type, const uint8_t *x_assigned, double alpha,
	const void *y, int y_type, const uint8_t *y_assigned, double beta, void *stream);
/* *result = *result (+) [(+)_i x_i (*) y_i] over the indices where x, y (y may
 * be NULL: a plain fold of x) and the mask are present; values of any type
 * code, computed in double; identity is the additive monoid's.  Covers
 * grb::dot and the vector-to-scalar grb::foldl / foldr (masked or not).
 * (alpb_vec_op and alpb_vec_reduce compute in double: the FP64 domain of the
 * two _dom forms below.) */
ALPB_API int alpb_vec_reduce(double *result, int add_op, double identity, int mul_op,
	uint32_t descr, int64_t n, const void *x, int x_type, const uint8_t *x_assigned,
	const void *y, int y_type, const uint8_t *y_assigned, const void *mask,
	const uint8_t *mask_assigned, int mask_type, int masked, void *stream);
/* The same two primitives computing in the operator's own domain: `domain` is
 * ALPB_FP64 (double), ALPB_INT64 (int64_t), ALPB_UINT64 (uint64_t), ALPB_INT32
 * (int32_t) or ALPB_UINT32 (uint32_t); the C++ backend passes the domain of
 * the operands' C++ types, as the reference's operators cast their operands
 * to theirs.  Integer domains compute exactly with two's-complement
 * wrap-around at their own width.  identity, alpha and beta hold the bits of
 * a value of the domain type in their low bytes (memcpy of a double, int64_t,
 * uint64_t, int32_t or uint32_t); *result of the reduction is a value of the
 * domain type (in: the scalar folded into; out: the result), folded on the
 * device. */
ALPB_API int alpb_vec_op_dom(int kind, int op, int monoid, uint64_t identity, int mul_op,
	uint32_t descr, int domain, int64_t n, void *z, int z_type, uint8_t *z_assigned,
	int64_t *z_nnz, const void *mask, const uint8_t *mask_assigned, int mask_type, int masked,
	const void *x, int x_type, const uint8_t *x_assigned, uint64_t alpha,
	const void *y, int y_type, const uint8_t *y_assigned, uint64_t beta, void *stream);
ALPB_API int alpb_vec_reduce_dom(void *result, int add_op, uint64_t identity, int mul_op,
	uint32_t descr, int domain, int64_t n, const void *x, int x_type,
	const uint8_t *x_assigned, const void *y, int y_type, const uint8_t *y_assigned,
	const void *mask, const uint8_t *mask_assigned, int mask_type, int masked, void *stream);

/* Several dense level-1 steps over the same n entries in ONE device pass
 * (the fusion of chains of grb::set / foldl / foldr / eWiseMul / eWiseMulAdd
 * calls that the C++ backend records, plus a closing grb::dot or fold to a
 * scalar).  No counterpart in the reference's C interface: its nonblocking
 * backend fuses such chains on the CPU (include/graphblas/nonblocking/).
 * values[s], types[s] (s < nslots <= ALPB_CHAIN_SLOTS): the dense vectors the
 * steps name by slot number; each is read from memory once (if a step reads
 * it before any step writes it) and written once (if a step writes it).  The
 * steps apply alpb_vec_op_dom's dense semantics in order, element by element,
 * in the given domain; every type must be the domain's own (FP64 for ALPB_FP64,
 * INT64/UINT64/INT32/UINT32 for theirs), so no value is rounded between steps.
 * A last step of kind ALPB_VEC_REDUCE folds x (*) y (y = -1: x alone) with op
 * into *result exactly as alpb_vec_reduce_dom does (same order: bit-identical).
 * left_assign_if is not accepted (it may leave entries unassigned). */
#define ALPB_VEC_REDUCE 5
#define ALPB_CHAIN_SLOTS 8
#define ALPB_CHAIN_STEPS 16
typedef struct alpb_vec_step {
	int32_t kind;      /* ALPB_VEC_SET, _FOLDL, _FOLDR, _MULADD, or ALPB_VEC_REDUCE (last) */
	int32_t op;        /* the operator (MULADD, REDUCE: the additive one); SET: unused */
	int32_t mul_op;    /* MULADD and REDUCE with y: the multiplicative operator */
	uint32_t descr;    /* SET: ALPB_DESC_USE_INDEX writes the index */
	int32_t z, x, y;   /* slots; x or y = -1: the scalar alpha or beta instead */
	int32_t reserved;
	uint64_t alpha, beta;  /* bits of domain values */
	uint64_t identity;     /* REDUCE: bits of the additive identity */
} alpb_vec_step;
ALPB_API int alpb_vec_chain(int domain, int64_t n, int nslots, void *const *values,
	const int *types, int nsteps, const alpb_vec_step *steps, void *result, void *stream);
/* number of assigned entries (synchronises). */
ALPB_API int alpb_count_assigned(const uint8_t *assigned, int64_t n, int64_t *count,
	void *stream);
/* reduce a dense vector to a host scalar: *result = *result op fold(x). */
ALPB_API int alpb_reduce_f64(double *result, int op, int64_t n, const double *x,
	const uint8_t *assigned, void *stream);

/* ======================================================================
 * Solvers
 * ====================================================================== */
/* Conjugate gradient with the numerics of
 * algorithms::preconditioned_conjugate_gradient (conjugate_gradient.hpp:
 * 191-483, unpreconditioned branch): relative tolerance tol*||b||, stops when
 * sqrt(r.r) < tol or after max_iter; *residual = r.r (not its root).  All
 * FP64.  Fused: two passes over HBM per iteration (SpMV + dot, then the
 * x/r/u updates + r.r), device-side scalars, no host sync per iteration.
 * x holds the initial guess on entry.  `work` is 4*n doubles of scratch
 * (16-byte aligned; otherwise, or when NULL, the solver allocates its own);
 * on return its first n doubles hold the final residual vector r.  Returns
 * ALPB_FAILED when not converged.  */
ALPB_API int alpb_cg_solve(int64_t n, const int64_t *row_ptr, const uint32_t *col_idx,
	const double *values, const double *b, double *x, int64_t max_iter, double tol,
	int64_t *iterations, double *residual, double *work, alpb_spmv_plan plan,
	void *stream);

/* Power-iteration PageRank with the numerics of algorithms::simple_pagerank
 * (simple_pagerank.hpp:146-533): pr_j <- alpha * sum_i L_ij pr_i / outdeg_i
 * + (alpha * dangling + 1 - alpha) / n, L1 residual, stop at residual <= conv.
 * Takes L's CCS (col_ptr, row_idx, values; values NULL = pattern of ones) and
 * the CRS offsets for the out-degrees.  pr holds the initial guess if
 * init_given != 0, else 1/n. */
ALPB_API int alpb_pagerank(int64_t n, const int64_t *crs_row_ptr,
	const uint32_t *crs_col_idx, const double *crs_values,
	const int64_t *ccs_col_ptr, const uint32_t *ccs_row_idx, const double *ccs_values,
	double *pr, int init_given, double alpha, double conv, int64_t max_iter,
	int64_t *iterations, double *residual, void *stream);

/* alpb_pagerank with caller-held state, so that repeated solves on one graph
 * skip the set-up: ccs_plan is a plan of the CCS offsets made by
 * alpb_spmv_plan_create (any schedule; the solver uses its merge-path tables),
 * or NULL; work is 3n doubles of device scratch, or NULL.  ALPB_MISMATCH when
 * the plan was made for other offsets.  (No counterpart in the reference: its
 * simple_pagerank keeps such state in the caller's vectors.) */
ALPB_API int alpb_pagerank_planned(int64_t n, const int64_t *crs_row_ptr,
	const uint32_t *crs_col_idx, const double *crs_values, const int64_t *ccs_col_ptr,
	const uint32_t *ccs_row_idx, const double *ccs_values, double *pr, int init_given,
	double alpha, double conv, int64_t max_iter, int64_t *iterations, double *residual,
	double *work, alpb_spmv_plan ccs_plan, void *stream);

/* ======================================================================
 * HPCG: algorithms::hpcg (hpcg/hpcg.hpp:97-223) with its multigrid V-cycle
 * (hpcg/multigrid_v_cycle.hpp:67-246) and multi-colour Gauss-Seidel smoother
 * (hpcg/red_black_gauss_seidel.hpp:55-123) on the device, for the system
 * build_hpcg_system makes (hpcg/system_building_utils.hpp:84-150).
 * ====================================================================== */
typedef struct alpb_hpcg_s *alpb_hpcg;
/* The 3-D 27-point box stencil of nx x ny x nz (diagonal `diag`, the other
 * 26 entries `off`, in the reference builder's in-row order) and its coarser
 * levels: each halves every dimension, while the smallest coarse dimension
 * stays >= min_size and at most max_levels are added; injection is the
 * coarsening; `colors` static colours (row index modulo colors).  nrhs right-
 * hand sides (1, 2, 4 or 8) are solved together. */
ALPB_API int alpb_hpcg_create(alpb_hpcg *h, int64_t nx, int64_t ny, int64_t nz, double diag,
	double off, int64_t colors, int64_t min_size, int64_t max_levels, int nrhs, void *stream);
ALPB_API int alpb_hpcg_destroy(alpb_hpcg h);
/* number of levels, finest rows and nonzeroes; fused_smoother = 1 when no two
 * neighbouring rows share a colour on any level (each colour step then
 * updates in place; otherwise it stores the products first). */
ALPB_API int alpb_hpcg_info(alpb_hpcg h, int64_t *levels, int64_t *n_finest,
	int64_t *nnz_finest, int *fused_smoother);
/* device storage of one level's matrix (level 0 is the system) */
ALPB_API int alpb_hpcg_matrix(alpb_hpcg h, int64_t level, const int64_t **offsets,
	const uint32_t **indices, const double **values, int64_t *n, int64_t *nnz);
/* b and x hold n * nrhs doubles, the nrhs values of a row side by side; x
 * holds the initial guesses.  Each right-hand side runs the reference loop:
 * stop after an iteration where iter >= max_iterations or
 * ||r|| / ||r_0|| <= tolerance.  iterations[k] and residuals[k] (||r||, not
 * squared) are host arrays of nrhs entries. */
ALPB_API int alpb_hpcg_solve(alpb_hpcg h, const double *b, double *x, int with_preconditioning,
	int64_t presmoother_steps, int64_t postsmoother_steps, int64_t max_iterations,
	double tolerance, int64_t *iterations, double *residuals, void *stream);
/* Whether a caller's multigrid level equals level `level` of this handle, so
 * that the caller's own HPCG data can be solved by this handle (the b200
 * overload of grb::algorithms::hpcg recognises build_hpcg_system's systems
 * this way; no counterpart in the reference).  Compared on the device: the
 * system matrix (n, nnz and the CRS arrays word for word), the diagonal
 * vector (every entry assigned and equal to `diag`; diagonal_flags NULL =
 * dense), the `colors` colour masks (host arrays of device pointers: mask c
 * assigned and true exactly at the rows i = c mod colors; a NULL flags entry =
 * dense) and, for level > 0, the coarsening matrix from the finer level
 * (coarse_nnz entries; row c holds one 1 at the injected fine row).
 * *matches = 1 when everything agrees, else 0. */
ALPB_API int alpb_hpcg_match_level(alpb_hpcg h, int64_t level, int64_t n, int64_t nnz,
	const int64_t *offsets, const uint32_t *indices, const double *values,
	const double *diagonal, const uint8_t *diagonal_flags, int64_t colors,
	const uint8_t *const *mask_values, const uint8_t *const *mask_flags, int64_t coarse_nnz,
	const int64_t *coarse_offsets, const uint32_t *coarse_indices,
	const double *coarse_values, int *matches, void *stream);

/* ======================================================================
 * Adjoint gradients of a CG solve (implicit function theorem; no iterate is
 * stored).  No counterpart exists in the reference: the reference checks
 * them by assembling -lambda_i x_j on the host after a reference CG on A^T.
 * ====================================================================== */
/* out[k] = alpha * lam[row(k)] * x[col(k)] over the stored pattern (CRS
 * order): the pattern-masked SDDMM.  plan may be NULL. */
ALPB_API int alpb_sddmm(alpb_spmv_plan plan, int64_t m, int64_t nnz, const int64_t *offsets,
	const uint32_t *indices, const double *lam, const double *x, double alpha, double *out,
	void *stream);
/* lambda = A^{-T} g by CG on A's CCS, then grad_values[k] = -lambda_i x_j on A's
 * CRS pattern (grad_values may be NULL).  dL/db = lambda. */
ALPB_API int alpb_cg_adjoint(int64_t n, const int64_t *row_ptr, const uint32_t *col_idx,
	const double *values, const int64_t *ccs_col_ptr, const uint32_t *ccs_row_idx,
	const double *ccs_values, const double *x, const double *g, double *lambda,
	double *grad_values, int64_t max_iter, double tol, int64_t *iterations, double *residual,
	alpb_spmv_plan plan_crs, alpb_spmv_plan plan_ccs, void *stream);
/* Loss L = 0.5 ||x - x_target||^2 of x = A^{-1} b: forward CG from x = 0, then
 * the adjoint; returns L, x, lambda = dL/db and dL/dA on the pattern.  work:
 * n + 1 doubles. */
ALPB_API int alpb_cg_grad(int64_t n, const int64_t *row_ptr, const uint32_t *col_idx,
	const double *values, const int64_t *ccs_col_ptr, const uint32_t *ccs_row_idx,
	const double *ccs_values, const double *b, const double *x_target, double *x,
	double *lambda, double *grad_values, double *work, int64_t max_iter, double tol,
	double *loss, int64_t *iterations_fwd, int64_t *iterations_adj,
	alpb_spmv_plan plan_crs, alpb_spmv_plan plan_ccs, void *stream);

/* ======================================================================
 * Personalised PageRank over a weighted graph and its adjoint (differentiable
 * PageRank).  Extends algorithms::simple_pagerank (simple_pagerank.hpp:146-533),
 * whose teleport is uniform and whose normalisation is the out-degree count,
 * to one-hot teleport vectors (seeds) and weighted out-degrees d_i =
 * sum_j w_ij; with unit weights the normalisation is the reference's.  No
 * counterpart of the seeds or of the adjoint exists in the reference.
 *
 * Per seed s (x_s row-major n x S, the S values of a row side by side):
 *   x_s = alpha M x_s + (alpha * dangling(x_s) + 1 - alpha) e_seed,
 *   M_ji = w_ij / d_i, dangling(x) = sum of x over rows with d_i = 0,
 * by simple_pagerank's power iteration (input pre-scaled by alpha / d_i, L1
 * residual, stop at residual <= conv; each seed stops on its own).
 * ====================================================================== */
typedef struct alpb_ppr_s *alpb_ppr;
/* The graph is n x n CRS (row i -> column j, weight w_ij >= 0), held by
 * reference: it must stay valid and unchanged while the handle lives.  nseeds
 * in [1, 128].  Builds the transpose and the chunk tables. */
ALPB_API int alpb_ppr_create(alpb_ppr *h, int64_t n, int64_t nnz, const int64_t *row_ptr,
	const uint32_t *col_idx, const double *weights, int nseeds, void *stream);
ALPB_API int alpb_ppr_destroy(alpb_ppr h);
/* New weights on the same pattern (held by reference, like the create call's).
 * ALPB_ILLEGAL when a weight is negative or not finite; the handle then keeps
 * its previous weights. */
ALPB_API int alpb_ppr_set_weights(alpb_ppr h, const double *weights, void *stream);
/* seeds: host array of nseeds rows.  x (device, n x nseeds) holds the initial
 * guesses if init_given != 0, else starts at 1/n.  iterations and residuals:
 * host arrays of nseeds (may be NULL).  ALPB_FAILED when a seed did not
 * reach conv within max_iter iterations (x still holds the last iterate). */
ALPB_API int alpb_ppr_solve(alpb_ppr h, const int64_t *seeds, double alpha, double conv,
	int64_t max_iter, double *x, int init_given, int64_t *iterations, double *residuals,
	void *stream);
/* Adjoint of the last solve's fixed point for dl_dx = dL/dx (n x nseeds):
 *   lambda_s = alpha M^T lambda_s + alpha [i dangling] lambda_s[seed_s] + dl_dx_s,
 * iterated from lambda = dl_dx with the same per-seed L1 stopping rule.
 * dL/d(teleport weight of seed s) = (1 - alpha) lambda_s[seed_s]. */
ALPB_API int alpb_ppr_adjoint(alpb_ppr h, const double *dl_dx, double *lambda, double conv,
	int64_t max_iter, int64_t *iterations, double *residuals, void *stream);
/* grad[k] = dL/dw_ij for every stored edge k = (i, j), CRS order:
 *   alpha / d_i * sum_s x_is (lambda_js - (M^T lambda_s)_i),  0 on dangling rows. */
ALPB_API int alpb_ppr_grad_weights(alpb_ppr h, const double *x, const double *lambda,
	double *grad, void *stream);
/* chunk counts of the two storages (CCS: forward gather; CRS: adjoint) and
 * how many rows span several chunks. */
ALPB_API int alpb_ppr_info(alpb_ppr h, int64_t *chunks_ccs, int64_t *multi_ccs,
	int64_t *chunks_crs, int64_t *multi_crs);

/* ======================================================================
 * Batched CG: many independent SPD systems of uneven size, stored as one
 * block-diagonal CRS (instance i owns rows [seg_rows[i], seg_rows[i+1])),
 * solved in ONE persistent cooperative launch with per-instance convergence
 * masks.  Each instance follows algorithms::conjugate_gradient
 * (conjugate_gradient.hpp:191-483) with its own relative tolerance
 * tol * ||b_i||.  No counterpart exists in the reference, which solves one
 * system per call; this replaces calling grb::algorithms::conjugate_gradient
 * once per instance.
 * ====================================================================== */
typedef struct alpb_batched_cg_s *alpb_batched_cg;
/* Plan the batch (tiles cut per instance) and reserve its work vectors. */
ALPB_API int alpb_batched_cg_create(alpb_batched_cg *h, int64_t n, int64_t nnz,
	const int64_t *row_ptr, const uint32_t *col_idx, const double *values, int64_t nseg,
	const int64_t *seg_rows, void *stream);
ALPB_API int alpb_batched_cg_destroy(alpb_batched_cg h);
/* One solve: x holds the initial guesses on entry (all instances). */
ALPB_API int alpb_batched_cg_solve(alpb_batched_cg h, const double *b, double *x,
	int64_t max_iter, double tol, void *stream);
/* Capture one solve on (b, x) into a CUDA graph, then replay it. */
ALPB_API int alpb_batched_cg_capture(alpb_batched_cg h, const double *b, double *x,
	int64_t max_iter, double tol, void *stream);
ALPB_API int alpb_batched_cg_replay(alpb_batched_cg h, void *stream);
/* Per-instance iterations, r.r and converged flags of the last solve
 * (synchronises); ALPB_FAILED if any instance did not converge. */
ALPB_API int alpb_batched_cg_results(alpb_batched_cg h, int64_t *iterations,
	double *residuals, int32_t *converged, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* ALP_B200_H */
