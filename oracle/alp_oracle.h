/*
 * alp_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement, in plain C, of the ALP/GraphBLAS reference backend's hot
 * path (SpMV gather over a semiring, the counting-sort matrix build, CG,
 * simple PageRank) and of the seeded synthetic generators the B200 library
 * uses.  It is the checker of the parity tests: only tests/, the smoke entry
 * and bench.py's CPU-baseline leg may load it.  The product never calls it.
 *
 * Parity pin: the restatement is checked against the reference itself
 * (oracle/_ref, compiled from the reference sources by oracle/Makefile) and
 * against the known answers in the reference's own tests
 * (tests/smoke/hpcg.cpp, tests/unit/masked_mxv.cpp, sparse_mxv.cpp, ...),
 * by tests/test_oracle_pin.py.
 *
 * Type and ring codes are those of include/alp_b200.h.
 */
#ifndef ALP_ORACLE_H
#define ALP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

uint64_t alpo_hash3(uint64_t seed, uint64_t a, uint64_t b);
void alpo_gen_values(void *out, int type, int64_t n, uint64_t seed, uint64_t sid,
	int32_t lo, int32_t hi, double p);
void alpo_rmat_keys(uint64_t *keys, int64_t n, int scale, double a, double b, double c,
	uint64_t seed);
int64_t alpo_sort_unique(uint64_t *keys, int64_t n);
void alpo_crs_from_sorted_keys(const uint64_t *keys, int64_t nnz, int64_t m,
	int64_t *row_ptr, uint32_t *col);
void alpo_edge_values(void *vals, int type, const int64_t *row_ptr, const uint32_t *col,
	int64_t m, uint64_t seed, int32_t lo, int32_t hi);
int64_t alpo_stencil_coo(int dims, const int64_t *sizes, double diag, double off,
	uint32_t *I, uint32_t *J, double *V);
void alpo_coo_to_crs(int64_t m, int64_t nnz, const uint32_t *I, const uint32_t *J,
	const void *V, int type, int64_t *row_ptr, uint32_t *col, void *vals);
void alpo_crs_transpose(int64_t m, int64_t n, const int64_t *row_ptr, const uint32_t *col,
	const void *vals, int type, int64_t *col_ptr, uint32_t *row, void *tvals);
int alpo_mxv(int ring, uint32_t descr, int form, int64_t m_out, int64_t n_in,
	int64_t nnz, const int64_t *offsets, const uint32_t *indices, const void *values,
	int value_type, void *u, uint8_t *u_assigned, int64_t *u_nnz,
	const void *u_mask, const uint8_t *u_mask_assigned, int u_mask_type,
	int64_t u_mask_count, const void *v, const uint8_t *v_assigned, int64_t v_count,
	const void *v_mask, const uint8_t *v_mask_assigned, int v_mask_type,
	int64_t v_mask_count);
int alpo_cg(int64_t n, const int64_t *row_ptr, const uint32_t *col, const double *val,
	const double *b, double *x, int64_t max_iter, double tol, int64_t *iterations,
	double *residual);
int alpo_pagerank(int64_t n, const int64_t *crs_row_ptr, const uint32_t *crs_col,
	const double *crs_val, const int64_t *ccs_col_ptr, const uint32_t *ccs_row,
	const double *ccs_val, double *pr, int init_given, double alpha, double conv,
	int64_t max_iter, int64_t *iterations, double *residual);

/* ppr_oracle.c: the C form of oracle/ppr.py (row-major n x S vectors) */
int alpo_ppr_forward(int64_t n, const int64_t *rp, const uint32_t *col, const double *w,
	int64_t S, const int64_t *seeds, double alpha, double conv, int64_t max_iter, int x_given,
	double *x, int64_t *iters, double *res);
int alpo_ppr_adjoint(int64_t n, const int64_t *rp, const uint32_t *col, const double *w,
	int64_t S, const int64_t *seeds, const double *g, double alpha, double conv,
	int64_t max_iter, double *lam, int64_t *iters, double *res);
int alpo_ppr_grad(int64_t n, const int64_t *rp, const uint32_t *col, const double *w,
	int64_t S, const double *x, const double *lam, double alpha, double *grad);

#ifdef __cplusplus
}
#endif
#endif
