/*
 * alp_oracle.c -- TEST INFRASTRUCTURE ONLY (see alp_oracle.h).
 *
 * Plain-C restatement of the ALP reference backend's hot path.  Each function
 * names the reference lines (paths relative to the ALP source tree) whose
 * behaviour it restates.  Sequential and deliberately simple: it is the
 * checker, never the thing measured as the product.
 */
#include "alp_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* type / ring / descriptor codes of include/alp_b200.h */
enum { T_VOID = 0, T_BOOL = 1, T_INT32 = 2, T_FP64 = 3, T_UINT32 = 4, T_INT64 = 5 };
enum {
	R_PT_F64 = 0, R_LORLAND = 1, R_MINPLUS_I32 = 2, R_PATTERN_F64 = 3, R_PT_I32 = 4,
	/* add<size_t> with right_assign_if<bool,size_t,size_t>: the degree ring of
	 * interfaces/pregel.hpp:381-386 */
	R_PLUS_RIGHTIF_U64 = 5,
	/* max<size_t> with left_assign_if<size_t,bool,size_t>: Pregel's message ring
	 * (pregel.hpp:714-720) under connected components
	 * (pregel_connected_components.hpp:148-151) */
	R_MAX_LEFTIF_U64 = 6,
	/* mul<double> as the additive monoid (identity 1) with add<double> as the
	 * product (identity 0): the switched ring of tests/unit/vmxa.cpp:62-67 */
	R_TIMES_PLUS_F64 = 7
};
#define D_INVERT 1u
#define D_STRUCTURAL 8u
#define D_DENSE 16u
#define D_ADD_IDENTITY 32u
#define D_USE_INDEX 64u
#define D_EXPLICIT_ZERO 512u
#define D_SAFE_OVERLAP 1024u

/* ------------------------------------------------------------ hashing --
 * splitmix64 finaliser (Steele, Lea, Flood, OOPSLA 2014) composed into a
 * three-input counter hash; identical to the device generators. */
static uint64_t mix64(uint64_t z) {
	z += 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}
uint64_t alpo_hash3(uint64_t seed, uint64_t a, uint64_t b) {
	return mix64(mix64(seed ^ mix64(a)) + b * 0xD1B54A32D192ED03ull);
}
static double u01(uint64_t h) { return (double) (h >> 11) * (1.0 / 9007199254740992.0); }

void alpo_gen_values(void *out, int type, int64_t n, uint64_t seed, uint64_t sid, int32_t lo,
	int32_t hi, double p) {
	for (int64_t k = 0; k < n; ++k) {
		const uint64_t h = alpo_hash3(seed, sid, (uint64_t) k);
		if (type == T_FP64) ((double *) out)[k] = u01(h);
		else if (type == T_INT32)
			((int32_t *) out)[k] = lo + (int32_t) (h % (uint64_t) ((int64_t) hi - lo + 1));
		else if (type == T_BOOL) ((uint8_t *) out)[k] = u01(h) < p ? 1 : 0;
	}
}

static uint64_t threshold_u64(double p) {
	if (p <= 0.0) return 0;
	if (p >= 1.0) return ~(uint64_t) 0;
	return (uint64_t) (p * 18446744073709551616.0);
}

/* R-MAT: per level one hash draw picks the quadrant (a | b | c | d). */
void alpo_rmat_keys(uint64_t *keys, int64_t n, int scale, double a, double b, double c,
	uint64_t seed) {
	const uint64_t ta = threshold_u64(a), tab = threshold_u64(a + b), tabc = threshold_u64(a + b + c);
	for (int64_t e = 0; e < n; ++e) {
		uint64_t r = 0, cc = 0;
		for (int l = 0; l < scale; ++l) {
			const uint64_t h = alpo_hash3(seed, (uint64_t) e, (uint64_t) l);
			const uint64_t rb = h >= tab ? 1u : 0u;
			const uint64_t cb = ((h >= ta && h < tab) || h >= tabc) ? 1u : 0u;
			r = (r << 1) | rb;
			cc = (cc << 1) | cb;
		}
		keys[e] = (r << 32) | cc;
	}
}

static int cmp_u64(const void *a, const void *b) {
	const uint64_t x = *(const uint64_t *) a, y = *(const uint64_t *) b;
	return x < y ? -1 : (x > y ? 1 : 0);
}

int64_t alpo_sort_unique(uint64_t *keys, int64_t n) {
	if (n <= 0) return 0;
	qsort(keys, (size_t) n, sizeof(uint64_t), cmp_u64);
	int64_t w = 1;
	for (int64_t k = 1; k < n; ++k)
		if (keys[k] != keys[w - 1]) keys[w++] = keys[k];
	return w;
}

void alpo_crs_from_sorted_keys(const uint64_t *keys, int64_t nnz, int64_t m, int64_t *row_ptr,
	uint32_t *col) {
	int64_t k = 0;
	for (int64_t i = 0; i <= m; ++i) {
		while (k < nnz && (int64_t) (keys[k] >> 32) < i) ++k;
		row_ptr[i] = k;
	}
	for (k = 0; k < nnz; ++k) col[k] = (uint32_t) (keys[k] & 0xffffffffu);
}

void alpo_edge_values(void *vals, int type, const int64_t *row_ptr, const uint32_t *col, int64_t m,
	uint64_t seed, int32_t lo, int32_t hi) {
	for (int64_t i = 0; i < m; ++i)
		for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
			const uint64_t key = ((uint64_t) i << 32) | col[k];
			const uint64_t h = alpo_hash3(seed, key, 0x5eedull);
			if (type == T_FP64) ((double *) vals)[k] = u01(h);
			else if (type == T_INT32)
				((int32_t *) vals)[k] = lo + (int32_t) (h % (uint64_t) ((int64_t) hi - lo + 1));
			else if (type == T_BOOL) ((uint8_t *) vals)[k] = 1;
		}
}

/* Box stencil of halo 1 in the order of matrix_generator_iterator
 * (algorithms/hpcg/ndim_matrix_builders.hpp:198-394): rows ascending,
 * columns with dimension 0 fastest, diag on i == j.  Returns nnz; with
 * I == NULL only counts. */
int64_t alpo_stencil_coo(int dims, const int64_t *sizes, double diag, double off, uint32_t *I,
	uint32_t *J, double *V) {
	int64_t m = 1, nz = 0;
	for (int d = 0; d < dims; ++d) m *= sizes[d];
	for (int64_t i = 0; i < m; ++i) {
		int64_t lo[4], hi[4], cur[4], stride[4], r = i, st = 1;
		for (int d = 0; d < dims; ++d) {
			const int64_t c = r % sizes[d];
			r /= sizes[d];
			lo[d] = c > 0 ? c - 1 : 0;
			hi[d] = c + 1 < sizes[d] ? c + 1 : sizes[d] - 1;
			cur[d] = lo[d];
			stride[d] = st;
			st *= sizes[d];
		}
		for (;;) {
			int64_t j = 0;
			for (int d = 0; d < dims; ++d) j += cur[d] * stride[d];
			if (I) {
				I[nz] = (uint32_t) i;
				J[nz] = (uint32_t) j;
				V[nz] = j == i ? diag : off;
			}
			++nz;
			int d = 0;
			for (; d < dims; ++d) {
				if (cur[d] < hi[d]) { ++cur[d]; break; }
				cur[d] = lo[d];
			}
			if (d == dims) break;
		}
	}
	return nz;
}

static size_t tsize(int type) {
	switch (type) {
	case T_BOOL: return 1;
	case T_INT32: case T_UINT32: return 4;
	case T_FP64: case T_INT64: return 8;
	}
	return 0;
}

/* Counting sort of buildMatrixUniqueImplSeq (reference/matrix.hpp:1854-1951):
 * counts, inclusive prefix sums, then a decrementing fill, which stores each
 * row's nonzeroes in the reverse of their input order. */
void alpo_coo_to_crs(int64_t m, int64_t nnz, const uint32_t *I, const uint32_t *J, const void *V,
	int type, int64_t *row_ptr, uint32_t *col, void *vals) {
	const size_t vs = tsize(type);
	memset(row_ptr, 0, sizeof(int64_t) * (size_t) (m + 1));
	for (int64_t k = 0; k < nnz; ++k) ++row_ptr[I[k]];
	for (int64_t i = 1; i < m; ++i) row_ptr[i] += row_ptr[i - 1];
	row_ptr[m] = nnz;
	for (int64_t k = 0; k < nnz; ++k) {
		const int64_t pos = --row_ptr[I[k]];
		col[pos] = J[k];
		if (vs) memcpy((char *) vals + pos * vs, (const char *) V + k * vs, vs);
	}
}

/* CCS from CRS, rows ascending inside each column */
void alpo_crs_transpose(int64_t m, int64_t n, const int64_t *row_ptr, const uint32_t *col,
	const void *vals, int type, int64_t *col_ptr, uint32_t *row, void *tvals) {
	const size_t vs = tsize(type);
	memset(col_ptr, 0, sizeof(int64_t) * (size_t) (n + 1));
	for (int64_t k = 0; k < row_ptr[m]; ++k) ++col_ptr[col[k] + 1];
	for (int64_t j = 0; j < n; ++j) col_ptr[j + 1] += col_ptr[j];
	int64_t *fill = (int64_t *) malloc(sizeof(int64_t) * (size_t) (n + 1));
	memcpy(fill, col_ptr, sizeof(int64_t) * (size_t) (n + 1));
	for (int64_t i = 0; i < m; ++i)
		for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
			const int64_t p = fill[col[k]]++;
			row[p] = (uint32_t) i;
			if (vs) memcpy((char *) tvals + p * vs, (const char *) vals + k * vs, vs);
		}
	free(fill);
}

/* ---------------------------------------------------------- semirings -- */
typedef union { double d; int32_t i; uint8_t b; uint64_t u; } val_t;

static val_t rzero(int ring) {
	val_t v;
	memset(&v, 0, sizeof(v));
	if (ring == R_MINPLUS_I32) v.i = INT_MAX;
	if (ring == R_TIMES_PLUS_F64) v.d = 1.0;
	return v;
}
static val_t rone(int ring) {
	val_t v;
	memset(&v, 0, sizeof(v));
	switch (ring) {
	case R_PT_F64: case R_PATTERN_F64: v.d = 1.0; break;
	case R_LORLAND: v.b = 1; break;
	case R_MINPLUS_I32: v.i = 0; break;
	case R_PT_I32: v.i = 1; break;
	case R_PLUS_RIGHTIF_U64: case R_MAX_LEFTIF_U64: v.u = 1; break;
	case R_TIMES_PLUS_F64: v.d = 0.0; break;
	}
	return v;
}
static val_t radd(int ring, val_t a, val_t b) {
	val_t v;
	memset(&v, 0, sizeof(v));
	switch (ring) {
	case R_PT_F64: case R_PATTERN_F64: v.d = a.d + b.d; break;
	case R_LORLAND: v.b = (a.b || b.b) ? 1 : 0; break;
	case R_MINPLUS_I32: v.i = a.i < b.i ? a.i : b.i; break;
	case R_PT_I32: v.i = (int32_t) ((uint32_t) a.i + (uint32_t) b.i); break;
	case R_PLUS_RIGHTIF_U64: v.u = a.u + b.u; break;
	case R_MAX_LEFTIF_U64: v.u = a.u > b.u ? a.u : b.u; break;
	case R_TIMES_PLUS_F64: v.d = a.d * b.d; break;
	}
	return v;
}
/* op(p, q): p is the left operand.  mxv applies op(A_ij, v_j), vxm applies
 * op(v_i, A_ij) (reference/blas2.hpp:124-160, leftOrRightHandedMul). */
static val_t rmul(int ring, val_t p, val_t q) {
	val_t v;
	memset(&v, 0, sizeof(v));
	switch (ring) {
	case R_PT_F64: v.d = p.d * q.d; break;
	case R_LORLAND: v.b = (p.b && q.b) ? 1 : 0; break;
	case R_MINPLUS_I32: v.i = (int32_t) ((uint32_t) p.i + (uint32_t) q.i); break;
	case R_PT_I32: v.i = (int32_t) ((uint32_t) p.i * (uint32_t) q.i); break;
	/* left_assign_if(p, q): q ? p : unchanged (= the additive identity the
	 * gather initialises the product with), base/internalops.hpp:485-520 */
	case R_PATTERN_F64: v.d = q.d != 0.0 ? p.d : 0.0; break;
	/* right_assign_if(p, q): p ? q : unchanged (base/internalops.hpp:580-660) */
	case R_PLUS_RIGHTIF_U64: v.u = p.u != 0 ? q.u : 0; break;
	case R_MAX_LEFTIF_U64: v.u = q.u != 0 ? p.u : 0; break;
	case R_TIMES_PLUS_F64: v.d = p.d + q.d; break;
	}
	return v;
}
static int requal(int ring, val_t a, val_t b) {
	switch (ring) {
	case R_PT_F64: case R_PATTERN_F64: case R_TIMES_PLUS_F64: return a.d == b.d;
	case R_LORLAND: return a.b == b.b;
	case R_PLUS_RIGHTIF_U64: case R_MAX_LEFTIF_U64: return a.u == b.u;
	default: return a.i == b.i;
	}
}
static int rtype(int ring) {
	switch (ring) {
	case R_PT_F64: case R_PATTERN_F64: case R_TIMES_PLUS_F64: return T_FP64;
	case R_LORLAND: return T_BOOL;
	case R_PLUS_RIGHTIF_U64: case R_MAX_LEFTIF_U64: return T_INT64;
	default: return T_INT32;
	}
}
static val_t load(int type, const void *p, int64_t k) {
	val_t v;
	memset(&v, 0, sizeof(v));
	if (type == T_FP64) v.d = ((const double *) p)[k];
	else if (type == T_INT32) v.i = ((const int32_t *) p)[k];
	else if (type == T_BOOL) v.b = ((const uint8_t *) p)[k] ? 1 : 0;
	else if (type == T_INT64) v.u = ((const uint64_t *) p)[k];
	return v;
}
static void store(int type, void *p, int64_t k, val_t v) {
	if (type == T_FP64) ((double *) p)[k] = v.d;
	else if (type == T_INT32) ((int32_t *) p)[k] = v.i;
	else if (type == T_BOOL) ((uint8_t *) p)[k] = v.b;
	else if (type == T_INT64) ((uint64_t *) p)[k] = v.u;
}
static val_t from_index(int ring, int64_t j) {
	val_t v;
	memset(&v, 0, sizeof(v));
	if (rtype(ring) == T_FP64) v.d = (double) j;
	else if (rtype(ring) == T_INT32) v.i = (int32_t) j;
	else if (rtype(ring) == T_INT64) v.u = (uint64_t) j;
	else v.b = j ? 1 : 0;
	return v;
}

/* utils::interpretMask (utils.hpp:318-341) */
static int mask_ok(const void *vals, const uint8_t *assigned, int type, uint32_t descr, int64_t i) {
	const int a = assigned ? assigned[i] != 0 : 1;
	int r;
	if ((descr & D_STRUCTURAL) || vals == NULL || type == T_VOID) r = a;
	else {
		r = 0;
		if (a) {
			if (type == T_BOOL) r = ((const uint8_t *) vals)[i] != 0;
			else if (type == T_INT32) r = ((const int32_t *) vals)[i] != 0;
			else if (type == T_FP64) r = ((const double *) vals)[i] != 0.0;
			else if (type == T_UINT32) r = ((const uint32_t *) vals)[i] != 0;
			else if (type == T_INT64) r = ((const int64_t *) vals)[i] != 0;
		}
	}
	return (descr & D_INVERT) ? !r : r;
}

/* vxm_generic + vxm_inner_kernel_gather / _scatter (reference/blas2.hpp:
 * 283-551, 617-745, 835-1528): trivial cases (:1001-1037), overlap checks
 * (:1040-1052), the loop choice of the sequential backend (:1108-1132,
 * :1311-1334), then per output index: output mask, immutable shortcut
 * (:351-357), identity (:360-385), the nonzero loop with input mask and input
 * sparsity (:398-497), and the accumulate into the output (:510-549).
 * Observable differences between the loops are kept: the CRS gather
 * (form & 2) under a non-inverted mask walks the mask's assigned set without
 * reading its values (:1256-1301; the CCS gather of :1470-1500 does read
 * them); the scatter reads the mask by value, adds the identity to
 * every processed input index regardless of the mask (:168-225, :678-691) and
 * never writes explicit zeroes.  The scatter's accumulation order (by input
 * index) is not kept: sums are formed per output index in storage order. */
int alpo_mxv(int ring, uint32_t descr, int form, int64_t m_out, int64_t n_in, int64_t nnz,
	const int64_t *offsets, const uint32_t *indices, const void *values, int value_type,
	void *u, uint8_t *u_assigned, int64_t *u_nnz, const void *u_mask,
	const uint8_t *u_mask_assigned, int u_mask_type, int64_t u_mask_count, const void *v,
	const uint8_t *v_assigned, int64_t v_count, const void *v_mask,
	const uint8_t *v_mask_assigned, int v_mask_type, int64_t v_mask_count) {
	const int T = rtype(ring);
	const int left = form & 1, rows = (form & 2) != 0;
	const int masked = u_mask_count >= 0, input_masked = v_mask_count >= 0;
	const int dense_hint = (descr & D_DENSE) != 0, invert = (descr & D_INVERT) != 0;
	if (value_type != T_VOID && value_type != T) return 6; /* UNSUPPORTED */
	if (dense_hint) {
		if (v_count < n_in) return 7;                                /* ILLEGAL */
		if (masked && u_mask_count < m_out) return 7;
		if (input_masked && v_mask_count < n_in) return 7;
	}
	if (v_count == 0 || n_in == 0 || m_out == 0 || nnz == 0 ||
		(masked && u_mask_count == 0 && !invert) || (input_masked && v_mask_count == 0 && !invert)) {
		if (descr & D_EXPLICIT_ZERO)
			for (int64_t i = 0; i < m_out; ++i)
				if (u_assigned && !u_assigned[i]) {
					store(T, u, i, rzero(ring));
					u_assigned[i] = 1;
					++*u_nnz;
				}
		return 0;
	}
	if (!(descr & D_SAFE_OVERLAP) && u == v) return 4;              /* OVERLAP */
	if (masked && u_mask != NULL && u == u_mask) return 4;
	const int64_t gather_loop = masked ? (m_out < 2 * u_mask_count ? m_out : 2 * u_mask_count) : m_out;
	int64_t sl = (input_masked && !invert) ? 2 * (v_mask_count < v_count ? v_mask_count : v_count)
										   : 2 * v_count;
	int64_t scatter_loop = dense_hint ? n_in : (n_in < sl ? n_in : sl);
	if (descr & 8192u) scatter_loop = gather_loop + 1; /* force_row_major */
	const int scatter = scatter_loop < gather_loop;
	const int by_structure = masked && !invert && !scatter && rows;
	for (int64_t i = 0; i < m_out; ++i) {
		int row_ok = 1;
		if (masked)
			row_ok = by_structure ? (u_mask_assigned == NULL || u_mask_assigned[i])
								  : mask_ok(u_mask, u_mask_assigned, u_mask_type, descr, i);
		const int id_row = (descr & D_ADD_IDENTITY) && (scatter || row_ok);
		if (!row_ok && !id_row) continue;
		const int u_has = u_assigned == NULL || u_assigned[i];
		const val_t yi = load(T, u, i);
		if (!scatter && ring == R_LORLAND && u_has && !requal(ring, yi, rzero(ring))) continue;
		val_t out = rzero(ring);
		int set = 0;
		if (id_row && i < n_in) {
			if ((!input_masked || mask_ok(v_mask, v_mask_assigned, v_mask_type, descr, i)) &&
				(dense_hint || v_assigned == NULL || v_assigned[i])) {
				const val_t xv = load(T, v, i);
				out = left ? rmul(ring, xv, rone(ring)) : rmul(ring, rone(ring), xv);
				set = 1;
			}
		}
		for (int64_t k = offsets[i]; row_ok && k < offsets[i + 1]; ++k) {
			const int64_t j = indices[k];
			if (input_masked && !mask_ok(v_mask, v_mask_assigned, v_mask_type, descr, j)) continue;
			if (!dense_hint && v_assigned != NULL && !v_assigned[j]) continue;
			const val_t a = value_type == T_VOID ? rone(ring) : load(T, values, k);
			const val_t xv = (descr & D_USE_INDEX) ? from_index(ring, j) : load(T, v, j);
			const val_t r = left ? rmul(ring, xv, a) : rmul(ring, a, xv);
			out = radd(ring, r, out); /* foldr( result, output ) */
			set = 1;
		}
		if (((descr & D_EXPLICIT_ZERO) && !scatter && row_ok) || set) {
			if (dense_hint || u_has) {
				store(T, u, i, radd(ring, yi, out)); /* foldl( y_i, output ) */
			} else {
				store(T, u, i, out);
			}
			if (!u_has && u_assigned) {
				u_assigned[i] = 1;
				++*u_nnz;
			}
		}
	}
	return 0;
}

/* ---------------------------------------------------------------- CG --
 * algorithms::preconditioned_conjugate_gradient, unpreconditioned branch
 * (algorithms/conjugate_gradient.hpp:191-483), operation for operation. */
static void crs_mxv_acc(int64_t n, const int64_t *rp, const uint32_t *col, const double *val,
	const double *x, double *y) {
	for (int64_t i = 0; i < n; ++i) {
		double out = 0.0;
		int set = 0;
		for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
			out = val[k] * x[col[k]] + out;
			set = 1;
		}
		if (set) y[i] = y[i] + out;
	}
}
static double dot(int64_t n, const double *a, const double *b) {
	double s = 0.0;
	for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
	return s;
}

int alpo_cg(int64_t n, const int64_t *rp, const uint32_t *col, const double *val, const double *b,
	double *x, int64_t max_iter, double tol, int64_t *iterations, double *residual) {
	if (tol <= 0 || max_iter == 0) return 7;
	double *r = (double *) calloc((size_t) n, 8), *u = (double *) calloc((size_t) n, 8),
		   *temp = (double *) calloc((size_t) n, 8);
	*iterations = 0;
	*residual = INFINITY;
	crs_mxv_acc(n, rp, col, val, x, temp);                 /* temp = A x        */
	for (int64_t i = 0; i < n; ++i) r[i] = (0.0 + b[i]) - temp[i];  /* r = b - temp */
	memcpy(u, r, (size_t) n * 8);                         /* u = r             */
	double sigma = dot(n, r, r), bnorm = dot(n, b, b), alpha, beta;
	tol *= sqrt(bnorm);
	int64_t iter = 0;
	double res = INFINITY;
	for (;;) {
		++iter;
		memset(temp, 0, (size_t) n * 8);
		crs_mxv_acc(n, rp, col, val, u, temp);             /* temp = A u        */
		beta = dot(n, temp, u);
		alpha = sigma / beta;
		for (int64_t i = 0; i < n; ++i) x[i] = x[i] + alpha * u[i];
		for (int64_t i = 0; i < n; ++i) temp[i] = alpha * temp[i];
		for (int64_t i = 0; i < n; ++i) r[i] = r[i] - temp[i];
		alpha = dot(n, r, r);
		res = alpha;
		if (sqrt(res) < tol || iter >= max_iter) break;
		beta = alpha;
		alpha = beta / sigma;
		for (int64_t i = 0; i < n; ++i) u[i] = alpha * u[i];
		for (int64_t i = 0; i < n; ++i) u[i] = r[i] + u[i];
		sigma = beta;
	}
	*iterations = iter;
	*residual = res;
	free(r);
	free(u);
	free(temp);
	return sqrt(res) >= tol ? 8 : 0; /* FAILED if not converged */
}

/* ---------------------------------------------------------- PageRank --
 * algorithms::simple_pagerank (algorithms/simple_pagerank.hpp:146-533), the
 * writableCaptured branch taken by the sequential reference backend. */
int alpo_pagerank(int64_t n, const int64_t *crs_rp, const uint32_t *crs_col, const double *crs_val,
	const int64_t *ccs_cp, const uint32_t *ccs_row, const double *ccs_val, double *pr,
	int init_given, double alpha, double conv, int64_t max_iter, int64_t *iterations,
	double *residual_out) {
	if (alpha <= 0 || alpha >= 1 || max_iter <= 0) return 7;
	double *row_sum = (double *) calloc((size_t) n, 8), *pr_next = (double *) calloc((size_t) n, 8),
		   *pr_nn = (double *) calloc((size_t) n, 8);
	if (!init_given)
		for (int64_t i = 0; i < n; ++i) pr[i] = 1.0 / (double) n;
	/* row sums under the pattern ring: count of nonzero-valued entries (:224-237) */
	for (int64_t i = 0; i < n; ++i) {
		double out = 0.0;
		for (int64_t k = crs_rp[i]; k < crs_rp[i + 1]; ++k) {
			const double a = crs_val ? crs_val[k] : 1.0;
			out = (a != 0.0 ? 1.0 : 0.0) + out;
		}
		row_sum[i] = 0.0 + out;
	}
	for (int64_t i = 0; i < n; ++i)
		if (row_sum[i] > 0.0) row_sum[i] = alpha / row_sum[i];      /* (:281-289) */
	int64_t iter = 0;
	double residual = 0.0;
	do {
		double dangling = 0.0;
		residual = 0.0;
		for (int64_t i = 0; i < n; ++i) {                             /* (:331-342) */
			if (row_sum[i] == 0.0) {
				dangling += pr[i];
				pr_next[i] = 0.0;
			} else {
				pr_next[i] = pr[i] * row_sum[i];
			}
		}
		dangling = (alpha * dangling + 1 - alpha) / (double) n;      /* (:390) */
		for (int64_t j = 0; j < n; ++j) {                             /* vxm, CCS gather */
			double out = 0.0;
			int set = 0;
			for (int64_t k = ccs_cp[j]; k < ccs_cp[j + 1]; ++k) {
				const double a = ccs_val ? ccs_val[k] : 1.0;
				out = pr_next[ccs_row[k]] * a + out;
				set = 1;
			}
			pr_nn[j] = set ? 0.0 + out : 0.0;
		}
		for (int64_t i = 0; i < n; ++i) {                             /* (:441-455) */
			const double old = pr[i];
			pr[i] = pr_nn[i] + dangling;
			residual += old > pr[i] ? old - pr[i] : pr[i] - old;
			pr_nn[i] = 0.0;
		}
		++iter;
		if (conv != 0.0 && residual <= conv) break;
	} while (iter < max_iter);
	*iterations = iter;
	*residual_out = residual;
	free(row_sum);
	free(pr_next);
	free(pr_nn);
	return residual <= conv ? 0 : 8;
}
