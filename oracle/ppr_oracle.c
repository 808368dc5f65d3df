/*
 * ppr_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C (OpenMP) restatement of oracle/ppr.py: personalised PageRank over a
 * weighted graph, its adjoint and the edge-weight gradient.  It forms the
 * same gathers in the same order as the numpy restatement (which
 * tests/test_oracle_ppr.py pins to the compiled reference's simple_pagerank),
 * so that the parity tests can check the device at the benchmark's scale,
 * where numpy's scatter-adds take minutes per iteration.  Only tests/ load it
 * (through oracle/oracle.py); the product never does.
 *
 * The iteration is algorithms::simple_pagerank
 * (include/graphblas/algorithms/simple_pagerank.hpp:146-533) with a one-hot
 * teleport vector per seed and the weighted out-degree d_i = sum_j w_ij:
 *   y = x * alpha / d (0 on dangling rows)                       (:281-289, :324-357)
 *   term_s = alpha * sum_{dangling i} x_is + 1 - alpha            (:390)
 *   x'_js = sum_{(i,j) stored} w_ij y_is  (+ term_s at j = seed_s) (:400, :440-470)
 *   residual_s = sum_i |x_is - x'_is|; a seed stops after the iteration whose
 *   residual is <= conv, or at max_iter                          (:490)
 * Adjoint of the fixed point x = alpha M x + alpha v 1_D^T x + (1 - alpha) v
 * (M_ji = w_ij / d_i):  lambda = alpha M^T lambda + alpha 1_D lambda[seed] + g.
 * Gradient: dL/dw_ij = alpha / d_i sum_s x_is (lambda_js - (M^T lambda_s)_i).
 *
 * Vectors are row-major n x S (entry i*S + s).  Every gather sums a column
 * (forward) or a row (adjoint) in the CRS storage order of its entries, as
 * numpy's scatter-adds do, so the iterates agree with oracle/ppr.py to the
 * last bits.  Column sums (per-seed residuals and dangling masses) add
 * partials of fixed blocks of 4096 rows in block order: the same terms as
 * numpy's axis-0 sums, grouped differently (relative 1e-16).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* CCS of the CRS (rp, col, w): for each column, its (row, weight) pairs in
 * increasing CRS position -- the order np.add.at visits them. */
static int ccs_of(int64_t n, const int64_t *rp, const uint32_t *col, const double *w,
	int64_t **cp_out, uint32_t **row_out, double **wt_out) {
	const int64_t nnz = rp[n];
	int64_t *cp = (int64_t *) calloc((size_t) n + 1, 8);
	uint32_t *row = (uint32_t *) malloc((size_t) (nnz ? nnz : 1) * 4);
	double *wt = (double *) malloc((size_t) (nnz ? nnz : 1) * 8);
	int64_t *fill = (int64_t *) malloc((size_t) (n + 1) * 8);
	if (!cp || !row || !wt || !fill) {
		free(cp); free(row); free(wt); free(fill);
		return 2;
	}
	for (int64_t k = 0; k < nnz; ++k) cp[col[k] + 1]++;
	for (int64_t j = 0; j < n; ++j) cp[j + 1] += cp[j];
	memcpy(fill, cp, (size_t) (n + 1) * 8);
	for (int64_t i = 0; i < n; ++i)
		for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
			const int64_t p = fill[col[k]]++;
			row[p] = (uint32_t) i;
			wt[p] = w[k];
		}
	free(fill);
	*cp_out = cp;
	*row_out = row;
	*wt_out = wt;
	return 0;
}

static double *weighted_degrees(int64_t n, const int64_t *rp, const double *w) {
	double *d = (double *) malloc((size_t) (n ? n : 1) * 8);
	if (!d) return NULL;
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < n; ++i) {
		double s = 0.0;
		for (int64_t k = rp[i]; k < rp[i + 1]; ++k) s += w[k];
		d[i] = s;
	}
	return d;
}

enum { kRowBlock = 4096 };

/* out1_s = sum_i |a_is - b_is| (b == NULL: sum_i a_is) over all rows, and
 * out2_s = sum_{i: d_i == 0} c_is (when out2), each from per-block partials
 * added in block order. */
static int column_sums(int64_t n, int64_t S, const double *a, const double *b,
	const double *d, const double *c, double *out1, double *out2) {
	const int64_t nb = (n + kRowBlock - 1) / kRowBlock;
	double *p1 = (double *) calloc((size_t) (nb * S), 8);
	double *p2 = (double *) calloc((size_t) (nb * S), 8);
	if (!p1 || !p2) {
		free(p1); free(p2);
		return 2;
	}
#pragma omp parallel for schedule(static)
	for (int64_t blk = 0; blk < nb; ++blk) {
		double *q1 = p1 + blk * S, *q2 = p2 + blk * S;
		const int64_t i1 = (blk + 1) * kRowBlock < n ? (blk + 1) * kRowBlock : n;
		for (int64_t i = blk * kRowBlock; i < i1; ++i) {
			for (int64_t s = 0; s < S; ++s)
				q1[s] += b ? fabs(a[i * S + s] - b[i * S + s]) : a[i * S + s];
			if (out2 && d[i] == 0.0)
				for (int64_t s = 0; s < S; ++s) q2[s] += c[i * S + s];
		}
	}
	for (int64_t s = 0; s < S; ++s) {
		double t1 = 0.0, t2 = 0.0;
		for (int64_t blk = 0; blk < nb; ++blk) {
			t1 += p1[blk * S + s];
			t2 += p2[blk * S + s];
		}
		out1[s] = t1;
		if (out2) out2[s] = t2;
	}
	free(p1);
	free(p2);
	return 0;
}

/* x: n*S in/out (taken as the initial guess when x_given, else 1/n). */
int alpo_ppr_forward(int64_t n, const int64_t *rp, const uint32_t *col, const double *w,
	int64_t S, const int64_t *seeds, double alpha, double conv, int64_t max_iter, int x_given,
	double *x, int64_t *iters, double *res) {
	if (n <= 0 || S <= 0) return 7;
	int64_t *cp;
	uint32_t *row;
	double *wt;
	if (ccs_of(n, rp, col, w, &cp, &row, &wt)) return 2;
	double *d = weighted_degrees(n, rp, w);
	double *rs = (double *) malloc((size_t) n * 8);
	double *y = (double *) malloc((size_t) (n * S) * 8);
	double *nw = (double *) malloc((size_t) (n * S) * 8);
	double *term = (double *) calloc((size_t) S, 8), *r = (double *) calloc((size_t) S, 8);
	double *dng = (double *) calloc((size_t) S, 8);
	char *active = (char *) malloc((size_t) S);
	int rc = 0;
	if (!d || !rs || !y || !nw || !term || !r || !dng || !active) {
		rc = 2;
		goto done;
	}
	for (int64_t i = 0; i < n; ++i) rs[i] = d[i] == 0.0 ? 0.0 : alpha / d[i];
	if (!x_given)
		for (int64_t q = 0; q < n * S; ++q) x[q] = 1.0 / (double) n;
	if (column_sums(n, S, x, NULL, d, x, r, dng)) {
		rc = 2;
		goto done;
	}
	for (int64_t s = 0; s < S; ++s) {
		term[s] = alpha * dng[s] + 1 - alpha;
		active[s] = 1;
		iters[s] = 0;
		res[s] = 0.0;
	}
	for (int64_t k = 0; k < max_iter; ++k) {
		int any = 0;
		for (int64_t s = 0; s < S; ++s) any |= active[s];
		if (!any) break;
#pragma omp parallel for schedule(static)
		for (int64_t i = 0; i < n; ++i)
			for (int64_t s = 0; s < S; ++s) y[i * S + s] = x[i * S + s] * rs[i];
#pragma omp parallel for schedule(dynamic, 256)
		for (int64_t j = 0; j < n; ++j) {
			double *o = nw + j * S;
			for (int64_t s = 0; s < S; ++s) o[s] = 0.0;
			for (int64_t p = cp[j]; p < cp[j + 1]; ++p) {
				const double a = wt[p];
				const double *yi = y + (int64_t) row[p] * S;
				for (int64_t s = 0; s < S; ++s) o[s] += a * yi[s];
			}
		}
		for (int64_t s = 0; s < S; ++s) nw[seeds[s] * S + s] += term[s];
		if (column_sums(n, S, x, nw, d, nw, r, dng)) {
			rc = 2;
			goto done;
		}
#pragma omp parallel for schedule(static)
		for (int64_t i = 0; i < n; ++i)
			for (int64_t s = 0; s < S; ++s)
				if (active[s]) x[i * S + s] = nw[i * S + s];
		for (int64_t s = 0; s < S; ++s) {
			if (!active[s]) continue;
			res[s] = r[s];
			iters[s] = k + 1;
			term[s] = alpha * dng[s] + 1 - alpha;
			if ((conv != 0.0 && r[s] <= conv) || k + 1 >= max_iter) active[s] = 0;
		}
	}
done:
	free(cp); free(row); free(wt); free(d); free(rs); free(y); free(nw);
	free(term); free(r); free(dng); free(active);
	return rc;
}

/* acc_is = sum_{k in row i} w_k lam_{col_k, s}, in storage order. */
static void adjoint_gather(int64_t n, const int64_t *rp, const uint32_t *col, const double *w,
	int64_t S, const double *lam, double *acc) {
#pragma omp parallel for schedule(dynamic, 256)
	for (int64_t i = 0; i < n; ++i) {
		double *o = acc + i * S;
		for (int64_t s = 0; s < S; ++s) o[s] = 0.0;
		for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
			const double a = w[k];
			const double *l = lam + (int64_t) col[k] * S;
			for (int64_t s = 0; s < S; ++s) o[s] += a * l[s];
		}
	}
}

/* lam: n*S out; g: dL/dx, n*S. */
int alpo_ppr_adjoint(int64_t n, const int64_t *rp, const uint32_t *col, const double *w,
	int64_t S, const int64_t *seeds, const double *g, double alpha, double conv,
	int64_t max_iter, double *lam, int64_t *iters, double *res) {
	if (n <= 0 || S <= 0) return 7;
	double *d = weighted_degrees(n, rp, w);
	double *inv_d = (double *) malloc((size_t) n * 8);
	double *acc = (double *) malloc((size_t) (n * S) * 8);
	double *nw = (double *) malloc((size_t) (n * S) * 8);
	double *term = (double *) calloc((size_t) S, 8), *r = (double *) calloc((size_t) S, 8);
	char *active = (char *) malloc((size_t) S);
	int rc = 0;
	if (!d || !inv_d || !acc || !nw || !term || !r || !active) {
		rc = 2;
		goto done;
	}
	for (int64_t i = 0; i < n; ++i) inv_d[i] = d[i] == 0.0 ? 0.0 : 1.0 / d[i];
	memcpy(lam, g, (size_t) (n * S) * 8);
	for (int64_t s = 0; s < S; ++s) {
		active[s] = 1;
		iters[s] = 0;
		res[s] = 0.0;
	}
	for (int64_t k = 0; k < max_iter; ++k) {
		int any = 0;
		for (int64_t s = 0; s < S; ++s) any |= active[s];
		if (!any) break;
		for (int64_t s = 0; s < S; ++s) term[s] = alpha * lam[seeds[s] * S + s];
		adjoint_gather(n, rp, col, w, S, lam, acc);
#pragma omp parallel for schedule(static)
		for (int64_t i = 0; i < n; ++i)
			for (int64_t s = 0; s < S; ++s)
				nw[i * S + s] = alpha * (acc[i * S + s] * inv_d[i]) +
					(d[i] == 0.0 ? term[s] : 0.0) + g[i * S + s];
		if (column_sums(n, S, nw, lam, d, NULL, r, NULL)) {
			rc = 2;
			goto done;
		}
#pragma omp parallel for schedule(static)
		for (int64_t i = 0; i < n; ++i)
			for (int64_t s = 0; s < S; ++s)
				if (active[s]) lam[i * S + s] = nw[i * S + s];
		for (int64_t s = 0; s < S; ++s) {
			if (!active[s]) continue;
			res[s] = r[s];
			iters[s] = k + 1;
			if ((conv != 0.0 && r[s] <= conv) || k + 1 >= max_iter) active[s] = 0;
		}
	}
done:
	free(d); free(inv_d); free(acc); free(nw); free(term); free(r); free(active);
	return rc;
}

/* grad: one entry per stored edge, in CRS order. */
int alpo_ppr_grad(int64_t n, const int64_t *rp, const uint32_t *col, const double *w,
	int64_t S, const double *x, const double *lam, double alpha, double *grad) {
	if (n <= 0 || S <= 0) return 7;
	double *d = weighted_degrees(n, rp, w);
	double *acc = (double *) malloc((size_t) (n * S) * 8);
	double *c = (double *) malloc((size_t) n * 8);
	if (!d || !acc || !c) {
		free(d); free(acc); free(c);
		return 2;
	}
	adjoint_gather(n, rp, col, w, S, lam, acc);
#pragma omp parallel for schedule(dynamic, 256)
	for (int64_t i = 0; i < n; ++i) {
		const double inv = d[i] == 0.0 ? 0.0 : 1.0 / d[i];
		double ci = 0.0;
		for (int64_t s = 0; s < S; ++s) ci += x[i * S + s] * (acc[i * S + s] * inv);
		c[i] = ci;
		for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
			const double *l = lam + (int64_t) col[k] * S;
			double dot = 0.0;
			for (int64_t s = 0; s < S; ++s) dot += x[i * S + s] * l[s];
			grad[k] = alpha * inv * (dot - ci);
		}
	}
	free(d); free(acc); free(c);
	return 0;
}
