/*
 * Driver of ALP's transition CG API (include/transition/solver.h), linked
 * once against ALP's src/transition/solver.cpp compiled for the b200 backend
 * and once against the same source on the reference backend (the checker).
 *
 *   transition_driver dii|diz|dzz precondition(0|1) nx tol max_iter x_out
 *
 * System: the 27-point nx^3 stencil (diagonal 26, off-diagonals -1, columns
 * increasing in a row), b = A 1.  With precondition = 1 a Jacobi
 * preconditioner (z = r / 26) is passed through the C callback.  Prints the
 * return codes, the iteration count and the residual; writes x (doubles).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "solver.h"

static int jacobi(double *const out, const double *const in, void *const data) {
	const size_t n = *(const size_t *) data;
	for (size_t i = 0; i < n; ++i) out[i] = in[i] / 26.0;
	return 0;
}

int main(int argc, char **argv) {
	if (argc != 7) {
		fprintf(stderr, "usage: %s dii|diz|dzz precondition nx tol max_iter x_out\n", argv[0]);
		return 2;
	}
	const char *var = argv[1];
	const int pre = atoi(argv[2]);
	const long nx = atol(argv[3]);
	const double tol = atof(argv[4]);
	const size_t max_iter = (size_t) atol(argv[5]);
	const size_t n = (size_t) (nx * nx * nx);
	size_t *ia = malloc((n + 1) * sizeof(size_t));
	size_t *ja = malloc(n * 27 * sizeof(size_t));
	double *a = malloc(n * 27 * sizeof(double));
	size_t nz = 0;
	ia[0] = 0;
	for (long z = 0; z < nx; ++z)
		for (long y = 0; y < nx; ++y)
			for (long x = 0; x < nx; ++x) {
				const size_t i = (size_t) ((z * nx + y) * nx + x);
				for (long dz = -1; dz <= 1; ++dz)
					for (long dy = -1; dy <= 1; ++dy)
						for (long dx = -1; dx <= 1; ++dx) {
							const long zz = z + dz, yy = y + dy, xx = x + dx;
							if (zz < 0 || yy < 0 || xx < 0 || zz >= nx || yy >= nx || xx >= nx) continue;
							const size_t j = (size_t) ((zz * nx + yy) * nx + xx);
							ja[nz] = j;
							a[nz] = i == j ? 26.0 : -1.0;
							++nz;
						}
				ia[i + 1] = nz;
			}
	double *b = malloc(n * sizeof(double)), *xs = calloc(n, sizeof(double));
	for (size_t i = 0; i < n; ++i) {
		double s = 0;
		for (size_t k = ia[i]; k < ia[i + 1]; ++k) s += a[k];
		b[i] = s;
	}
	int *ja32 = malloc(nz * sizeof(int)), *ia32 = malloc((n + 1) * sizeof(int));
	for (size_t k = 0; k < nz; ++k) ja32[k] = (int) ja[k];
	for (size_t i = 0; i <= n; ++i) ia32[i] = (int) ia[i];
	sparse_cg_handle_t h = NULL;
	sparse_err_t e_init, e_tol, e_max, e_pre = NO_ERROR, e_solve, e_it, e_res, e_dest;
	size_t iters = 0;
	double residual = 0;
	if (strcmp(var, "dii") == 0) {
		e_init = sparse_cg_init_dii(&h, n, a, ja32, ia32);
		e_tol = sparse_cg_set_tolerance_dii(h, tol);
		e_max = sparse_cg_set_max_iter_count_dii(h, max_iter);
		if (pre) e_pre = sparse_cg_set_preconditioner_dii(h, jacobi, (void *) &n);
		e_solve = sparse_cg_solve_dii(h, xs, b);
		e_it = sparse_cg_get_iter_count_dii(h, &iters);
		e_res = sparse_cg_get_residual_dii(h, &residual);
		e_dest = sparse_cg_destroy_dii(h);
	} else if (strcmp(var, "diz") == 0) {
		e_init = sparse_cg_init_diz(&h, n, a, ja32, ia);
		e_tol = sparse_cg_set_tolerance_diz(h, tol);
		e_max = sparse_cg_set_max_iter_count_diz(h, max_iter);
		if (pre) e_pre = sparse_cg_set_preconditioner_diz(h, jacobi, (void *) &n);
		e_solve = sparse_cg_solve_diz(h, xs, b);
		e_it = sparse_cg_get_iter_count_diz(h, &iters);
		e_res = sparse_cg_get_residual_diz(h, &residual);
		e_dest = sparse_cg_destroy_diz(h);
	} else {
		e_init = sparse_cg_init_dzz(&h, n, a, ja, ia);
		e_tol = sparse_cg_set_tolerance_dzz(h, tol);
		e_max = sparse_cg_set_max_iter_count_dzz(h, max_iter);
		if (pre) e_pre = sparse_cg_set_preconditioner_dzz(h, jacobi, (void *) &n);
		e_solve = sparse_cg_solve_dzz(h, xs, b);
		e_it = sparse_cg_get_iter_count_dzz(h, &iters);
		e_res = sparse_cg_get_residual_dzz(h, &residual);
		e_dest = sparse_cg_destroy_dzz(h);
	}
	printf("rc_init %d\nrc_tol %d\nrc_max %d\nrc_pre %d\nrc_solve %d\nrc_iter %d\nrc_res %d\n"
		"rc_destroy %d\niterations %zu\nresidual %.17g\n", (int) e_init, (int) e_tol, (int) e_max,
		(int) e_pre, (int) e_solve, (int) e_it, (int) e_res, (int) e_dest, iters, residual);
	FILE *f = fopen(argv[6], "wb");
	if (f) {
		fwrite(xs, sizeof(double), n, f);
		fclose(f);
	}
	return 0;
}
