/*
 * Driver of ALP's sparse-BLAS transition API (include/transition/blas_sparse.h),
 * linked once against ALP's src/transition/sparseblas.cpp compiled for the
 * b200 backend and once against the same source on the reference backend.
 *
 *   sparseblas_driver m n seed y_out
 *
 * Builds an m x n matrix of about 12 m random entries (half by
 * BLAS_duscr_insert_entries, half row by row), then runs
 *   y1 = 1.0 A x + y0,  y2 = 2.5 A x + y0,  y3 = 2.5 A^T z + w0
 * with BLAS_dusmv; prints the return codes and the stored nonzero count and
 * writes y1, y2, y3 (doubles) to y_out.
 */
#include <stdio.h>
#include <stdlib.h>

#include "blas_sparse.h"

static unsigned long long state;
static double urand(void) {
	state = state * 6364136223846793005ULL + 1442695040888963407ULL;
	return (double) (state >> 11) / 9007199254740992.0;
}

int main(int argc, char **argv) {
	if (argc != 5) {
		fprintf(stderr, "usage: %s m n seed y_out\n", argv[0]);
		return 2;
	}
	const int m = atoi(argv[1]), n = atoi(argv[2]);
	state = (unsigned long long) atoll(argv[3]);
	/* distinct (row, col) pairs: row-major scan with a random keep decision */
	const int per = 12;
	int *rows = malloc(sizeof(int) * m * per), *cols = malloc(sizeof(int) * m * per);
	double *vals = malloc(sizeof(double) * m * per);
	int nz = 0;
	for (int i = 0; i < m; ++i) {
		int c = (int) (urand() * 4);
		for (int k = 0; k < per && c < n; ++k) {
			rows[nz] = i;
			cols[nz] = c;
			vals[nz] = urand() - 0.5;
			++nz;
			c += 1 + (int) (urand() * (2.0 * n / per));
		}
	}
	blas_sparse_matrix A = BLAS_duscr_begin(m, n);
	const int half = nz / 2;
	int rc_ins = BLAS_duscr_insert_entries(A, half, vals, rows, cols);
	for (int k = half; k < nz;) {     /* the rest row by row */
		int e = k;
		while (e < nz && rows[e] == rows[k]) ++e;
		const int rc = BLAS_duscr_insert_row(A, rows[k], e - k, vals + k, cols + k);
		if (rc) rc_ins = rc;
		k = e;
	}
	const int rc_end = BLAS_duscr_end(A);
	int stored = -1;
	const int rc_nz = EXTBLAS_dusm_nz(A, &stored);
	double *x = malloc(sizeof(double) * n), *z = malloc(sizeof(double) * m);
	double *y = malloc(sizeof(double) * 3 * (m > n ? m : n));
	double *y1 = y, *y2 = y + m, *y3 = y + 2 * m;
	for (int j = 0; j < n; ++j) x[j] = urand() - 0.5;
	for (int i = 0; i < m; ++i) z[i] = urand() - 0.5;
	for (int i = 0; i < m; ++i) y1[i] = y2[i] = urand();
	for (int j = 0; j < n; ++j) y3[j] = urand();
	const int rc1 = BLAS_dusmv(blas_no_trans, 1.0, A, x, 1, y1, 1);
	const int rc2 = BLAS_dusmv(blas_no_trans, 2.5, A, x, 1, y2, 1);
	const int rc3 = BLAS_dusmv(blas_trans, 2.5, A, z, 1, y3, 1);
	const int rc_ds = BLAS_usds(A);
	printf("rc_insert %d\nrc_end %d\nrc_nz %d\nnnz %d\nstored %d\nrc_mv1 %d\nrc_mv2 %d\nrc_mv3 %d\n"
		"rc_destroy %d\n", rc_ins, rc_end, rc_nz, nz, stored, rc1, rc2, rc3, rc_ds);
	FILE *f = fopen(argv[4], "wb");
	if (f) {
		fwrite(y1, sizeof(double), m, f);
		fwrite(y2, sizeof(double), m, f);
		fwrite(y3, sizeof(double), n, f);
		fclose(f);
	}
	EXTBLAS_free();
	return 0;
}
