// Adjoint (implicit-function) gradients of a CG solve.
//
// For x = A^{-1} b and a loss L(x) with dL/dx = g, the implicit function
// theorem gives, with lambda = A^{-T} g:
//     dL/db      = lambda
//     dL/dA_ij   = -lambda_i x_j   on A's stored pattern only
// so no CG iterate is stored.  The adjoint system A^T lambda = g is solved by
// the same fused CG (cg.cu) on A's CCS, which IS the CRS of A^T: the
// transpose product needs neither atomics nor a second orientation build
// beyond the CCS the reference also keeps (reference/matrix.hpp:1298-1301).
// The gradient with respect to the stored values is a pattern-masked
// SDDMM (sampled dense-dense product) over A's CRS, on warp merge-path tiles
// so that every nonzero is written once, coalesced, whatever the row lengths.
#include "common.cuh"
#include "merge.cuh"
#include "wmerge.cuh"
#include "spmv.cuh"

#include <cmath>

namespace alpb {

// out[k] = alpha * lam[row(k)] * x[col(k)] for every stored k (CRS order),
// one warp merge tile (wmerge.cuh geometry) at a time
constexpr int SDDMM_WARPS = 8;

__global__ void __launch_bounds__(32 * SDDMM_WARPS)
k_sddmm(MergeTables mt, const int64_t *__restrict__ offsets, const uint32_t *__restrict__ indices,
	const double *__restrict__ lam, const double *__restrict__ x, double alpha,
	double *__restrict__ out) {
	__shared__ int32_t row_end_s[SDDMM_WARPS][WM_TILE + 2];
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	int32_t *row_end = row_end_s[w];
	const int64_t m = mt.m, nnz = mt.nnz;
	for (int64_t t = int64_t(blockIdx.x) * SDDMM_WARPS + w; t < mt.ntiles;
		 t += int64_t(gridDim.x) * SDDMM_WARPS) {
		const int64_t i0 = mt.tile_row[t], i1 = mt.tile_row[t + 1];
		int64_t d0, d1;
		if (mt.tile_d) {  // row-aligned or per-segment tiles
			d0 = mt.tile_d[t];
			d1 = mt.tile_d[t + 1];
		} else {
			d0 = t * WM_TILE;
			d1 = d0 + WM_TILE;
			if (d1 > m + nnz) d1 = m + nnz;
		}
		const int64_t j0 = d0 - i0, j1 = d1 - i1;
		const int nrows = int(i1 - i0), nnzt = int(j1 - j0);
		for (int k = lane; k <= nrows + 1; k += 32) {
			int64_t v;
			if (k == 0) v = offsets[i0] - j0;
			else {
				const int64_t r = i0 + k;
				v = (r <= m ? offsets[r] : j1 + 1) - j0;
			}
			if (v > WM_TILE + 1) v = WM_TILE + 1;
			if (v < -1) v = -1;
			row_end[k] = int32_t(v);
		}
		__syncwarp();
		for (int k = lane; k < nnzt; k += 32) {
			// tile row of nonzero k: the first r with end(r) > k
			int lo = 0, hi = nrows;
			while (lo < hi) {
				const int mid = (lo + hi) >> 1;
				if (row_end[mid + 1] > k) hi = mid; else lo = mid + 1;
			}
			const int64_t i = i0 + lo;
			const uint32_t j = __ldcs(indices + j0 + k);
			__stcs(out + j0 + k, alpha * __ldg(lam + i) * __ldg(x + j));
		}
		__syncwarp();
	}
}

__global__ void k_axpby(double *__restrict__ out, const double *__restrict__ a, double sa,
	const double *__restrict__ b, double sb, int64_t n) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x)
		out[i] = sa * a[i] + sb * b[i];
}

int dot_device(double *d_out, int add_op, int mul_op, int64_t n, const double *x,
	const uint8_t *xa, const double *y, const uint8_t *ya, int accumulate, cudaStream_t s);

} // namespace alpb

using namespace alpb;

extern "C" {

int alpb_sddmm(alpb_spmv_plan plan, int64_t m, int64_t nnz, const int64_t *offsets,
	const uint32_t *indices, const double *lam, const double *x, double alpha, double *out,
	void *stream) {
	ALPB_CHECK(m >= 0 && nnz >= 0, ALPB_ILLEGAL, "alpb_sddmm: negative size");
	if (m == 0 || nnz == 0) return ALPB_SUCCESS;
	cudaStream_t s = as_stream(stream);
	if (plan)
		ALPB_CHECK(plan->m == m && plan->nnz == nnz && plan->tile == WM_TILE, ALPB_MISMATCH,
			"alpb_sddmm: plan was made for another storage");
	alpb_spmv_plan own = nullptr;
	if (!plan) {
		int rc = plan_create_tiles(&own, m, nnz, offsets, ALPB_SCHED_MERGE_PATH, 0, WM_TILE, s);
		if (rc != ALPB_SUCCESS) return rc;
		plan = own;
	}
	int64_t grid = (plan->ntiles + SDDMM_WARPS - 1) / SDDMM_WARPS;
	if (grid > int64_t(sm_count()) * 8) grid = int64_t(sm_count()) * 8;
	k_sddmm<<<unsigned(grid), 32 * SDDMM_WARPS, 0, s>>>(merge_tables(*plan), offsets, indices, lam,
		x, alpha, out);
	ALPB_LAUNCHED();
	if (own) {
		ALPB_CUDA(cudaStreamSynchronize(s));
		alpb_spmv_plan_destroy(own);
	}
	return ALPB_SUCCESS;
}

int alpb_cg_adjoint(int64_t n, const int64_t *row_ptr, const uint32_t *col_idx,
	const double *values, const int64_t *ccs_col_ptr, const uint32_t *ccs_row_idx,
	const double *ccs_values, const double *x, const double *g, double *lambda, double *grad_values,
	int64_t max_iter, double tol, int64_t *iterations, double *residual, alpb_spmv_plan plan_crs,
	alpb_spmv_plan plan_ccs, void *stream) {
	ALPB_CHECK(n >= 0 && iterations && residual, ALPB_ILLEGAL, "alpb_cg_adjoint: bad arguments");
	if (n == 0) return ALPB_SUCCESS;
	cudaStream_t s = as_stream(stream);
	// A^T lambda = g on the CCS, from lambda = 0
	ALPB_CUDA(cudaMemsetAsync(lambda, 0, size_t(n) * 8, s));
	int rc = alpb_cg_solve(n, ccs_col_ptr, ccs_row_idx, ccs_values, g, lambda, max_iter, tol,
		iterations, residual, nullptr, plan_ccs, stream);
	if (rc != ALPB_SUCCESS) return rc;
	if (grad_values) {
		int64_t nnz = 0;
		if (plan_crs) nnz = plan_crs->nnz;
		else {
			ALPB_CUDA(cudaMemcpyAsync(&nnz, row_ptr + n, 8, cudaMemcpyDeviceToHost, s));
			ALPB_CUDA(cudaStreamSynchronize(s));
		}
		rc = alpb_sddmm(plan_crs, n, nnz, row_ptr, col_idx, lambda, x, -1.0, grad_values, stream);
	}
	(void) values;
	return rc;
}

int alpb_cg_grad(int64_t n, const int64_t *row_ptr, const uint32_t *col_idx, const double *values,
	const int64_t *ccs_col_ptr, const uint32_t *ccs_row_idx, const double *ccs_values,
	const double *b, const double *x_target, double *x, double *lambda, double *grad_values,
	double *work, int64_t max_iter, double tol, double *loss, int64_t *iterations_fwd,
	int64_t *iterations_adj, alpb_spmv_plan plan_crs, alpb_spmv_plan plan_ccs, void *stream) {
	ALPB_CHECK(loss && iterations_fwd && iterations_adj && work, ALPB_ILLEGAL,
		"alpb_cg_grad: null argument");
	cudaStream_t s = as_stream(stream);
	double res = 0;
	// forward: A x = b from x = 0
	ALPB_CUDA(cudaMemsetAsync(x, 0, size_t(n) * 8, s));
	int rc = alpb_cg_solve(n, row_ptr, col_idx, values, b, x, max_iter, tol, iterations_fwd, &res,
		nullptr, plan_crs, stream);
	if (rc != ALPB_SUCCESS) return rc;
	// g = dL/dx = x - x*, L = 0.5 g.g
	double *gvec = work;
	k_axpby<<<grid_for(n, 256), 256, 0, s>>>(gvec, x, 1.0, x_target, -1.0, n);
	ALPB_LAUNCHED();
	double *d_loss = work + n;
	rc = dot_device(d_loss, ALPB_OP_ADD, ALPB_OP_MUL, n, gvec, nullptr, gvec, nullptr, 0, s);
	if (rc != ALPB_SUCCESS) return rc;
	double h = 0;
	ALPB_CUDA(cudaMemcpyAsync(&h, d_loss, 8, cudaMemcpyDeviceToHost, s));
	rc = alpb_cg_adjoint(n, row_ptr, col_idx, values, ccs_col_ptr, ccs_row_idx, ccs_values, x, gvec,
		lambda, grad_values, max_iter, tol, iterations_adj, &res, plan_crs, plan_ccs, stream);
	ALPB_CUDA(cudaStreamSynchronize(s));
	*loss = 0.5 * h;
	return rc;
}

} // extern "C"
