// Fused conjugate gradient: algorithms::preconditioned_conjugate_gradient,
// unpreconditioned branch (include/graphblas/algorithms/conjugate_gradient.hpp:
// 191-483), as ONE persistent cooperative launch.
//
// The reference makes, per iteration, one mxv and nine passes over n-vectors
// with three host-visible dot products.  Here an iteration is two phases
// separated by a bounded grid barrier, with every scalar kept on the device:
//
//   A: temp = A u_new, gathering u_new_j = r_j + gamma u_old_j on the fly
//      (merge-path tiles, merge.cuh); the row epilogue writes temp_i and
//      u_new_i and forms the terms of beta = temp . u_new.
//   B: alpha = sigma / beta; x += alpha u_new; r -= alpha temp; r . r.
//
// The u update of the reference (u = r + (r.r / sigma) u, :455-468) is thus
// folded into the next SpMV's gather, with u double-buffered so that no
// block overwrites an entry another block still gathers.  Convergence is
// tested exactly as the reference does (sqrt(r.r) < tol * ||b||, :437), and
// the returned residual is r.r.
#include "common.cuh"
#include "merge.cuh"
#include "persist.cuh"
#include "spmv.cuh"

#include <cmath>

namespace alpb {

using RF = RingPlusTimesF64;

struct CgState {
	GridSync gs;
	int64_t iterations;
	double residual;
	double tol_abs;
	int converged;
};

struct CgArgs {
	MergeTables mt;
	const int64_t *offsets;
	const uint32_t *indices;
	const double *values;
	const double *b;
	double *x, *r, *u0, *u1, *temp;
	double *own, *span, *own2, *span2;  // [ntiles] tile terms / spanning-row terms
	double *blk;                        // [grid] block partials of r.r
	int64_t n, max_iter;
	double tol;
	CgState *st;
};

struct PreludeEpi {
	const CgArgs *a;
	double acc_rr = 0.0, acc_bb = 0.0;
	__device__ __forceinline__ void terms(int64_t i, double v, bool has, double &rr, double &bb) {
		const double t = has ? 0.0 + v : 0.0;      // temp = 0; temp += A x
		const double bi = a->b[i];
		const double ri = (0.0 + bi) - t;           // r = 0; r += b; r -= temp
		a->r[i] = ri;
		a->u0[i] = 0.0;
		rr = ri * ri;
		bb = bi * bi;
	}
	__device__ __forceinline__ void row(int64_t i, double v, bool has) {
		double rr, bb;
		terms(i, v, has, rr, bb);
		acc_rr += rr;
		acc_bb += bb;
	}
	__device__ __forceinline__ void row_span(int64_t first, int64_t i, double v, bool has) {
		double rr, bb;
		terms(i, v, has, rr, bb);
		a->span[first] = rr;
		a->span2[first] = bb;
	}
};

struct GatherU {
	const double *r, *u_old;
	double gamma;
	// r and u_old were written by other blocks before the last barrier: read
	// them through L2 (ld.global.cg) so no stale L1 line can be hit
	__device__ __forceinline__ double operator()(uint32_t j) const {
		return __ldcg(r + j) + gamma * __ldcg(u_old + j);
	}
};

struct IterEpi {
	const CgArgs *a;
	const double *u_old;
	double *u_new;
	double gamma;
	double acc = 0.0;
	__device__ __forceinline__ double term(int64_t i, double v, bool has) {
		const double t = has ? 0.0 + v : 0.0;      // temp = 0; temp += A u
		a->temp[i] = t;
		const double un = __ldcg(a->r + i) + gamma * __ldcg(u_old + i);
		u_new[i] = un;
		return t * un;
	}
	__device__ __forceinline__ void row(int64_t i, double v, bool has) { acc += term(i, v, has); }
	__device__ __forceinline__ void row_span(int64_t first, int64_t i, double v, bool has) {
		a->span[first] = term(i, v, has);
	}
};

__global__ void __launch_bounds__(MP_BLOCK) k_cg(CgArgs a) {
	__shared__ MergeSmem<RF> sm;
	__shared__ double red[33];
	CgState *st = a.st;
	const int64_t G = gridDim.x;
	const int64_t nt = a.mt.ntiles;
	for (int64_t t = blockIdx.x; t < nt; t += G) {
		a.span[t] = 0.0;
		a.span2[t] = 0.0;
	}
	if (!grid_sync(&st->gs)) return;

	// prelude: r = b - A x, u = r (by gamma = 0 below), sigma = r.r, |b|^2
	{
		PreludeEpi epi{&a};
		PlainX<double> xl{a.x};
		for (int64_t t = blockIdx.x; t < nt; t += G) {
			epi.acc_rr = epi.acc_bb = 0.0;
			merge_tile<RF>(t, a.mt, a.offsets, a.indices, a.values, xl, epi, 0, sm);
			const double s1 = block_sum(epi.acc_rr, red);
			const double s2 = block_sum(epi.acc_bb, red);
			if (threadIdx.x == 0) {
				a.own[t] = s1;
				a.own2[t] = s2;
			}
		}
	}
	if (!grid_sync(&st->gs)) return;
	double sigma = block_sum_array(a.own, nt, red) + block_sum_array(a.span, nt, red);
	const double bnorm = block_sum_array(a.own2, nt, red) + block_sum_array(a.span2, nt, red);
	const double tol_abs = a.tol * sqrt(bnorm);

	const int64_t chunk = (a.n + G - 1) / G;
	const int64_t rb = blockIdx.x * chunk;
	const int64_t re = rb + chunk < a.n ? rb + chunk : a.n;
	double gamma = 0.0;
	double rr = 0.0;
	int64_t iter = 0;
	double *u_old = a.u0, *u_new = a.u1;
	for (;;) {
		++iter;
		// phase A: temp = A u_new, u_new = r + gamma u_old, beta terms
		{
			IterEpi epi{&a, u_old, u_new, gamma};
			GatherU xl{a.r, u_old, gamma};
			for (int64_t t = blockIdx.x; t < nt; t += G) {
				epi.acc = 0.0;
				merge_tile<RF>(t, a.mt, a.offsets, a.indices, a.values, xl, epi, 0, sm);
				const double s = block_sum(epi.acc, red);
				if (threadIdx.x == 0) a.own[t] = s;
			}
		}
		if (!grid_sync(&st->gs)) return;
		// phase B: alpha = sigma / beta, x += alpha u, r -= alpha temp, r.r
		const double beta = block_sum_array(a.own, nt, red) + block_sum_array(a.span, nt, red);
		const double alpha = sigma / beta;
		double part = 0.0;
		for (int64_t i = rb + threadIdx.x; i < re; i += blockDim.x) {
			const double un = __ldcg(u_new + i);
			a.x[i] = a.x[i] + alpha * un;
			const double ri = __ldcg(a.r + i) - alpha * __ldcg(a.temp + i);
			a.r[i] = ri;
			part += ri * ri;
		}
		part = block_sum(part, red);
		if (threadIdx.x == 0) a.blk[blockIdx.x] = part;
		if (!grid_sync(&st->gs)) return;
		rr = block_sum_array(a.blk, G, red);
		if (sqrt(rr) < tol_abs || iter >= a.max_iter) break;
		gamma = rr / sigma;  // alpha = beta / sigma in the reference's naming
		sigma = rr;
		double *tmp = u_old;
		u_old = u_new;
		u_new = tmp;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		st->iterations = iter;
		st->residual = rr;
		st->tol_abs = tol_abs;
		st->converged = sqrt(rr) < tol_abs ? 1 : 0;
	}
}

} // namespace alpb

using namespace alpb;

extern "C" int alpb_cg_solve(int64_t n, const int64_t *row_ptr, const uint32_t *col_idx,
	const double *values, const double *b, double *x, int64_t max_iter, double tol,
	int64_t *iterations, double *residual, double *work, alpb_spmv_plan plan, void *stream) {
	ALPB_CHECK(n >= 0, ALPB_ILLEGAL, "alpb_cg_solve: negative size");
	ALPB_CHECK(tol > 0, ALPB_ILLEGAL, "alpb_cg_solve: tolerance must be strictly positive");
	ALPB_CHECK(max_iter > 0, ALPB_ILLEGAL, "alpb_cg_solve: at least one iteration is required");
	ALPB_CHECK(iterations && residual, ALPB_ILLEGAL, "alpb_cg_solve: null output");
	*iterations = 0;
	*residual = INFINITY;
	if (n == 0) return ALPB_SUCCESS;
	cudaStream_t s = as_stream(stream);
	if (plan)
		ALPB_CHECK(plan->m == n && plan->offsets == row_ptr, ALPB_MISMATCH,
			"alpb_cg_solve: plan was made for another storage");
	alpb_spmv_plan own_plan = nullptr;
	if (!plan || plan->tile != MP_TILE) {
		// the fused kernel runs block tiles: it needs tables cut at MP_TILE
		int64_t nnz = 0;
		ALPB_CUDA(cudaMemcpyAsync(&nnz, row_ptr + n, 8, cudaMemcpyDeviceToHost, s));
		ALPB_CUDA(cudaStreamSynchronize(s));
		int rc = plan_create_tiles(&own_plan, n, nnz, row_ptr, ALPB_SCHED_MERGE_PATH, 0, MP_TILE, s);
		if (rc != ALPB_SUCCESS) return rc;
		plan = own_plan;
	}
	const int64_t nt = plan->ntiles;
	int grid = cooperative_grid(k_cg, MP_BLOCK, 0, 0);
	ALPB_CHECK(grid > 0, ALPB_PANIC, "alpb_cg_solve: no cooperative occupancy");
	// a few blocks per SM: the per-iteration scalar reductions read every
	// tile's partial in every block
	if (grid > 2 * sm_count()) grid = 2 * sm_count();
	double *wk = work, *own_work = nullptr, *scratch = nullptr;
	CgState *st = nullptr;
	if (!wk) {
		ALPB_CUDA(cudaMallocAsync(&own_work, size_t(4 * n) * 8, s));
		wk = own_work;
	}
	ALPB_CUDA(cudaMallocAsync(&scratch, size_t(4 * nt + grid) * 8, s));
	ALPB_CUDA(cudaMallocAsync(&st, sizeof(CgState), s));
	ALPB_CUDA(cudaMemsetAsync(st, 0, sizeof(CgState), s));
	CgArgs a;
	a.mt = merge_tables(*plan);
	a.offsets = row_ptr;
	a.indices = col_idx;
	a.values = values;
	a.b = b;
	a.x = x;
	a.r = wk;
	a.u0 = wk + n;
	a.u1 = wk + 2 * n;
	a.temp = wk + 3 * n;
	a.own = scratch;
	a.span = scratch + nt;
	a.own2 = scratch + 2 * nt;
	a.span2 = scratch + 3 * nt;
	a.blk = scratch + 4 * nt;
	a.n = n;
	a.max_iter = max_iter;
	a.tol = tol;
	a.st = st;
	void *args[] = {&a};
	ALPB_CUDA(cudaLaunchCooperativeKernel((void *) k_cg, dim3(grid), dim3(MP_BLOCK), args, 0, s));
	ALPB_LAUNCHED();
	CgState h;
	ALPB_CUDA(cudaMemcpyAsync(&h, st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaFreeAsync(scratch, s));
	ALPB_CUDA(cudaFreeAsync(st, s));
	if (own_work) ALPB_CUDA(cudaFreeAsync(own_work, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	if (own_plan) alpb_spmv_plan_destroy(own_plan);
	ALPB_CHECK(h.gs.err == 0, ALPB_PANIC, "alpb_cg_solve: grid barrier timed out");
	*iterations = h.iterations;
	*residual = h.residual;
	if (!h.converged) {
		set_error("alpb_cg_solve: not converged after %lld iterations (sqrt(r.r) = %g, tol %g)",
			(long long) h.iterations, sqrt(h.residual), h.tol_abs);
		return ALPB_FAILED;
	}
	return ALPB_SUCCESS;
}
