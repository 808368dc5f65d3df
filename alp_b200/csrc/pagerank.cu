// Fused PageRank: algorithms::simple_pagerank
// (include/graphblas/algorithms/simple_pagerank.hpp:146-533) as ONE
// persistent cooperative launch with one bounded grid barrier per iteration.
//
// Per iteration the reference pre-scales pr by alpha / outdegree (keeping
// the dangling mass apart), runs vxm over L (a gather over L's CCS), adds the
// teleport + dangling term and measures the L1 change.  Here the CCS gather
// runs on merge-path tiles and its row epilogue does all of the rest for the
// column it just finished: new pr_j, |new - old|, and already the pre-scaled
// input of the NEXT iteration (pr_next, double-buffered) with its dangling
// mass, so the next gather can start right after the barrier.
#include "common.cuh"
#include "merge.cuh"
#include "wmerge.cuh"
#include "persist.cuh"
#include "spmv.cuh"

#include <cmath>

namespace alpb {

using RF = RingPlusTimesF64;

struct PrState {
	GridSync gs;
	int64_t iterations;
	double residual;
};

struct PrArgs {
	MergeTables mt;                // over the CCS
	const int64_t *ccs_ptr;
	const uint32_t *ccs_row;
	const double *ccs_val;
	const int64_t *crs_ptr;
	const double *crs_val;
	double *pr, *rs, *next0, *next1;
	double *blk;                   // [5][grid]: setup dangling mass; per iteration
	                               // parity p, residual [1+2p] and dangling [2+2p]
	int64_t n, max_iter;
	double alpha, conv;
	int init_given;
	PrState *st;
};

constexpr int PR_WARPS = 4;

struct PrWarpSmem {
	WarpSmem<RF> tile;
	double old_pr[WM_TILE];
	double rs[WM_TILE];
};

struct PrEpi {
	const PrArgs *a;
	PrWarpSmem *sm;
	double *next_out;
	double d;
	int64_t base = 0;
	double acc_res = 0.0, acc_dang = 0.0;
	__device__ __forceinline__ void begin_tile(int64_t i0, int nrows, int lane) {
		base = i0;
		for (int k = lane; k < nrows; k += 32) {
			sm->old_pr[k] = __ldcg(a->pr + i0 + k);
			sm->rs[k] = __ldg(a->rs + i0 + k);
		}
	}
	__device__ __forceinline__ void row(int64_t j, double v, bool has) {
		const double nn = has ? 0.0 + v : 0.0;       // pr_nextnext = 0; += pr_next L
		const double old = sm->old_pr[j - base];
		const double nw = nn + d;                    // pr = pr_nextnext + dangling
		a->pr[j] = nw;
		acc_res += old > nw ? old - nw : nw - old;
		const double rsj = sm->rs[j - base];
		if (rsj == 0.0) {                            // input of the next iteration
			next_out[j] = 0.0;
			acc_dang += nw;
		} else {
			next_out[j] = nw * rsj;
		}
	}
};

struct GatherL2 {
	const double *x;
	__device__ __forceinline__ double operator()(uint32_t j) const { return __ldcg(x + j); }
};

// One barrier per iteration; the block partials of iteration k live in the
// parity-(k & 1) slots, so a block that already writes iteration k+1's never
// overwrites what a slower block still reads of iteration k.
__global__ void __launch_bounds__(32 * PR_WARPS, 6) k_pagerank(PrArgs a) {
	__shared__ PrWarpSmem sm[PR_WARPS];
	__shared__ double red[33];
	PrState *st = a.st;
	int *err = &st->gs.err;
	const int64_t G = gridDim.x, n = a.n, nt = a.mt.ntiles;
	const int lane = threadIdx.x & 31;
	const int w = threadIdx.x >> 5;
	const int64_t gw = int64_t(blockIdx.x) * PR_WARPS + w, nw = G * PR_WARPS;
	// setup: out-degree counts of nonzero-valued entries (the pattern ring of
	// :224-237), alpha / count (:281-289), initial guess, pre-scaled input
	double dang = 0.0;
	for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < nt;
		 t += G * blockDim.x)
		a.mt.ready[t] = 0;
	for (int64_t i = gw; i < n; i += nw) {
		const int64_t b = a.crs_ptr[i], e = a.crs_ptr[i + 1];
		double cnt = 0.0;
		for (int64_t k = b + lane; k < e; k += 32)
			cnt += (a.crs_val == nullptr || a.crs_val[k] != 0.0) ? 1.0 : 0.0;
		for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
		if (lane == 0) {
			const double rsi = cnt > 0.0 ? a.alpha / cnt : 0.0;
			a.rs[i] = rsi;
			const double p = a.init_given ? a.pr[i] : 1.0 / double(n);
			a.pr[i] = p;
			if (rsi == 0.0) {
				a.next0[i] = 0.0;
				dang += p;
			} else {
				a.next0[i] = p * rsi;
			}
		}
	}
	dang = block_sum(dang, red);
	if (threadIdx.x == 0) a.blk[blockIdx.x] = dang;
	if (!grid_sync(&st->gs)) return;
	dang = block_sum_array(a.blk, G, red);

	int64_t iter = 0;
	double residual = 0.0;
	double *cur = a.next0, *nxt = a.next1;
	for (;;) {
		const double d = (a.alpha * dang + 1 - a.alpha) / double(n);  // (:390)
		PrEpi epi{&a, &sm[w], nxt, d};
		GatherL2 xl{cur};
		const int32_t epoch = int32_t(iter + 1);
		int64_t t = gw;
		WmMeta g = wm_meta(a.mt, t);
		while (t < nt) {
			const WmMeta next = wm_meta(a.mt, t + nw);
			if (!warp_tile_ordered<RF>(t, g, a.mt, a.ccs_ptr, a.ccs_row, a.ccs_val, xl, epi, 1,
					sm[w].tile, epoch, err))
				break;
			t += nw;
			g = next;
		}
		double *blk_res = a.blk + (1 + 2 * (iter & 1)) * G;
		double *blk_dang = a.blk + (2 + 2 * (iter & 1)) * G;
		const double s1 = block_sum(epi.acc_res, red);
		const double s2 = block_sum(epi.acc_dang, red);
		if (threadIdx.x == 0) {
			blk_res[blockIdx.x] = s1;
			blk_dang[blockIdx.x] = s2;
		}
		if (!grid_sync(&st->gs)) return;
		residual = block_sum_array(blk_res, G, red);
		dang = block_sum_array(blk_dang, G, red);
		++iter;
		if (a.conv != 0.0 && residual <= a.conv) break;   // (:490)
		if (iter >= a.max_iter) break;
		double *tmp = cur;
		cur = nxt;
		nxt = tmp;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		st->iterations = iter;
		st->residual = residual;
	}
}

// The solve proper.  plan: a WM_TILE plan of the CCS offsets, or null (one is
// made and destroyed here); work: 3n doubles of scratch, or null.
static int pagerank_run(int64_t n, const int64_t *crs_row_ptr, const double *crs_values,
	const int64_t *ccs_col_ptr, const uint32_t *ccs_row_idx, const double *ccs_values, double *pr,
	int init_given, double alpha, double conv, int64_t max_iter, int64_t *iterations,
	double *residual, double *work, alpb_spmv_plan plan, cudaStream_t s) {
	alpb_spmv_plan own_plan = nullptr;
	if (!plan) {
		int64_t nnz = 0;
		ALPB_CUDA(cudaMemcpyAsync(&nnz, ccs_col_ptr + n, 8, cudaMemcpyDeviceToHost, s));
		ALPB_CUDA(cudaStreamSynchronize(s));
		int rc = plan_create_tiles(&own_plan, n, nnz, ccs_col_ptr, ALPB_SCHED_MERGE_PATH, 0,
			WM_TILE, s);
		if (rc != ALPB_SUCCESS) return rc;
		plan = own_plan;
	}
	const int grid = solver_grid(k_pagerank, 32 * PR_WARPS, plan->ntiles, PR_WARPS);
	if (grid <= 0) {
		alpb_spmv_plan_destroy(own_plan);
		set_error("alpb_pagerank: no cooperative occupancy");
		return ALPB_PANIC;
	}
	double *vecs = work, *own_vecs = nullptr, *blk = nullptr;
	PrState *st = nullptr;
	if (!vecs) {
		ALPB_CUDA(cudaMallocAsync(&own_vecs, size_t(3 * n) * 8, s));
		vecs = own_vecs;
	}
	ALPB_CUDA(cudaMallocAsync(&blk, size_t(5 * int64_t(grid)) * 8, s));
	ALPB_CUDA(cudaMallocAsync(&st, sizeof(PrState), s));
	ALPB_CUDA(cudaMemsetAsync(st, 0, sizeof(PrState), s));
	PrArgs a;
	a.mt = merge_tables(*plan);
	a.ccs_ptr = ccs_col_ptr;
	a.ccs_row = ccs_row_idx;
	a.ccs_val = ccs_values;
	a.crs_ptr = crs_row_ptr;
	a.crs_val = crs_values;
	a.pr = pr;
	a.rs = vecs;
	a.next0 = vecs + n;
	a.next1 = vecs + 2 * n;
	a.blk = blk;
	a.n = n;
	a.max_iter = max_iter;
	a.alpha = alpha;
	a.conv = conv;
	a.init_given = init_given;
	a.st = st;
	void *args[] = {&a};
	ALPB_CUDA(cudaLaunchCooperativeKernel((void *) k_pagerank, dim3(grid), dim3(32 * PR_WARPS), args,
		0, s));
	ALPB_LAUNCHED();
	PrState h;
	ALPB_CUDA(cudaMemcpyAsync(&h, st, sizeof(PrState), cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaFreeAsync(blk, s));
	ALPB_CUDA(cudaFreeAsync(st, s));
	if (own_vecs) ALPB_CUDA(cudaFreeAsync(own_vecs, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	alpb_spmv_plan_destroy(own_plan);
	ALPB_CHECK(h.gs.err == 0, ALPB_PANIC, "alpb_pagerank: a grid barrier or tile wait timed out");
	*iterations = h.iterations;
	*residual = h.residual;
	if (!(h.residual <= conv)) {
		set_error("alpb_pagerank: not converged after %lld iterations (residual %g)",
			(long long) h.iterations, h.residual);
		return ALPB_FAILED;
	}
	return ALPB_SUCCESS;
}

static int pagerank_checks(int64_t n, double alpha, int64_t max_iter, const int64_t *iterations,
	const double *residual) {
	ALPB_CHECK(alpha > 0 && alpha < 1, ALPB_ILLEGAL, "alpb_pagerank: alpha must be in (0, 1)");
	ALPB_CHECK(max_iter > 0, ALPB_ILLEGAL, "alpb_pagerank: max must be positive");
	ALPB_CHECK(iterations && residual, ALPB_ILLEGAL, "alpb_pagerank: null output");
	ALPB_CHECK(n > 0, ALPB_ILLEGAL, "alpb_pagerank: empty graph");
	return ALPB_SUCCESS;
}

} // namespace alpb

using namespace alpb;

extern "C" int alpb_pagerank(int64_t n, const int64_t *crs_row_ptr, const uint32_t *crs_col_idx,
	const double *crs_values, const int64_t *ccs_col_ptr, const uint32_t *ccs_row_idx,
	const double *ccs_values, double *pr, int init_given, double alpha, double conv,
	int64_t max_iter, int64_t *iterations, double *residual, void *stream) {
	(void) crs_col_idx;
	const int rc = pagerank_checks(n, alpha, max_iter, iterations, residual);
	if (rc != ALPB_SUCCESS) return rc;
	return pagerank_run(n, crs_row_ptr, crs_values, ccs_col_ptr, ccs_row_idx, ccs_values, pr,
		init_given, alpha, conv, max_iter, iterations, residual, nullptr, nullptr,
		as_stream(stream));
}

extern "C" int alpb_pagerank_planned(int64_t n, const int64_t *crs_row_ptr,
	const uint32_t *crs_col_idx, const double *crs_values, const int64_t *ccs_col_ptr,
	const uint32_t *ccs_row_idx, const double *ccs_values, double *pr, int init_given,
	double alpha, double conv, int64_t max_iter, int64_t *iterations, double *residual,
	double *work, alpb_spmv_plan ccs_plan, void *stream) {
	(void) crs_col_idx;
	const int rc = pagerank_checks(n, alpha, max_iter, iterations, residual);
	if (rc != ALPB_SUCCESS) return rc;
	ALPB_CHECK(!ccs_plan || (ccs_plan->m == n && ccs_plan->offsets == ccs_col_ptr &&
			ccs_plan->tile == WM_TILE), ALPB_MISMATCH,
		"alpb_pagerank_planned: plan was made for another storage");
	return pagerank_run(n, crs_row_ptr, crs_values, ccs_col_ptr, ccs_row_idx, ccs_values, pr,
		init_given, alpha, conv, max_iter, iterations, residual, work, ccs_plan,
		as_stream(stream));
}
