// Fused conjugate gradient: algorithms::preconditioned_conjugate_gradient,
// unpreconditioned branch (include/graphblas/algorithms/conjugate_gradient.hpp:
// 191-483), as ONE persistent cooperative launch.
//
// The reference makes, per iteration, one mxv and nine passes over n-vectors
// with three host-visible dot products.  Here an iteration is two phases
// separated by a bounded grid barrier, with every scalar kept on the device:
//
//   A: temp = A u_new, gathering u_new_j = r_j + gamma u_old_j on the fly
//      (warp merge-path tiles, wmerge.cuh); the row epilogue writes temp_i
//      and u_new_i and forms the terms of beta = temp . u_new.
//   B: alpha = sigma / beta; x += alpha u_new; r -= alpha temp; r . r.
//
// The u update of the reference (u = r + (r.r / sigma) u, :455-468) is thus
// folded into the next SpMV's gather.  r and u are stored side by side, one
// 16-byte pair per row, so that the gather of a nonzero is ONE load (one L1
// wavefront) that brings both; phase A writes u_new to its own array, which
// phase B folds back into the pairs, so no block overwrites a pair that
// another block still gathers.  Convergence is tested exactly as the
// reference does (sqrt(r.r) < tol * ||b||, :437), and the returned residual
// is r.r.  Work space: pairs (2n doubles), u_new (n), temp (n); on return
// its first n doubles hold the final residual vector r.
#include "common.cuh"
#include "merge.cuh"
#include "wmerge.cuh"
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
	double *x;
	double2 *pr;   // (r_i, u_i)
	double *u_new, *temp;
	double *r_out; // the first n doubles of the work space: r on return
	double *blk;  // [4][grid] block partials: prelude r.r, prelude b.b, beta, r.r
	int64_t n, max_iter;
	double tol;
	CgState *st;
};

// Warps per block: 16 for systems of few tiles (every warp then holds about
// one tile, so the latency of a phase is that of one tile), 8 otherwise.
// Measured on B200, us per iteration (27-point grids): 32^3 -- 25.4 with 4
// warps, 18.5 with 8, 16.5 with 16; 64^3 -- 58.3, 56.7, 61.1.
constexpr int64_t CG_FEW_TILES = 8192;

// Shared memory of one warp: the tile engine's staging plus the epilogue's
// prefetched vector entries for the rows that end in the tile.
struct CgWarpSmem {
	WarpSmem<RF> tile;
	double p0[WM_TILE];
	double p1[WM_TILE];
};

struct PreludeEpi {
	const CgArgs *a;
	CgWarpSmem *sm;
	int64_t base = 0;
	double acc_rr = 0.0, acc_bb = 0.0;
	__device__ __forceinline__ void begin_tile(int64_t i0, int nrows, int lane) {
		base = i0;
		for (int k = lane; k < nrows; k += 32) sm->p0[k] = a->b[i0 + k];
	}
	__device__ __forceinline__ void row(int64_t i, double v, bool has) {
		const double t = has ? 0.0 + v : 0.0;      // temp = 0; temp += A x
		const double bi = sm->p0[i - base];
		const double ri = (0.0 + bi) - t;           // r = 0; r += b; r -= temp
		a->pr[i] = make_double2(ri, 0.0);            // u = 0: gamma = 0 takes u = r
		acc_rr += ri * ri;
		acc_bb += bi * bi;
	}
};

struct GatherU {
	const double2 *pr;
	double gamma;
	// the pairs were written by other blocks before the last barrier: read
	// them through L2 (ld.global.cg) so no stale L1 line can be hit
	__device__ __forceinline__ double operator()(uint32_t j) const {
		const double2 p = __ldcg(pr + j);
		return p.x + gamma * p.y;
	}
};

struct IterEpi {
	const CgArgs *a;
	CgWarpSmem *sm;
	double gamma;
	int64_t base = 0;
	double acc = 0.0;
	__device__ __forceinline__ void begin_tile(int64_t i0, int nrows, int lane) {
		base = i0;
		for (int k = lane; k < nrows; k += 32) {
			const double2 p = __ldcg(a->pr + i0 + k);
			sm->p0[k] = p.x;
			sm->p1[k] = p.y;
		}
	}
	__device__ __forceinline__ void row(int64_t i, double v, bool has) {
		const double t = has ? 0.0 + v : 0.0;      // temp = 0; temp += A u
		a->temp[i] = t;
		const double un = sm->p0[i - base] + gamma * sm->p1[i - base];
		a->u_new[i] = un;
		acc += t * un;
	}
};

// Rows are finished by fixed tiles (warp_tile_ordered) and every partial is
// reduced in a fixed order (lane terms in tile order, block_sum, then the
// block partials in block order): the iterates are deterministic for a given
// grid size.
template <int CG_WARPS>
__global__ void __launch_bounds__(32 * CG_WARPS, 24 / CG_WARPS) k_cg(CgArgs a) {
	extern __shared__ __align__(16) unsigned char cg_smem[];
	CgWarpSmem *sm = reinterpret_cast<CgWarpSmem *>(cg_smem);  // one per warp
	__shared__ double red[33];
	CgState *st = a.st;
	int *err = &st->gs.err;
	const int64_t G = gridDim.x;
	const int64_t nt = a.mt.ntiles;
	const int w = threadIdx.x >> 5;
	const int64_t gw = int64_t(blockIdx.x) * CG_WARPS + w, nw = G * CG_WARPS;
	double *blk_rr0 = a.blk, *blk_bb0 = a.blk + G, *blk_beta = a.blk + 2 * G,
		   *blk_rr = a.blk + 3 * G;
	for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < nt;
		 t += G * blockDim.x)
		a.mt.ready[t] = 0;
	if (!grid_sync(&st->gs)) return;
	int32_t epoch = 0;

	// prelude: r = b - A x, u = r (by gamma = 0 below), sigma = r.r, |b|^2
	{
		PreludeEpi epi{&a, &sm[w]};
		PlainX<double> xl{a.x};
		++epoch;
		int64_t t = gw;
		WmMeta g = wm_meta(a.mt, t);
		while (t < nt) {
			const WmMeta next = wm_meta(a.mt, t + nw);
			if (!warp_tile_ordered<RF>(t, g, a.mt, a.offsets, a.indices, a.values, xl, epi, 0,
					sm[w].tile, epoch, err))
				break;
			t += nw;
			g = next;
		}
		const double s1 = block_sum(epi.acc_rr, red);
		const double s2 = block_sum(epi.acc_bb, red);
		if (threadIdx.x == 0) {
			blk_rr0[blockIdx.x] = s1;
			blk_bb0[blockIdx.x] = s2;
		}
	}
	if (!grid_sync(&st->gs)) return;
	double sigma = block_sum_array(blk_rr0, G, red);
	const double bnorm = block_sum_array(blk_bb0, G, red);
	const double tol_abs = a.tol * sqrt(bnorm);

	const int64_t chunk = (a.n + G - 1) / G;
	const int64_t rb = blockIdx.x * chunk;
	const int64_t re = rb + chunk < a.n ? rb + chunk : a.n;
	double gamma = 0.0;
	double rr = 0.0;
	int64_t iter = 0;
	for (;;) {
		++iter;
		// phase A: temp = A u_new, u_new = r + gamma u_old, beta terms
		{
			IterEpi epi{&a, &sm[w], gamma};
			GatherU xl{a.pr, gamma};
			++epoch;
			int64_t t = gw;
			WmMeta g = wm_meta(a.mt, t);
			while (t < nt) {
				const WmMeta next = wm_meta(a.mt, t + nw);
				if (!warp_tile_ordered<RF>(t, g, a.mt, a.offsets, a.indices, a.values, xl, epi, 0,
						sm[w].tile, epoch, err))
					break;
				t += nw;
				g = next;
			}
			const double s = block_sum(epi.acc, red);
			if (threadIdx.x == 0) blk_beta[blockIdx.x] = s;
		}
		if (!grid_sync(&st->gs)) return;
		// phase B: alpha = sigma / beta, x += alpha u, r -= alpha temp, r.r
		const double beta = block_sum_array(blk_beta, G, red);
		const double alpha = sigma / beta;
		double part = 0.0;
		for (int64_t i = rb + threadIdx.x; i < re; i += blockDim.x) {
			const double un = __ldcg(a.u_new + i);
			a.x[i] = a.x[i] + alpha * un;
			const double ri = __ldcg(a.pr + i).x - alpha * __ldcg(a.temp + i);
			a.pr[i] = make_double2(ri, un);
			part += ri * ri;
		}
		part = block_sum(part, red);
		if (threadIdx.x == 0) blk_rr[blockIdx.x] = part;
		if (!grid_sync(&st->gs)) return;
		rr = block_sum_array(blk_rr, G, red);
		if (sqrt(rr) < tol_abs || iter >= a.max_iter) break;
		gamma = rr / sigma;  // alpha = beta / sigma in the reference's naming
		sigma = rr;
	}
	// r out to the first n doubles of the work space, which the pairs occupy:
	// through temp, with a barrier between reading the pairs and overwriting them
	for (int64_t i = rb + threadIdx.x; i < re; i += blockDim.x) a.temp[i] = __ldcg(a.pr + i).x;
	if (!grid_sync(&st->gs)) return;
	for (int64_t i = rb + threadIdx.x; i < re; i += blockDim.x) a.r_out[i] = __ldcg(a.temp + i);
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
		ALPB_CHECK(plan->m == n && plan->offsets == row_ptr && plan->tile == WM_TILE,
			ALPB_MISMATCH, "alpb_cg_solve: plan was made for another storage");
	alpb_spmv_plan own_plan = nullptr;
	if (!plan) {
		int64_t nnz = 0;
		ALPB_CUDA(cudaMemcpyAsync(&nnz, row_ptr + n, 8, cudaMemcpyDeviceToHost, s));
		ALPB_CUDA(cudaStreamSynchronize(s));
		int rc = plan_create_tiles(&own_plan, n, nnz, row_ptr, ALPB_SCHED_MERGE_PATH, 0, WM_TILE, s);
		if (rc != ALPB_SUCCESS) return rc;
		plan = own_plan;
	}
	const bool few = plan->ntiles <= CG_FEW_TILES;
	const int warps = few ? 16 : 8;
	const size_t smem = sizeof(CgWarpSmem) * warps;
	static bool smem_set = false;
	if (!smem_set) {
		ALPB_CUDA(cudaFuncSetAttribute(k_cg<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			int(sizeof(CgWarpSmem) * 16)));
		ALPB_CUDA(cudaFuncSetAttribute(k_cg<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			int(sizeof(CgWarpSmem) * 8)));
		smem_set = true;
	}
	const int grid = few ? solver_grid(k_cg<16>, 32 * 16, plan->ntiles, 16, smem)
						 : solver_grid(k_cg<8>, 32 * 8, plan->ntiles, 8, smem);
	ALPB_CHECK(grid > 0, ALPB_PANIC, "alpb_cg_solve: no cooperative occupancy");
	// the (r, u) pairs take 16-byte loads: a work space that is not 16-byte
	// aligned is replaced by an internal one
	double *wk = (reinterpret_cast<uintptr_t>(work) & 15) ? nullptr : work;
	double *own_work = nullptr, *scratch = nullptr;
	CgState *st = nullptr;
	if (!wk) {
		ALPB_CUDA(cudaMallocAsync(&own_work, size_t(4 * n) * 8, s));
		wk = own_work;
	}
	ALPB_CUDA(cudaMallocAsync(&scratch, size_t(4 * grid) * 8, s));
	ALPB_CUDA(cudaMallocAsync(&st, sizeof(CgState), s));
	ALPB_CUDA(cudaMemsetAsync(st, 0, sizeof(CgState), s));
	CgArgs a;
	a.mt = merge_tables(*plan);
	a.offsets = row_ptr;
	a.indices = col_idx;
	a.values = values;
	a.b = b;
	a.x = x;
	a.pr = reinterpret_cast<double2 *>(wk);
	a.u_new = wk + 2 * n;
	a.temp = wk + 3 * n;
	a.r_out = wk;
	a.blk = scratch;
	a.n = n;
	a.max_iter = max_iter;
	a.tol = tol;
	a.st = st;
	void *args[] = {&a};
	ALPB_CUDA(cudaLaunchCooperativeKernel(few ? (void *) k_cg<16> : (void *) k_cg<8>, dim3(grid),
		dim3(32 * warps), args, smem, s));
	ALPB_LAUNCHED();
	CgState h;
	ALPB_CUDA(cudaMemcpyAsync(&h, st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaFreeAsync(scratch, s));
	ALPB_CUDA(cudaFreeAsync(st, s));
	if (own_work) ALPB_CUDA(cudaFreeAsync(own_work, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	if (own_plan) alpb_spmv_plan_destroy(own_plan);
	ALPB_CHECK(h.gs.err == 0, ALPB_PANIC, "alpb_cg_solve: a grid barrier or tile wait timed out");
	*iterations = h.iterations;
	*residual = h.residual;
	if (!h.converged) {
		set_error("alpb_cg_solve: not converged after %lld iterations (sqrt(r.r) = %g, tol %g)",
			(long long) h.iterations, sqrt(h.residual), h.tol_abs);
		return ALPB_FAILED;
	}
	return ALPB_SUCCESS;
}
