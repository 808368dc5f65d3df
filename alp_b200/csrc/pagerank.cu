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

// ------------------------------------------------ large graphs: per-step --
// For large graphs one cooperative kernel is the wrong shape: its columns
// that cross warp tiles wait on each other in tile order, and its grid is
// capped at what stays co-resident.  There every iteration is instead three
// ordinary launches -- the product over the CCS with the same row epilogue
// (k_pr_step; a column that crosses tiles leaves per-tile partials), the
// crossing columns' epilogue (k_pr_fix), and one block that sums the block
// partials in a fixed order and decides whether to stop (k_pr_finish).
// Iterations are queued in chunks; once the stop is decided every queued
// kernel returns at once, and the host reads the state once per chunk.
constexpr int PRS_WARPS = 4;
constexpr int PRS_CHUNK = 8;

struct PrStepState {
	int64_t iterations;
	double residual, d;
	int done;
};

struct PrStepArgs {
	MergeTables mt;                // over the CCS
	const int64_t *ccs_ptr;
	const uint32_t *ccs_row;
	const double *ccs_val;
	const int64_t *crs_ptr;
	const double *crs_val;
	double *pr, *rs, *next0, *next1;
	double *blk;                   // [2][grid]: residual, dangling of k_pr_step
	double *fix;                   // [2][fix_grid]: the same of k_pr_fix
	int grid, fix_grid;
	int64_t n, max_iter;
	double alpha, conv;
	int init_given;
	PrStepState *st;
};

// the row epilogue of both kernels (old pr and the row scale read directly)
struct PrStepEpi {
	const PrStepArgs *a;
	PrWarpSmem *sm;                // null: no per-tile prefetch (the crossing columns)
	double *next_out;
	double d;
	int64_t base = 0;
	double acc_res = 0.0, acc_dang = 0.0;
	__device__ __forceinline__ void begin_tile(int64_t i0, int nrows, int lane) {
		base = i0;
		for (int k = lane; k < nrows; k += 32) {
			sm->old_pr[k] = a->pr[i0 + k];
			sm->rs[k] = __ldg(a->rs + i0 + k);
		}
	}
	__device__ __forceinline__ void row(int64_t j, double v, bool has) {
		const double nn = has ? 0.0 + v : 0.0;       // pr_nextnext = 0; += pr_next L
		const double old = sm ? sm->old_pr[j - base] : a->pr[j];
		const double nw = nn + d;                    // pr = pr_nextnext + dangling
		a->pr[j] = nw;
		acc_res += old > nw ? old - nw : nw - old;
		const double rsj = sm ? sm->rs[j - base] : a->rs[j];
		if (rsj == 0.0) {                            // input of the next iteration
			next_out[j] = 0.0;
			acc_dang += nw;
		} else {
			next_out[j] = nw * rsj;
		}
	}
};

struct GatherRO {
	const double *__restrict__ x;
	__device__ __forceinline__ double operator()(uint32_t j) const { return __ldg(x + j); }
};

// set-up (:224-289 and the initial guess): row scales, pr, the pre-scaled
// first input and the blocks' dangling mass
__global__ void __launch_bounds__(256) k_pr_setup(PrStepArgs a) {
	__shared__ double red[33];
	const int lane = threadIdx.x & 31;
	const int64_t warp = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
	const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
	double dang = 0.0;
	for (int64_t i = warp; i < a.n; i += nwarps) {
		const int64_t b = a.crs_ptr[i], e = a.crs_ptr[i + 1];
		double cnt = 0.0;
		for (int64_t k = b + lane; k < e; k += 32)
			cnt += (a.crs_val == nullptr || a.crs_val[k] != 0.0) ? 1.0 : 0.0;
		for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
		if (lane == 0) {
			const double rsi = cnt > 0.0 ? a.alpha / cnt : 0.0;
			a.rs[i] = rsi;
			const double p = a.init_given ? a.pr[i] : 1.0 / double(a.n);
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
	if (threadIdx.x == 0) {
		a.blk[blockIdx.x] = 0.0;
		a.blk[a.grid + blockIdx.x] = dang;
	}
}

__global__ void __launch_bounds__(32 * PRS_WARPS, 6) k_pr_step(PrStepArgs a, int parity) {
	if (a.st->done) return;
	__shared__ PrWarpSmem sm[PRS_WARPS];
	__shared__ double red[33];
	const int w = threadIdx.x >> 5;
	PrStepEpi epi{&a, &sm[w], parity ? a.next0 : a.next1, a.st->d};
	GatherRO xl{parity ? a.next1 : a.next0};
	const int64_t nw = int64_t(gridDim.x) * PRS_WARPS;
	int64_t t = int64_t(blockIdx.x) * PRS_WARPS + w;
	WmMeta g = wm_meta(a.mt, t);
	while (t < a.mt.ntiles) {
		const WmMeta next = wm_meta(a.mt, t + nw);
		warp_tile<RF>(t, g, a.mt, a.ccs_ptr, a.ccs_row, a.ccs_val, xl, epi, 0, sm[w].tile);
		t += nw;
		g = next;
	}
	const double s1 = block_sum(epi.acc_res, red);
	const double s2 = block_sum(epi.acc_dang, red);
	if (threadIdx.x == 0) {
		a.blk[blockIdx.x] = s1;
		a.blk[a.grid + blockIdx.x] = s2;
	}
}

// columns that cross tiles: their partials summed in tile order (tail slots
// of the first..last-1 tiles, head slot of the last), then the epilogue
__global__ void __launch_bounds__(256) k_pr_fix(PrStepArgs a, int parity) {
	if (a.st->done) return;
	__shared__ double red[33];
	const MergeTables &mt = a.mt;
	PrStepEpi epi{&a, nullptr, parity ? a.next0 : a.next1, a.st->d};
	const int lane = threadIdx.x & 31;
	const int64_t warp = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
	const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
	for (int64_t base = warp * 32; base < mt.ntiles; base += nwarps * 32) {
		const int64_t t = base + lane;
		const int32_t n = t < mt.ntiles ? mt.span_len[t] : 0;
		if (n > 0 && n <= 32) {
			double v = wm_sum_slots<RF>(0.0, mt.tail_val, t, t + n - 1);
			v += load_bits<double>(mt.head_val + t + n - 1);
			epi.row(mt.tile_row[t + 1], v, true);
		}
		unsigned long_rows = __ballot_sync(0xffffffffu, n > 32);
		while (long_rows) {
			const int src = __ffs(long_rows) - 1;
			long_rows &= long_rows - 1;
			const int64_t f = base + src;
			const int32_t nn = __shfl_sync(0xffffffffu, n, src);
			double v = wm_sum_slots32<RF>(0.0, mt.tail_val, f + lane, f + nn - 1);
			for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
			if (lane == 0) {
				v += load_bits<double>(mt.head_val + f + nn - 1);
				epi.row(mt.tile_row[f + 1], v, true);
			}
		}
	}
	const double s1 = block_sum(epi.acc_res, red);
	const double s2 = block_sum(epi.acc_dang, red);
	if (threadIdx.x == 0) {
		a.fix[blockIdx.x] = s1;
		a.fix[a.fix_grid + blockIdx.x] = s2;
	}
}

// residual and dangling mass in a fixed order; the next teleport term; stop
// after an iteration whose residual is <= conv (:490) or at max_iter.
// setup != 0: only the first term (no iteration has run).
// The four sums of k_pr_finish in one pass: a thread's loads of all four
// arrays are in flight together, and each sum keeps block_sum_array's order
// (the thread's elements in stride order, then block_sum's tree), so the
// values are those of four block_sum_array calls bit for bit.
__device__ __forceinline__ void pr_finish_sums(const PrStepArgs &a, int setup,
	double (*smem)[33], double out[4]) {
	double v[4] = {0.0, 0.0, 0.0, 0.0};
	for (int64_t k = threadIdx.x; k < a.grid; k += blockDim.x) {
		v[0] += a.blk[k];
		v[1] += a.blk[a.grid + k];
	}
	if (!setup)
		for (int64_t k = threadIdx.x; k < a.fix_grid; k += blockDim.x) {
			v[2] += a.fix[k];
			v[3] += a.fix[a.fix_grid + k];
		}
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
	for (int q = 0; q < 4; ++q)
		for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
	if (lane == 0)
		for (int q = 0; q < 4; ++q) smem[q][wid] = v[q];
	__syncthreads();
	if (wid == 0) {
		const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
		for (int q = 0; q < 4; ++q) {
			double w = lane < nw ? smem[q][lane] : 0.0;
			for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
			if (lane == 0) smem[q][32] = w;
		}
	}
	__syncthreads();
	for (int q = 0; q < 4; ++q) out[q] = smem[q][32];
}

__global__ void __launch_bounds__(256) k_pr_finish(PrStepArgs a, int setup) {
	__shared__ double red[4][33];
	PrStepState *st = a.st;
	if (st->done) return;
	double sums[4];
	pr_finish_sums(a, setup, red, sums);
	const double r1 = sums[0], d1 = sums[1];
	const double r2 = setup ? 0.0 : sums[2];
	const double d2 = setup ? 0.0 : sums[3];
	if (threadIdx.x == 0) {
		const double dang = d1 + d2;
		st->d = (a.alpha * dang + 1 - a.alpha) / double(a.n);     // (:390)
		if (!setup) {
			st->residual = r1 + r2;
			st->iterations += 1;
			if ((a.conv != 0.0 && st->residual <= a.conv) || st->iterations >= a.max_iter)
				st->done = 1;
		}
	}
}

static int pagerank_steps(const PrStepArgs &tmpl, alpb_spmv_plan plan, int64_t *iterations,
	double *residual, cudaStream_t s) {
	PrStepArgs a = tmpl;
	static int per_sm = 0;
	if (!per_sm) {
		ALPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pr_step,
			32 * PRS_WARPS, 0));
		if (per_sm < 1) per_sm = 1;
	}
	int64_t g = (plan->ntiles + PRS_WARPS - 1) / PRS_WARPS;
	if (g > int64_t(per_sm) * sm_count()) g = int64_t(per_sm) * sm_count();
	a.grid = int(g < 1 ? 1 : g);
	a.fix_grid = int(grid_for((plan->ntiles + 31) / 32 * 32, 256));
	double *part = nullptr;
	PrStepState *st = nullptr;
	ALPB_CUDA(cudaMallocAsync(&part, size_t(2 * a.grid + 2 * a.fix_grid) * 8, s));
	ALPB_CUDA(cudaMallocAsync(&st, sizeof(PrStepState), s));
	ALPB_CUDA(cudaMemsetAsync(st, 0, sizeof(PrStepState), s));
	a.blk = part;
	a.fix = part + 2 * a.grid;
	a.st = st;
	k_pr_setup<<<a.grid, 256, 0, s>>>(a);
	ALPB_LAUNCHED();
	k_pr_finish<<<1, 256, 0, s>>>(a, 1);
	ALPB_LAUNCHED();
	PrStepState h{};
	int64_t queued = 0;
	while (queued < a.max_iter) {
		const int64_t chunk = a.max_iter - queued < PRS_CHUNK ? a.max_iter - queued : PRS_CHUNK;
		for (int64_t k = 0; k < chunk; ++k) {
			const int parity = int((queued + k) & 1);
			k_pr_step<<<a.grid, 32 * PRS_WARPS, 0, s>>>(a, parity);
			ALPB_LAUNCHED();
			k_pr_fix<<<a.fix_grid, 256, 0, s>>>(a, parity);
			ALPB_LAUNCHED();
			k_pr_finish<<<1, 256, 0, s>>>(a, 0);
			ALPB_LAUNCHED();
		}
		queued += chunk;
		ALPB_CUDA(cudaMemcpyAsync(&h, st, sizeof(PrStepState), cudaMemcpyDeviceToHost, s));
		ALPB_CUDA(cudaStreamSynchronize(s));
		if (h.done) break;
	}
	ALPB_CUDA(cudaFreeAsync(part, s));
	ALPB_CUDA(cudaFreeAsync(st, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	*iterations = h.iterations;
	*residual = h.residual;
	if (!(h.residual <= a.conv)) {
		set_error("alpb_pagerank: not converged after %lld iterations (residual %g)",
			(long long) h.iterations, h.residual);
		return ALPB_FAILED;
	}
	return ALPB_SUCCESS;
}

// Graphs from this many nonzeroes on take the per-step launches.
constexpr int64_t kPrStepNnz = int64_t(1) << 23;

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
	if (plan->nnz >= kPrStepNnz) {
		double *vecs = work, *own_vecs = nullptr;
		if (!vecs) {
			ALPB_CUDA(cudaMallocAsync(&own_vecs, size_t(3 * n) * 8, s));
			vecs = own_vecs;
		}
		PrStepArgs a{};
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
		a.n = n;
		a.max_iter = max_iter;
		a.alpha = alpha;
		a.conv = conv;
		a.init_given = init_given;
		const int rc = pagerank_steps(a, plan, iterations, residual, s);
		if (own_vecs) {
			cudaFreeAsync(own_vecs, s);
			cudaStreamSynchronize(s);
		}
		alpb_spmv_plan_destroy(own_plan);
		return rc;
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
