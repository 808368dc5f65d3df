// Batched conjugate gradient: many independent SPD systems of uneven size,
// solved together in ONE persistent cooperative launch.
//
// The instances are stored as one block-diagonal CRS (instance i owns rows
// [seg_rows[i], seg_rows[i+1])).  Tiles are cut per instance, so every tile
// belongs to exactly one instance and every instance scalar (beta, alpha,
// r.r, gamma, sigma) is a sum over that instance's tiles.  Two tilings:
//   - systems whose rows hold at most 32 nonzeroes get a sliced copy of the
//     matrix (ELL-32 per instance: entry q of 32 consecutive rows is one
//     contiguous line), and a tile is a slice computed one row per lane;
//   - other systems use warp tiles of the merge-path engine
//     (merge_plan_segmented), rows crossing tiles handled by ordered waits.
// An iteration is the single-system solver's two phases (cg.cu), each
// followed by a per-instance reduction of the tile partials (one block per
// instance, fixed order: deterministic), with a grid barrier after each of
// the four steps.  Warps walk only the tiles of the instances still
// iterating (a list every block rebuilds after each convergence step).  An
// instance that converges (its own relative tolerance, as
// algorithms::conjugate_gradient tests it, conjugate_gradient.hpp:377-378,
// :437) or exhausts the iteration budget is masked out; the launch ends when
// no instance is active.
#include "common.cuh"
#include "merge.cuh"
#include "wmerge.cuh"
#include "persist.cuh"
#include "spmv.cuh"

#include <cub/device/device_scan.cuh>

#include <cmath>
#include <vector>

namespace alpb {

using RF = RingPlusTimesF64;

// ------------------------------------------------------ segmented tables --
// Tiles per instance: whole-row tiles of `rpt` rows when rpt > 0, else
// merge-path tiles of `tile` items.  An instance without rows is flagged.
__global__ void k_seg_tile_counts(const int64_t *offsets, const int64_t *seg_rows, int64_t nseg,
	int64_t *counts, int64_t tile, int64_t rpt, int32_t *empty) {
	for (int64_t s = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; s <= nseg;
		 s += int64_t(gridDim.x) * blockDim.x) {
		if (s == nseg) { counts[s] = 0; continue; }
		const int64_t r0 = seg_rows[s], r1 = seg_rows[s + 1];
		if (r1 <= r0) atomicExch(empty, 1);
		const int64_t items = (r1 - r0) + (offsets[r1] - offsets[r0]);
		counts[s] = rpt ? (r1 - r0 + rpt - 1) / rpt : (items + tile - 1) / tile;
	}
}

// Whole-row tiles: tile t of instance s holds rows [r0 + k rpt, r0 + (k+1) rpt).
__global__ void k_seg_aligned(const int64_t *offsets, const int64_t *seg_rows,
	const int64_t *seg_tile, int64_t nseg, int64_t m, int64_t nnz, int64_t rpt, int64_t *tile_d,
	int64_t *tile_row, int32_t *tile_seg, int64_t *head_first, int64_t *tail_first,
	int32_t *span_len) {
	for (int64_t s = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; s < nseg;
		 s += int64_t(gridDim.x) * blockDim.x) {
		const int64_t r0 = seg_rows[s], r1 = seg_rows[s + 1];
		for (int64_t t = seg_tile[s]; t < seg_tile[s + 1]; ++t) {
			int64_t r = r0 + (t - seg_tile[s]) * rpt;
			if (r > r1) r = r1;
			tile_row[t] = r;
			tile_d[t] = r + offsets[r];
			tile_seg[t] = int32_t(s);
			head_first[t] = -1;
			tail_first[t] = -1;
			span_len[t] = 0;
		}
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		tile_d[seg_tile[nseg]] = m + nnz;
		tile_row[seg_tile[nseg]] = m;
	}
}

__global__ void k_seg_tile_d(const int64_t *offsets, const int64_t *seg_rows, const int64_t *seg_tile,
	int64_t nseg, int64_t m, int64_t nnz, int64_t *tile_d, int32_t *tile_seg, int64_t tile) {
	for (int64_t s = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; s < nseg;
		 s += int64_t(gridDim.x) * blockDim.x) {
		const int64_t r0 = seg_rows[s];
		const int64_t base = r0 + offsets[r0];
		for (int64_t t = seg_tile[s]; t < seg_tile[s + 1]; ++t) {
			tile_d[t] = base + (t - seg_tile[s]) * tile;
			tile_seg[t] = int32_t(s);
		}
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) tile_d[seg_tile[nseg]] = m + nnz;
}

__device__ __forceinline__ int64_t merge_search_d(const int64_t *offsets, int64_t m, int64_t nnz,
	int64_t d) {
	int64_t lo = d - nnz > 0 ? d - nnz : 0;
	int64_t hi = d < m ? d : m;
	while (lo < hi) {
		const int64_t pivot = (lo + hi) >> 1;
		if (offsets[pivot + 1] <= d - pivot - 1) lo = pivot + 1; else hi = pivot;
	}
	return lo;
}

__global__ void k_seg_tile_rows(const int64_t *offsets, int64_t m, int64_t nnz, int64_t ntiles,
	const int64_t *tile_d, int64_t *tile_row) {
	for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t <= ntiles;
		 t += int64_t(gridDim.x) * blockDim.x)
		tile_row[t] = merge_search_d(offsets, m, nnz, tile_d[t]);
}

// tile containing diagonal d: last t with tile_d[t] <= d
__device__ __forceinline__ int64_t tile_of(const int64_t *tile_d, int64_t ntiles, int64_t d) {
	int64_t lo = 0, hi = ntiles - 1;
	while (lo < hi) {
		const int64_t mid = (lo + hi + 1) >> 1;
		if (tile_d[mid] <= d) lo = mid; else hi = mid - 1;
	}
	return lo;
}

__global__ void k_seg_tables(const int64_t *offsets, int64_t m, int64_t ntiles,
	const int64_t *tile_d, const int64_t *tile_row, int64_t *head_first, int64_t *tail_first,
	int32_t *span_len) {
	for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < ntiles;
		 t += int64_t(gridDim.x) * blockDim.x) {
		const int64_t i0 = tile_row[t], i1 = tile_row[t + 1];
		const int64_t d0 = tile_d[t], d1 = tile_d[t + 1];
		const int64_t j0 = d0 - i0, j1 = d1 - i1;
		head_first[t] = (i1 > i0 && offsets[i0] < j0) ? tile_of(tile_d, ntiles, i0 + offsets[i0]) : -1;
		int64_t tf = -1;
		if (i1 < m) {
			const int64_t start = offsets[i1] > j0 ? offsets[i1] : j0;
			if (j1 > start) tf = tile_of(tile_d, ntiles, i1 + offsets[i1]);
		}
		tail_first[t] = tf;
		span_len[t] = (tf == t)
			? int32_t(tile_of(tile_d, ntiles, i1 + offsets[i1 + 1]) - t + 1) : 0;
	}
}

int merge_plan_segmented(alpb_spmv_plan_s *p, const int64_t *offsets, int64_t nseg,
	const int64_t *seg_rows, SegmentedTiles *st, cudaStream_t s) {
	st->nseg = nseg;
	double maxlen = 0, sumsq = 0;
	int rc = row_profile(offsets, p->m, &maxlen, &sumsq, s);
	if (rc != ALPB_SUCCESS) return rc;
	const int64_t rpt = aligned_rows_per_tile(maxlen, p->m ? double(p->nnz) / double(p->m) : 0.0,
		WM_TILE);
	ALPB_CUDA(cudaMalloc(&st->seg_tile, size_t(nseg + 1) * 8));
	int64_t *counts = nullptr;
	int32_t *empty = nullptr;
	void *tmp = nullptr;
	size_t tb = 0;
	ALPB_CUDA(cudaMallocAsync(&counts, size_t(nseg + 1) * 8, s));
	ALPB_CUDA(cudaMallocAsync(&empty, 4, s));
	ALPB_CUDA(cudaMemsetAsync(empty, 0, 4, s));
	k_seg_tile_counts<<<grid_for(nseg + 1, 256), 256, 0, s>>>(offsets, seg_rows, nseg, counts,
		WM_TILE, rpt, empty);
	ALPB_LAUNCHED();
	ALPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, counts, st->seg_tile, nseg + 1, s));
	ALPB_CUDA(cudaMallocAsync(&tmp, tb, s));
	ALPB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, counts, st->seg_tile, nseg + 1, s));
	g_launches.fetch_add(1);
	int64_t nt = 0;
	int32_t h_empty = 0;
	ALPB_CUDA(cudaMemcpyAsync(&nt, st->seg_tile + nseg, 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaMemcpyAsync(&h_empty, empty, 4, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaFreeAsync(counts, s));
	ALPB_CUDA(cudaFreeAsync(empty, s));
	ALPB_CUDA(cudaFreeAsync(tmp, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	// an instance without rows would never finish its iterations
	ALPB_CHECK(h_empty == 0, ALPB_ILLEGAL, "segmented plan: an instance has no rows");
	ALPB_CHECK(nt > 0, ALPB_ILLEGAL, "segmented plan: no work");
	p->ntiles = nt;
	p->tile = WM_TILE;
	const size_t n = size_t(nt);
	ALPB_CUDA(cudaMalloc(&st->tile_d, (n + 1) * 8));
	ALPB_CUDA(cudaMalloc(&st->tile_seg, n * 4));
	ALPB_CUDA(cudaMalloc(&p->tile_row, (n + 1) * 8));
	ALPB_CUDA(cudaMalloc(&p->head_first, n * 8));
	ALPB_CUDA(cudaMalloc(&p->tail_first, n * 8));
	ALPB_CUDA(cudaMalloc(&p->span_len, n * 4));
	ALPB_CUDA(cudaMalloc(&p->counter, n * 4));
	ALPB_CUDA(cudaMalloc(&p->head_val, n * 8));
	ALPB_CUDA(cudaMalloc(&p->tail_val, n * 8));
	ALPB_CUDA(cudaMalloc(&p->head_has, n));
	ALPB_CUDA(cudaMalloc(&p->tail_has, n));
	ALPB_CUDA(cudaMalloc(&p->ready, n * 4));
	ALPB_CUDA(cudaMemsetAsync(p->counter, 0, n * 4, s));
	ALPB_CUDA(cudaMemsetAsync(p->ready, 0, n * 4, s));
	if (rpt) {
		k_seg_aligned<<<grid_for(nseg, 256), 256, 0, s>>>(offsets, seg_rows, st->seg_tile, nseg,
			p->m, p->nnz, rpt, st->tile_d, p->tile_row, st->tile_seg, p->head_first, p->tail_first,
			p->span_len);
		ALPB_LAUNCHED();
	} else {
		k_seg_tile_d<<<grid_for(nseg, 256), 256, 0, s>>>(offsets, seg_rows, st->seg_tile, nseg,
			p->m, p->nnz, st->tile_d, st->tile_seg, WM_TILE);
		ALPB_LAUNCHED();
		k_seg_tile_rows<<<grid_for(nt + 1, 256), 256, 0, s>>>(offsets, p->m, p->nnz, nt,
			st->tile_d, p->tile_row);
		ALPB_LAUNCHED();
		k_seg_tables<<<grid_for(nt, 256), 256, 0, s>>>(offsets, p->m, nt, st->tile_d, p->tile_row,
			p->head_first, p->tail_first, p->span_len);
		ALPB_LAUNCHED();
	}
	st->seg_rows = const_cast<int64_t *>(seg_rows);
	return ALPB_SUCCESS;
}

void segmented_free(SegmentedTiles *st) {
	cudaFree(st->seg_tile);
	cudaFree(st->tile_d);
	cudaFree(st->tile_seg);
	st->seg_tile = st->tile_d = nullptr;
	st->tile_seg = nullptr;
}

// ------------------------------------------------------------ batched CG --
struct BcgInst {       // per-instance device state
	double sigma, gamma, alpha, tol_abs, rr;
	int64_t iterations;
	int32_t done, converged;
	int32_t cnt;       // arrival counter of the instance's tiles (zero between phases)
	int32_t pad;
};

struct BcgArgs {
	MergeTables mt;                    // warp tiles cut per instance (tile_d)
	const int64_t *offsets;
	const uint32_t *indices;
	const double *values;
	const double *b;
	double *x, *r, *u0, *u1, *temp;
	double *own, *own2;                // [ntiles] per-tile partials
	const int32_t *tile_seg;           // [ntiles]
	const int64_t *seg_tile;           // [nseg+1]
	BcgInst *inst;                     // [nseg]
	int64_t nseg, max_iter;
	double tol;
	int32_t *active;                   // instances still iterating
	GridSync *gs;
	// sliced storage of short-row systems (slices of 32 rows of one instance;
	// entry q of the slice's lane-th row at sl_off[t] + 32 q + lane)
	const int64_t *sl_row;             // [nslices+1] first row of each slice
	const int64_t *sl_off;             // [nslices+1] first entry of each slice
	const uint32_t *sl_idx;
	const double *sl_val;
	const uint8_t *sl_len;             // [n] row lengths
};

constexpr int BCG_WARPS = 4;

struct BcgWarpSmem {
	WarpSmem<RF> tile;
	double p0[WM_TILE];
	double p1[WM_TILE];
};

struct BcgPrelude {
	const BcgArgs *a;
	BcgWarpSmem *sm;
	int64_t base = 0;
	double acc_rr = 0.0, acc_bb = 0.0;
	__device__ __forceinline__ void begin_tile(int64_t i0, int nrows, int lane) {
		base = i0;
		for (int k = lane; k < nrows; k += 32) sm->p0[k] = a->b[i0 + k];
	}
	__device__ __forceinline__ void row(int64_t i, double v, bool has) {
		const double t = has ? 0.0 + v : 0.0;
		const double bi = sm->p0[i - base];
		const double ri = (0.0 + bi) - t;
		a->r[i] = ri;
		a->u0[i] = 0.0;
		acc_rr += ri * ri;
		acc_bb += bi * bi;
	}
};

struct BcgGather {
	const double *r, *u_old;
	double gamma;
	__device__ __forceinline__ double operator()(uint32_t j) const {
		return __ldcg(r + j) + gamma * __ldcg(u_old + j);
	}
};

struct BcgIter {
	const BcgArgs *a;
	BcgWarpSmem *sm;
	const double *u_old;
	double *u_new;
	double gamma;
	int64_t base = 0;
	double acc = 0.0;
	__device__ __forceinline__ void begin_tile(int64_t i0, int nrows, int lane) {
		base = i0;
		for (int k = lane; k < nrows; k += 32) {
			sm->p0[k] = __ldcg(a->r + i0 + k);
			sm->p1[k] = __ldcg(u_old + i0 + k);
		}
	}
	__device__ __forceinline__ void row(int64_t i, double v, bool has) {
		const double t = has ? 0.0 + v : 0.0;
		a->temp[i] = t;
		const double un = sm->p0[i - base] + gamma * sm->p1[i - base];
		u_new[i] = un;
		acc += t * un;
	}
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		const double w = __shfl_xor_sync(0xffffffffu, v, o);
		v += w;
	}
	return v;
}

// Sum of the per-tile partials own[t0..t1) in a fixed order (lane-strided,
// then the xor tree), the same in every lane.
__device__ __forceinline__ double warp_sum_tiles(const double *own, int64_t t0, int64_t t1,
	int lane) {
	double v = 0.0;
	for (int64_t k = t0 + lane; k < t1; k += 32) v += __ldcg(own + k);
	return warp_sum(v);
}

// One slice (32 rows of one instance, at most 32 nonzeroes per row) of the
// sliced storage: lane l owns row sl_row[t] + l and sums its products in
// storage order (product rounded, then added: the order of the restated
// CG).  Entry q of all 32 rows is one contiguous line of indices and two of
// values, so every load is coalesced; the loads of NB entries are issued
// before their gathers and sums.
template <class XF, class RowF>
__device__ __forceinline__ void bcg_slice(const BcgArgs &a, int64_t t, int lane, const XF &xf,
	RowF &&row) {
	constexpr int NB = 4;
	const int64_t r0 = __ldg(a.sl_row + t), r1 = __ldg(a.sl_row + t + 1);
	const int64_t e0 = __ldg(a.sl_off + t);
	const int w = int((__ldg(a.sl_off + t + 1) - e0) >> 5);
	const int64_t i = r0 + lane;
	const int len = i < r1 ? int(__ldg(a.sl_len + i)) : 0;
	double acc = 0.0;
	for (int q0 = 0; q0 < w; q0 += NB) {
		uint32_t j[NB];
		double v[NB], x[NB];
#pragma unroll
		for (int u = 0; u < NB; ++u) {
			const int q = q0 + u;
			const int64_t e = e0 + 32 * int64_t(q) + lane;
			j[u] = q < w ? __ldcs(a.sl_idx + e) : 0u;
			v[u] = q < w ? __ldcs(a.sl_val + e) : 0.0;
		}
#pragma unroll
		for (int u = 0; u < NB; ++u) x[u] = q0 + u < len ? xf(j[u]) : 0.0;
#pragma unroll
		for (int u = 0; u < NB; ++u)
			if (q0 + u < len) acc = __dadd_rn(acc, __dmul_rn(v[u], x[u]));
	}
	if (i < r1) row(i, acc);
}

// Sum of the per-tile partials own[t0..t1) by a whole block, in a fixed
// order (eight interleaved accumulators per thread, then the block tree), the
// same in every thread.  One block per instance keeps the scalar steps short
// for the largest instances (thousands of tiles).
__device__ __forceinline__ double block_sum_tiles(const double *own, int64_t t0, int64_t t1,
	double *red) {
	const int64_t nth = blockDim.x;
	double v[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
	int64_t k = t0 + threadIdx.x;
	for (; k + 7 * nth < t1; k += 8 * nth) {
#pragma unroll
		for (int u = 0; u < 8; ++u) v[u] += __ldcg(own + k + u * nth);
	}
	for (; k < t1; k += nth) v[0] += __ldcg(own + k);
	return block_sum(((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7])), red);
}

// The instance of tile t and its state for the current phase, fetched one
// tile ahead by the phase loops.
struct BcgTileState {
	int32_t seg = 0;
	int32_t done = 1;
	double scalar = 0.0;  // gamma in phase A, alpha in phase B
};

template <bool ALPHA>
__device__ __forceinline__ BcgTileState bcg_tile_state(const BcgArgs &a, int64_t t) {
	BcgTileState st;
	if (t < a.mt.ntiles) {
		st.seg = __ldg(a.tile_seg + t);
		const BcgInst *in = a.inst + st.seg;
		st.done = __ldcg(&in->done);
		st.scalar = ALPHA ? __ldcg(&in->alpha) : __ldcg(&in->gamma);
	}
	return st;
}

// Tiles of the instances still iterating, rebuilt by every block after each
// convergence step (done flags change only there): the active instances in
// increasing order and the exclusive prefix of their tile counts, so a warp's
// work items k = gw, gw + nw, ... map to increasing tiles and converged
// instances cost nothing.  Up to BCG_LIST_MAX instances; more use the walk
// over all tiles.
constexpr int BCG_LIST_MAX = 1024;
constexpr int BCG_RB = 4;    // rows per lane whose loads phase B issues together
#ifndef ALPB_BCG_ROWS_MINB
#define ALPB_BCG_ROWS_MINB 8   // resident blocks per SM of the row-aligned variant
#endif

struct BcgList {
	int32_t n;                         // active instances
	int32_t seg[BCG_LIST_MAX];
	int32_t off[BCG_LIST_MAX + 1];     // tile prefix; off[n] = active tiles
};

__device__ void bcg_build_list(const BcgArgs &a, BcgList &L, int32_t *scan) {
	const int nseg = int(a.nseg), nth = blockDim.x, tid = threadIdx.x;
	const int per = (nseg + nth - 1) / nth;
	const int s0 = tid * per, s1 = s0 + per < nseg ? s0 + per : nseg;
	int ci = 0, ct = 0;
	for (int s = s0; s < s1; ++s) {
		if (!__ldcg(&a.inst[s].done)) {
			++ci;
			ct += int(a.seg_tile[s + 1] - a.seg_tile[s]);
		}
	}
	// block exclusive scan of (ci, ct) in thread order
	scan[tid] = ci;
	scan[nth + tid] = ct;
	__syncthreads();
	for (int o = 1; o < nth; o <<= 1) {
		const int vi = tid >= o ? scan[tid - o] : 0;
		const int vt = tid >= o ? scan[nth + tid - o] : 0;
		__syncthreads();
		scan[tid] += vi;
		scan[nth + tid] += vt;
		__syncthreads();
	}
	int pi = scan[tid] - ci, pt = scan[nth + tid] - ct;
	for (int s = s0; s < s1; ++s) {
		if (!__ldcg(&a.inst[s].done)) {
			L.seg[pi] = s;
			L.off[pi] = pt;
			++pi;
			pt += int(a.seg_tile[s + 1] - a.seg_tile[s]);
		}
	}
	if (tid == nth - 1) {
		L.n = scan[tid];
		L.off[scan[tid]] = scan[nth + tid];
	}
	__syncthreads();
}

// Work item k of the active list -> tile and instance; j is the caller's
// cursor into the list (items are visited in increasing order).
__device__ __forceinline__ int64_t bcg_item_tile(const BcgArgs &a, const BcgList &L, int32_t k,
	int &j, int32_t &seg) {
	while (L.off[j + 1] <= k) ++j;
	seg = L.seg[j];
	return a.seg_tile[seg] + (k - L.off[j]);
}

// Each iteration: phase A (tiles: temp = A u_new, u_new, beta terms) |
// per-instance alpha | phase B (rows: x, r, r.r terms) | per-instance
// convergence, gamma; a grid barrier after each.  Per-tile partials are
// reduced per instance by one warp in a fixed order (deterministic).
struct BcgNoSmem {};
template <bool ROWS> struct BcgTileSmem { typedef BcgWarpSmem type[BCG_WARPS]; };
template <> struct BcgTileSmem<true> { typedef BcgNoSmem type[1]; };

// ROWS: every tile is row-aligned (the plan's tile_d), so all phases run the
// lane-per-row code and the merge engine's staging memory is not needed.
template <bool LIST, bool ROWS>
__global__ void __launch_bounds__(32 * BCG_WARPS, ROWS ? ALPB_BCG_ROWS_MINB : (LIST ? 5 : 6))
k_batched_cg(BcgArgs a) {
	__shared__ typename BcgTileSmem<ROWS>::type sm;
	__shared__ BcgList L;
	__shared__ int32_t scan[2 * 32 * BCG_WARPS];
	__shared__ double red[33];
	const int64_t G = gridDim.x, nt = a.mt.ntiles;
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int64_t gw = int64_t(blockIdx.x) * BCG_WARPS + w, nw = G * BCG_WARPS;
	int *err = &a.gs->err;
	if constexpr (!ROWS) {
		for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < nt;
			 t += G * blockDim.x)
			a.mt.ready[t] = 0;
	}
	if (!grid_sync(a.gs)) return;
	int32_t epoch = 1;

	// prelude per instance: r = b - A x, sigma = r.r, tol * ||b||
	if constexpr (ROWS) {
		for (int64_t t = gw; t < nt; t += nw) {
			double rr = 0.0, bb = 0.0;
			bcg_slice(a, t, lane, [&](uint32_t j) { return __ldcg(a.x + j); },
				[&](int64_t i, double v) {
					const double bi = a.b[i];
					const double ri = (0.0 + bi) - v;
					a.r[i] = ri;
					a.u0[i] = 0.0;
					rr += ri * ri;
					bb += bi * bi;
				});
			const double s1 = warp_sum(rr), s2 = warp_sum(bb);
			if (lane == 0) {
				a.own[t] = s1;
				a.own2[t] = s2;
			}
		}
	} else {
		PlainX<double> xl{a.x};
		for (int64_t t = gw; t < nt; t += nw) {
			BcgPrelude epi{&a, &sm[w]};
			const WmMeta g = wm_meta(a.mt, t);
			if (!warp_tile_ordered<RF, PlainX<double>, BcgPrelude, 0>(t, g, a.mt, a.offsets,
					a.indices, a.values, xl, epi, 0, sm[w].tile, epoch, err))
				break;
			const double s1 = warp_sum(epi.acc_rr), s2 = warp_sum(epi.acc_bb);
			if (lane == 0) {
				a.own[t] = s1;
				a.own2[t] = s2;
			}
		}
	}
	if (!grid_sync(a.gs)) return;
	for (int64_t s = blockIdx.x; s < a.nseg; s += G) {
		BcgInst *in = a.inst + s;
		const double sigma = block_sum_tiles(a.own, a.seg_tile[s], a.seg_tile[s + 1], red);
		const double bnorm = block_sum_tiles(a.own2, a.seg_tile[s], a.seg_tile[s + 1], red);
		if (threadIdx.x == 0) {
			in->sigma = sigma;
			in->gamma = 0.0;
			in->tol_abs = a.tol * sqrt(bnorm);
			in->iterations = 0;
			in->done = 0;
			in->converged = 0;
		}
	}
	if (!grid_sync(a.gs)) return;

	int64_t iter = 0;
	double *u_old = a.u0, *u_new = a.u1;
	if (LIST) bcg_build_list(a, L, scan);
	for (;;) {
		++iter;
		++epoch;
		// phase A over the tiles of active instances
		if constexpr (LIST) {
			const int32_t ntot = L.off[L.n];
			int j = 0, jn = 0;
			int32_t seg = 0, segn = 0;
			int32_t k = int32_t(gw);
			int64_t t = k < ntot ? bcg_item_tile(a, L, k, j, seg) : nt;
			WmMeta g = ROWS ? WmMeta{0, 0, -1, -1} : wm_meta(a.mt, t);
			double gamma = k < ntot ? __ldcg(&a.inst[seg].gamma) : 0.0;
			while (k < ntot) {
				const int32_t kn = k + int32_t(nw);
				jn = j;
				const int64_t tn = kn < ntot ? bcg_item_tile(a, L, kn, jn, segn) : nt;
				const WmMeta gn = ROWS ? WmMeta{0, 0, -1, -1} : wm_meta(a.mt, tn);
				const double gamman = kn < ntot && segn != seg ? __ldcg(&a.inst[segn].gamma) : gamma;
				double part;
				if constexpr (ROWS) {
					double acc = 0.0;
					bcg_slice(a, t, lane,
						[&](uint32_t j) { return __ldcg(a.r + j) + gamma * __ldcg(u_old + j); },
						[&](int64_t i, double v) {
							a.temp[i] = v;
							const double un = __ldcg(a.r + i) + gamma * __ldcg(u_old + i);
							u_new[i] = un;
							acc += v * un;
						});
					part = warp_sum(acc);
				} else {
					BcgIter epi{&a, &sm[w], u_old, u_new, gamma};
					BcgGather xl{a.r, u_old, gamma};
					if (!warp_tile_ordered<RF, BcgGather, BcgIter, 0>(t, g, a.mt, a.offsets,
							a.indices, a.values, xl, epi, 0, sm[w].tile, epoch, err))
						break;
					part = warp_sum(epi.acc);
				}
				if (lane == 0) a.own[t] = part;
				k = kn;
				j = jn;
				seg = segn;
				t = tn;
				g = gn;
				gamma = gamman;
			}
		} else {
			int64_t t = gw;
			BcgTileState cur = bcg_tile_state<false>(a, t);
			WmMeta g = wm_meta(a.mt, t);
			while (t < nt) {
				const BcgTileState nxt = bcg_tile_state<false>(a, t + nw);
				const WmMeta gn = wm_meta(a.mt, t + nw);
				if (!cur.done) {
					BcgIter epi{&a, &sm[w], u_old, u_new, cur.scalar};
					BcgGather xl{a.r, u_old, cur.scalar};
					if (!warp_tile_ordered<RF, BcgGather, BcgIter, 0>(t, g, a.mt, a.offsets,
							a.indices, a.values, xl, epi, 0, sm[w].tile, epoch, err))
						break;
					const double part = warp_sum(epi.acc);
					if (lane == 0) a.own[t] = part;
				}
				t += nw;
				cur = nxt;
				g = gn;
			}
		}
		if (!grid_sync(a.gs)) return;
		for (int64_t j = blockIdx.x; j < (LIST ? int64_t(L.n) : a.nseg); j += G) {
			const int64_t s = LIST ? L.seg[j] : j;
			BcgInst *in = a.inst + s;
			if (!LIST && __ldcg(&in->done)) continue;
			const double beta = block_sum_tiles(a.own, a.seg_tile[s], a.seg_tile[s + 1], red);
			if (threadIdx.x == 0) in->alpha = in->sigma / beta;
		}
		if (!grid_sync(a.gs)) return;
		// phase B: the rows that end in each active tile
		if constexpr (ROWS) {
			// one row per lane and slice: PB slices per step, their loads together
			constexpr int PB = 4;
			const int32_t ntot = L.off[L.n];
			int j = 0;
			for (int32_t k0 = int32_t(gw); k0 < ntot; k0 += PB * int32_t(nw)) {
				int64_t tt[PB], ii[PB];
				double al[PB], xv[PB], uv[PB], rv[PB], tv[PB];
				bool ok[PB];
#pragma unroll
				for (int u = 0; u < PB; ++u) {
					const int32_t k = k0 + u * int32_t(nw);
					ok[u] = false;
					tt[u] = 0;
					if (k < ntot) {
						int32_t sg;
						tt[u] = bcg_item_tile(a, L, k, j, sg);
						al[u] = __ldcg(&a.inst[sg].alpha);
						ii[u] = __ldg(a.sl_row + tt[u]) + lane;
						ok[u] = ii[u] < __ldg(a.sl_row + tt[u] + 1);
					}
				}
#pragma unroll
				for (int u = 0; u < PB; ++u) {
					if (ok[u]) {
						xv[u] = __ldcg(a.x + ii[u]);
						uv[u] = __ldcg(u_new + ii[u]);
						rv[u] = __ldcg(a.r + ii[u]);
						tv[u] = __ldcg(a.temp + ii[u]);
					}
				}
#pragma unroll
				for (int u = 0; u < PB; ++u) {
					double part = 0.0;
					if (ok[u]) {
						a.x[ii[u]] = xv[u] + al[u] * uv[u];
						const double ri = rv[u] - al[u] * tv[u];
						a.r[ii[u]] = ri;
						part = ri * ri;
					}
					if (k0 + u * int32_t(nw) < ntot) {
						part = warp_sum(part);
						if (lane == 0) a.own[tt[u]] = part;
					}
				}
			}
		} else if constexpr (LIST) {
			const int32_t ntot = L.off[L.n];
			int j = 0;
			int32_t seg = -1, sg = 0;
			double alpha = 0.0;
			for (int32_t k = int32_t(gw); k < ntot; k += int32_t(nw)) {
				const int64_t t = bcg_item_tile(a, L, k, j, sg);
				if (sg != seg) {
					seg = sg;
					alpha = __ldcg(&a.inst[seg].alpha);
				}
				double part = 0.0;
				const int64_t r0 = ROWS ? a.sl_row[t] : a.mt.tile_row[t];
				const int64_t r1 = ROWS ? a.sl_row[t + 1] : a.mt.tile_row[t + 1];
				for (int64_t i0 = r0; i0 < r1; i0 += 32 * BCG_RB) {
					double xv[BCG_RB], uv[BCG_RB], rv[BCG_RB], tv[BCG_RB];
#pragma unroll
					for (int q = 0; q < BCG_RB; ++q) {
						const int64_t i = i0 + lane + 32 * q;
						if (i < r1) {
							xv[q] = __ldcg(a.x + i);
							uv[q] = __ldcg(u_new + i);
							rv[q] = __ldcg(a.r + i);
							tv[q] = __ldcg(a.temp + i);
						}
					}
#pragma unroll
					for (int q = 0; q < BCG_RB; ++q) {
						const int64_t i = i0 + lane + 32 * q;
						if (i < r1) {
							a.x[i] = xv[q] + alpha * uv[q];
							const double ri = rv[q] - alpha * tv[q];
							a.r[i] = ri;
							part += ri * ri;
						}
					}
				}
				part = warp_sum(part);
				if (lane == 0) a.own[t] = part;
			}
		} else {
			int64_t t = gw;
			BcgTileState cur = bcg_tile_state<true>(a, t);
			while (t < nt) {
				const BcgTileState nxt = bcg_tile_state<true>(a, t + nw);
				if (!cur.done) {
					const double alpha = cur.scalar;
					double part = 0.0;
					const int64_t r0 = a.mt.tile_row[t], r1 = a.mt.tile_row[t + 1];
					for (int64_t i = r0 + lane; i < r1; i += 32) {
						a.x[i] = a.x[i] + alpha * __ldcg(u_new + i);
						const double ri = __ldcg(a.r + i) - alpha * __ldcg(a.temp + i);
						a.r[i] = ri;
						part += ri * ri;
					}
					part = warp_sum(part);
					if (lane == 0) a.own[t] = part;
				}
				t += nw;
				cur = nxt;
			}
		}
		if (!grid_sync(a.gs)) return;
		for (int64_t j = blockIdx.x; j < (LIST ? int64_t(L.n) : a.nseg); j += G) {
			const int64_t s = LIST ? L.seg[j] : j;
			BcgInst *in = a.inst + s;
			if (!LIST && __ldcg(&in->done)) continue;
			const double rr = block_sum_tiles(a.own, a.seg_tile[s], a.seg_tile[s + 1], red);
			if (threadIdx.x == 0) {
				in->rr = rr;
				in->iterations = iter;
				if (sqrt(rr) < in->tol_abs || iter >= a.max_iter) {
					in->converged = sqrt(rr) < in->tol_abs ? 1 : 0;
					in->done = 1;
					atomicSub(a.active, 1);
				} else {
					in->gamma = rr / in->sigma;
					in->sigma = rr;
				}
			}
		}
		if (!grid_sync(a.gs)) return;
		if (((volatile int32_t *) a.active)[0] == 0) break;
		if (LIST) bcg_build_list(a, L, scan);
		double *tmp = u_old;
		u_old = u_new;
		u_new = tmp;
	}
}


// ------------------------------------ sliced batched CG, two barriers --
// Systems whose rows hold at most 32 nonzeroes, on the sliced storage (slices
// of 32 rows of one instance, entry q of the slice's rows contiguous).  One
// CG iteration of every active instance is
//     phase A (products) | grid barrier | phase B (updates) | grid barrier |
//     scalar step (no barrier of its own)
// Work split: the active instances' slices, in instance order, are cut in ONE
// contiguous run per warp (warp g of nw takes items [ntot g / nw,
// ntot (g+1) / nw)), so a warp streams consecutive slices and rows.  A block
// leaves one partial per instance its warps' runs touch (the warps' partials
// added in warp order), in slot slot0[j] + b - (first block of instance j);
// an instance's sum is the sum of its slots in slot order, formed by whoever
// needs it -- the same slots in the same order, hence the same bits
// everywhere.  So the phase-B warps form alpha themselves,
// and after the second barrier every block forms every active instance's r.r,
// convergence test, gamma and sigma in its own shared memory (identical in
// all blocks) and rebuilds its active list; block 0 publishes the results.
// The search direction travels with the residual as a 16-byte pair (r_i,
// p_i), double-buffered by iteration: a product gathers ONE pair per nonzero
// and forms p_j = r_j + gamma p_j(old); phase B forms p_i the same way (same
// operands, same bits), updates x and r and writes the next pair.  Per row
// the arithmetic is that of k_batched_cg and of the single-system solver;
// only the grouping of the instance dot products differs.
#ifndef ALPB_BCS_WARPS
#define ALPB_BCS_WARPS 8
#endif
#ifndef ALPB_BCS_MINB
#define ALPB_BCS_MINB 3
#endif
#ifndef ALPB_BCS_WMAX
#define ALPB_BCS_WMAX 6
#endif
#ifndef ALPB_BCS_RB
#define ALPB_BCS_RB 2
#endif
#ifndef ALPB_BCS_SU
#define ALPB_BCS_SU 4
#endif
constexpr int BCS_WARPS = ALPB_BCS_WARPS;  // warps per block (ALPB_BCS_MINB blocks per SM)
constexpr int BCS_WMAX = ALPB_BCS_WMAX;    // widest slice of the unrolled product path
constexpr int BCS_RB = ALPB_BCS_RB;        // rows per lane whose loads phase B issues together
constexpr int BCS_SU = ALPB_BCS_SU;        // instances whose slot sums a warp forms together
// Slices per warp at least, when fewer than all warps suffice (the tail, when
// few instances are left): measured 18.42 ms with 1 or 2, 18.94 ms with 8.
#ifndef ALPB_BCS_MINRUN
#define ALPB_BCS_MINRUN 2
#endif
constexpr int32_t BCS_MINRUN = ALPB_BCS_MINRUN;

struct BcsArgs {
	const int64_t *seg_rows;       // [nseg+1]
	const int64_t *seg_slice;      // [nseg+1]
	const int64_t *sl_off;         // [nslices+1]
	const uint32_t *sl_idx;
	const double *sl_val;
	const uint8_t *sl_len;         // [n]
	const double *b;
	double *x;
	double2 *pair[2];              // (r_i, p_i) of the current / next iteration
	double *temp;                  // A p
	double *slot_a, *slot_b;       // per-(warp, instance) partials
	BcgInst *inst;
	int64_t nseg, max_iter;
	double tol;
	GridSync *gs;
};

struct BcsShared {
	int32_t n;                             // active instances
	int32_t ntot;                          // their slices
	int64_t nwe;                           // warps with a run (at most ntot / BCS_MINRUN)
	int32_t seg[BCG_LIST_MAX];
	int32_t off[BCG_LIST_MAX + 1];         // slice prefix of the active instances
	int32_t slot0[BCG_LIST_MAX + 1];       // first partial slot of each
	int32_t nsl[BCG_LIST_MAX];             // slices of every instance
	double sigma[BCG_LIST_MAX], gamma[BCG_LIST_MAX], tol_abs[BCG_LIST_MAX];
	uint8_t done[BCG_LIST_MAX];
	int32_t scan[32];
	// partials of the first and the last instance of each warp's run (the
	// ones a neighbouring warp may share), combined per block in warp order
	int32_t edge_j[BCS_WARPS][2];
	double2 edge_v[BCS_WARPS][2];
};

// first item of warp g's run
__device__ __forceinline__ int64_t bcs_kb(int64_t ntot, int64_t g, int64_t nw) {
	return ntot * g / nw;
}
// warp whose run holds item k: the largest g with bcs_kb(g) <= k
__device__ __forceinline__ int64_t bcs_warp_of(int64_t ntot, int64_t k, int64_t nw) {
	return ((k + 1) * nw - 1) / ntot;
}

// block whose warps' runs hold item k
__device__ __forceinline__ int64_t bcs_block_of(int64_t ntot, int64_t k, int64_t nw) {
	return bcs_warp_of(ntot, k, nw) / BCS_WARPS;
}

// block-wide exclusive scan of one int per thread (thread order); returns
// the thread's prefix, *total the sum.  buf: one int per warp.
__device__ __forceinline__ int32_t bcs_scan(int32_t v, int32_t *buf, int32_t *total) {
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	const int nwarps = int(blockDim.x + 31) >> 5;
	int32_t x = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
		if (lane >= o) x += y;
	}
	if (lane == 31) buf[wid] = x;
	__syncthreads();
	if (wid == 0) {
		int32_t t = lane < nwarps ? buf[lane] : 0;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int32_t y = __shfl_up_sync(0xffffffffu, t, o);
			if (lane >= o) t += y;
		}
		if (lane < nwarps) buf[lane] = t;
	}
	__syncthreads();
	const int32_t before = wid > 0 ? buf[wid - 1] : 0;
	*total = buf[nwarps - 1];
	__syncthreads();  // buf is reused by the next scan
	return before + x - v;
}

// Active list of the instances not done, their slice prefix and their slot
// layout for nw warps; identical in every block.
__device__ __noinline__ void bcs_build_list(BcsShared &S, int64_t nseg, int64_t nw) {
	const int tid = threadIdx.x, nth = blockDim.x;
	const int per = int((nseg + nth - 1) / nth);
	const int s0 = tid * per, s1 = s0 + per < int(nseg) ? s0 + per : int(nseg);
	int32_t ci = 0, ct = 0;
	for (int s = s0; s < s1; ++s)
		if (!S.done[s]) {
			++ci;
			ct += S.nsl[s];
		}
	int32_t ni, ntot;
	int32_t pi = bcs_scan(ci, S.scan, &ni);
	int32_t pt = bcs_scan(ct, S.scan, &ntot);
	for (int s = s0; s < s1; ++s)
		if (!S.done[s]) {
			S.seg[pi] = s;
			S.off[pi] = pt;
			++pi;
			pt += S.nsl[s];
		}
	if (tid == 0) {
		S.n = ni;
		S.ntot = ntot;
		S.off[ni] = ntot;
		const int64_t want = (int64_t(ntot) + BCS_MINRUN - 1) / BCS_MINRUN;
		S.nwe = nw < want ? nw : want;
	}
	__syncthreads();
	// slots: one per block whose warps touch instance j (every active
	// instance has at least one slice, so at least one warp; with nwe warps
	// every run holds at least one item, so each block from the instance's
	// first to its last writes its slot)
	nw = S.nwe;
	const int pj = (ni + nth - 1) / nth;
	const int j0 = tid * pj, j1 = j0 + pj < ni ? j0 + pj : ni;
	int32_t cs = 0;
	for (int j = j0; j < j1; ++j)
		cs += int32_t(bcs_block_of(ntot, S.off[j + 1] - 1, nw) - bcs_block_of(ntot, S.off[j], nw) + 1);
	int32_t nslots;
	int32_t ps = bcs_scan(cs, S.scan, &nslots);
	for (int j = j0; j < j1; ++j) {
		S.slot0[j] = ps;
		ps += int32_t(bcs_block_of(ntot, S.off[j + 1] - 1, nw) - bcs_block_of(ntot, S.off[j], nw) + 1);
	}
	if (tid == 0) S.slot0[ni] = nslots;
	__syncthreads();
}

// list entry holding item k (off[j] <= k < off[j+1])
__device__ __forceinline__ int bcs_find(const BcsShared &S, int64_t k) {
	int lo = 0, hi = S.n - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (S.off[mid] <= k) lo = mid; else hi = mid - 1;
	}
	return lo;
}

// sum of slots [a, b) in a fixed order, the same in every lane
__device__ __forceinline__ double bcs_slot_sum(const double *slots, int32_t a, int32_t b,
	int lane) {
	double v = 0.0;
	int32_t k = a + lane;
	for (; k + 7 * 32 < b; k += 8 * 32) {   // eight loads in flight, added in order
		double t[8];
#pragma unroll
		for (int u = 0; u < 8; ++u) t[u] = __ldcg(slots + k + 32 * u);
#pragma unroll
		for (int u = 0; u < 8; ++u) v += t[u];
	}
	for (; k < b; k += 32) v += __ldcg(slots + k);
	return warp_sum(v);
}

// The same sums for list entries j0 .. j0 + BCS_SU - 1 (those below S.n),
// their first loads issued together; out[u] in every lane.
__device__ __forceinline__ void bcs_slot_sums(const double *slots, const BcsShared &S, int j0,
	int lane, double *out) {
	double v[BCS_SU];
#pragma unroll
	for (int u = 0; u < BCS_SU; ++u) {
		v[u] = 0.0;
		if (j0 + u < S.n) {
			const int32_t a = S.slot0[j0 + u], b = S.slot0[j0 + u + 1];
			if (a + lane < b) v[u] = __ldcg(slots + a + lane);
		}
	}
#pragma unroll
	for (int u = 0; u < BCS_SU; ++u) {
		if (j0 + u < S.n) {
			const int32_t a = S.slot0[j0 + u], b = S.slot0[j0 + u + 1];
			int32_t k = a + lane + 32;
			for (; k + 7 * 32 < b; k += 8 * 32) {
				double t[8];
#pragma unroll
				for (int q = 0; q < 8; ++q) t[q] = __ldcg(slots + k + 32 * q);
#pragma unroll
				for (int q = 0; q < 8; ++q) v[u] += t[q];
			}
			for (; k < b; k += 32) v[u] += __ldcg(slots + k);
		}
		out[u] = warp_sum(v[u]);
	}
}

// Products of ns consecutive slices of one instance, the first at slice t0
// and row r0 (slice c holds rows r0 + 32c .. , up to the instance end rend):
// lane l of slice c computes row i = r0 + 32c + l as the sum, in storage order,
// of the rounded products (as the restated CG).  pre(i, valid) loads what the
// row epilogue needs before the gathers are issued; row(i, acc, pre) finishes
// the row.  The slices' entry offsets are fetched 32 slices at a time.
template <class XF, class PreF, class RowF>
__device__ __forceinline__ void bcs_products(const BcsArgs &a, int64_t t0, int64_t ns,
	int64_t r0, int64_t rend, int lane, const XF &xf, const PreF &pre, RowF &&row) {
	for (int64_t cb = 0; cb < ns; cb += 32) {
		const int cnt = ns - cb < 32 ? int(ns - cb) : 32;
		const int64_t my_off = lane < cnt ? __ldg(a.sl_off + t0 + cb + lane) : 0;
		const int64_t end_off = __ldg(a.sl_off + t0 + cb + cnt);
		// the column indices and row length of slice c (narrow slices only),
		// fetched one slice ahead so that they arrive while the slice before
		// gathers
		const auto fetch = [&](int c, uint32_t *j, int &len) {
			const int64_t e0 = __shfl_sync(0xffffffffu, my_off, c);
			const int64_t e1 = c + 1 < cnt ? __shfl_sync(0xffffffffu, my_off, c + 1) : end_off;
			const int w = int((e1 - e0) >> 5);
			const int64_t i = r0 + 32 * (cb + c) + lane;
			len = i < rend ? int(__ldg(a.sl_len + i)) : 0;
#pragma unroll
			for (int q = 0; q < BCS_WMAX; ++q)
				j[q] = q < w && w <= BCS_WMAX ? __ldcs(a.sl_idx + e0 + 32 * q + lane) : 0u;
		};
		uint32_t jn[BCS_WMAX];
		int lenn;
		fetch(0, jn, lenn);
		for (int c = 0; c < cnt; ++c) {
			uint32_t j[BCS_WMAX];
#pragma unroll
			for (int q = 0; q < BCS_WMAX; ++q) j[q] = jn[q];
			const int len = lenn;
			const int64_t e0 = __shfl_sync(0xffffffffu, my_off, c);
			const int64_t e1 = c + 1 < cnt ? __shfl_sync(0xffffffffu, my_off, c + 1) : end_off;
			const int w = int((e1 - e0) >> 5);
			const int64_t i = r0 + 32 * (cb + c) + lane;
			const bool valid = i < rend;
			if (c + 1 < cnt) fetch(c + 1, jn, lenn);
			double acc = 0.0;
			if (w <= BCS_WMAX) {
				double v[BCS_WMAX], g[BCS_WMAX];
#pragma unroll
				for (int q = 0; q < BCS_WMAX; ++q)
					v[q] = q < w ? __ldcs(a.sl_val + e0 + 32 * q + lane) : 0.0;
				const auto own = pre(i, valid);
#pragma unroll
				for (int q = 0; q < BCS_WMAX; ++q) g[q] = q < len ? xf(j[q]) : 0.0;
#pragma unroll
				for (int q = 0; q < BCS_WMAX; ++q)
					if (q < len) acc = __dadd_rn(acc, __dmul_rn(v[q], g[q]));
				if (valid) row(i, acc, own);
			} else {
				const auto own = pre(i, valid);
				for (int q0 = 0; q0 < w; q0 += 4) {
					uint32_t jj[4];
					double v[4], g[4];
#pragma unroll
					for (int u = 0; u < 4; ++u) {
						const int64_t e = e0 + 32 * int64_t(q0 + u) + lane;
						jj[u] = q0 + u < w ? __ldcs(a.sl_idx + e) : 0u;
						v[u] = q0 + u < w ? __ldcs(a.sl_val + e) : 0.0;
					}
#pragma unroll
					for (int u = 0; u < 4; ++u) g[u] = q0 + u < len ? xf(jj[u]) : 0.0;
#pragma unroll
					for (int u = 0; u < 4; ++u)
						if (q0 + u < len) acc = __dadd_rn(acc, __dmul_rn(v[u], g[u]));
				}
				if (valid) row(i, acc, own);
			}
		}
	}
}

// The warp's run, instance by instance: fn(j, s, k, e) for its items [k, e)
// of list entry j (instance s).  Warps from nwe on have none.
template <class F>
__device__ __forceinline__ void bcs_walk(const BcsShared &S, int64_t g, F &&fn) {
	const int64_t ntot = S.ntot, nw = S.nwe;
	if (g >= nw) return;
	int64_t k = bcs_kb(ntot, g, nw);
	const int64_t kend = bcs_kb(ntot, g + 1, nw);
	if (k >= kend) return;
	int j = bcs_find(S, k);
	while (k < kend) {
		const int64_t e = kend < S.off[j + 1] ? kend : S.off[j + 1];
		fn(j, S.seg[j], k, e);
		k = e;
		++j;
	}
}

// Convergence test of instance s after an iteration with residual r.r = rr
// (conjugate_gradient.hpp:437), then gamma and sigma for the next one; block
// 0 publishes the instance's state.
__device__ __forceinline__ void bcs_instance_step(const BcsArgs &a, BcsShared &S, int s,
	double rr, int64_t iter) {
	const bool fin = sqrt(rr) < S.tol_abs[s] || iter >= a.max_iter;
	if (blockIdx.x == 0) {
		BcgInst *in = a.inst + s;
		in->rr = rr;
		in->iterations = iter;
		if (fin) {
			in->converged = sqrt(rr) < S.tol_abs[s] ? 1 : 0;
			in->done = 1;
		}
	}
	if (fin) {
		S.done[s] = 1;
	} else {
		S.gamma[s] = rr / S.sigma[s];
		S.sigma[s] = rr;
	}
}

// The warp's run with one partial (or a pair of partials) per instance
// segment, fn(j, s, k, e) -> double2, reduced to one slot per (block,
// instance): an instance inside a warp's run (no other warp touches it) is
// written by the warp; the first and the last instance of each run go to the
// block's edge table, and thread 0 sums them in warp order.  Slot of
// (instance j, block b): slot0[j] + b - (first block of j).  ya: slots of
// the first partials, yb: of the second (null: none).  Every thread of the
// block calls this.
template <class F>
__device__ __forceinline__ void bcs_walk_slots(BcsShared &S, int64_t g, int lane, double *ya,
	double *yb, F &&fn) {
	const int w = threadIdx.x >> 5;
	const int64_t b = blockIdx.x;
	const auto slot = [&](int j) {
		return S.slot0[j] + int32_t(b - bcs_block_of(S.ntot, S.off[j], S.nwe));
	};
	// lane 0 keeps the latest segment in edge slot 1 until the next one shows
	// that it lay inside the run
	if (lane == 0) {
		S.edge_j[w][0] = -1;
		S.edge_j[w][1] = -1;
	}
	bool first = true;
	bcs_walk(S, g, [&](int j, int s, int64_t k, int64_t e) {
		const double2 v = fn(j, s, k, e);
		if (lane == 0) {
			if (first) {
				S.edge_j[w][0] = j;
				S.edge_v[w][0] = v;
			} else {
				const int jp = S.edge_j[w][1];
				if (jp >= 0) {
					const int32_t sl = slot(jp);
					ya[sl] = S.edge_v[w][1].x;
					if (yb) yb[sl] = S.edge_v[w][1].y;
				}
				S.edge_j[w][1] = j;
				S.edge_v[w][1] = v;
			}
		}
		first = false;
	});
	__syncthreads();
	if (threadIdx.x == 0) {
		int jc = -1;
		double2 acc = make_double2(0.0, 0.0);
		for (int u = 0; u < BCS_WARPS; ++u)
			for (int q = 0; q < 2; ++q) {
				const int j = S.edge_j[u][q];
				if (j < 0) continue;
				const double2 v = S.edge_v[u][q];
				if (j != jc) {
					if (jc >= 0) {
						const int32_t sl = slot(jc);
						ya[sl] = acc.x;
						if (yb) yb[sl] = acc.y;
					}
					jc = j;
					acc = v;
				} else {
					acc.x += v.x;
					acc.y += v.y;
				}
			}
		if (jc >= 0) {
			const int32_t sl = slot(jc);
			ya[sl] = acc.x;
			if (yb) yb[sl] = acc.y;
		}
	}
}

__global__ void __launch_bounds__(32 * BCS_WARPS, ALPB_BCS_MINB) k_bcg_sliced(BcsArgs a) {
	__shared__ BcsShared S;
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int64_t g = int64_t(blockIdx.x) * BCS_WARPS + w;
	const int64_t nw = int64_t(gridDim.x) * BCS_WARPS;
	for (int s = threadIdx.x; s < int(a.nseg); s += blockDim.x) {
		S.nsl[s] = int32_t(a.seg_slice[s + 1] - a.seg_slice[s]);
		S.done[s] = 0;
		S.gamma[s] = 0.0;
		if (blockIdx.x == 0) {
			BcgInst *in = a.inst + s;
			in->iterations = 0;
			in->done = 0;
			in->converged = 0;
		}
	}
	__syncthreads();
	bcs_build_list(S, a.nseg, nw);

	// prelude: r = b - A x, pairs (r, 0); partials r.r -> slot_a, b.b -> slot_b
	bcs_walk_slots(S, g, lane, a.slot_a, a.slot_b, [&](int j, int s, int64_t k, int64_t e) {
		const int64_t q0 = k - S.off[j];
		const int64_t R0 = __ldg(a.seg_rows + s), R1 = __ldg(a.seg_rows + s + 1);
		double rr = 0.0, bb = 0.0;
		bcs_products(a, __ldg(a.seg_slice + s) + q0, e - k, R0 + 32 * q0, R1, lane,
			[&](uint32_t c) { return __ldcg(a.x + c); },
			[&](int64_t i, bool valid) { return valid ? a.b[i] : 0.0; },
			[&](int64_t i, double v, double bi) {
				const double ri = (0.0 + bi) - v;
				a.pair[0][i] = make_double2(ri, 0.0);
				rr += ri * ri;
				bb += bi * bi;
			});
		return make_double2(warp_sum(rr), warp_sum(bb));
	});
	if (!grid_sync(a.gs)) return;
	for (int j0 = w * BCS_SU; j0 < S.n; j0 += BCS_WARPS * BCS_SU) {
		double sg[BCS_SU], bn[BCS_SU];
		bcs_slot_sums(a.slot_a, S, j0, lane, sg);
		bcs_slot_sums(a.slot_b, S, j0, lane, bn);
		if (lane == 0)
			for (int u = 0; u < BCS_SU && j0 + u < S.n; ++u) {
				const int s = S.seg[j0 + u];
				S.sigma[s] = sg[u];
				S.tol_abs[s] = a.tol * sqrt(bn[u]);
			}
	}
	__syncthreads();

	int cur = 0;
	for (int64_t iter = 1;; ++iter) {
		const double2 *pc = a.pair[cur];
		double2 *pn = a.pair[cur ^ 1];
		// phase A: temp = A p, partials p.(A p) -> slot_a
		bcs_walk_slots(S, g, lane, a.slot_a, nullptr, [&](int j, int s, int64_t k, int64_t e) {
			const int64_t q0 = k - S.off[j];
			const int64_t R0 = __ldg(a.seg_rows + s), R1 = __ldg(a.seg_rows + s + 1);
			const double gamma = S.gamma[s];
			double acc = 0.0;
			bcs_products(a, __ldg(a.seg_slice + s) + q0, e - k, R0 + 32 * q0, R1, lane,
				[&](uint32_t c) {
					const double2 p = __ldcg(pc + c);
					return p.x + gamma * p.y;
				},
				[&](int64_t i, bool valid) { return valid ? __ldcg(pc + i) : make_double2(0.0, 0.0); },
				[&](int64_t i, double v, double2 p) {
					a.temp[i] = v;
					const double un = p.x + gamma * p.y;
					acc += v * un;
				});
			return make_double2(warp_sum(acc), 0.0);
		});
		if (!grid_sync(a.gs)) return;
		// phase B: alpha from the instance's slots; x += alpha p, r -= alpha A p,
		// the next pairs; partials r.r -> slot_b
		bcs_walk_slots(S, g, lane, a.slot_b, nullptr, [&](int j, int s, int64_t k, int64_t e) {
			const double alpha = S.sigma[s] / bcs_slot_sum(a.slot_a, S.slot0[j], S.slot0[j + 1], lane);
			const double gamma = S.gamma[s];
			const int64_t q0 = k - S.off[j];
			const int64_t R0 = __ldg(a.seg_rows + s), R1 = __ldg(a.seg_rows + s + 1);
			const int64_t i0 = R0 + 32 * q0;
			int64_t i1 = R0 + 32 * (e - S.off[j]);
			if (i1 > R1) i1 = R1;
			double part = 0.0;
			for (int64_t ib = i0; ib < i1; ib += 32 * BCS_RB) {
				double2 p[BCS_RB];
				double xv[BCS_RB], tv[BCS_RB];
#pragma unroll
				for (int u = 0; u < BCS_RB; ++u) {
					const int64_t i = ib + lane + 32 * u;
					if (i < i1) {
						p[u] = __ldcg(pc + i);
						xv[u] = __ldcg(a.x + i);
						tv[u] = __ldcg(a.temp + i);
					}
				}
#pragma unroll
				for (int u = 0; u < BCS_RB; ++u) {
					const int64_t i = ib + lane + 32 * u;
					if (i < i1) {
						const double un = p[u].x + gamma * p[u].y;
						a.x[i] = xv[u] + alpha * un;
						const double ri = p[u].x - alpha * tv[u];
						pn[i] = make_double2(ri, un);
						part += ri * ri;
					}
				}
			}
			return make_double2(warp_sum(part), 0.0);
		});
		if (!grid_sync(a.gs)) return;
		// scalar step, in every block: r.r, convergence, gamma, sigma; a warp
		// takes BCS_SU instances at a time, their slot loads issued together
		for (int j0 = w * BCS_SU; j0 < S.n; j0 += BCS_WARPS * BCS_SU) {
			double rr[BCS_SU];
			bcs_slot_sums(a.slot_b, S, j0, lane, rr);
			if (lane < BCS_SU && j0 + lane < S.n) {
				double v = rr[0];
#pragma unroll
				for (int u = 1; u < BCS_SU; ++u)
					if (lane == u) v = rr[u];
				bcs_instance_step(a, S, S.seg[j0 + lane], v, iter);
			}
		}
		__syncthreads();
		bcs_build_list(S, a.nseg, nw);
		if (S.n == 0) break;
		cur ^= 1;
	}
}

} // namespace alpb

using namespace alpb;

// ------------------------------------------------ sliced storage (ELL-32) --
// Slices of 32 rows, cut per instance (the last slice of an instance may be
// short); a slice's width is its longest row.  Built once per handle from the
// CRS: the solver then reads entry q of 32 rows as one coalesced line.
__global__ void k_sell_slices(const int64_t *seg_rows, int64_t nseg, int64_t *count) {
	for (int64_t s = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; s <= nseg;
		 s += int64_t(gridDim.x) * blockDim.x)
		count[s] = s < nseg ? (seg_rows[s + 1] - seg_rows[s] + 31) / 32 : 0;
}

__global__ void k_sell_rows(const int64_t *seg_rows, const int64_t *seg_slice, int64_t nseg,
	int64_t *sl_row, int64_t nslices) {
	for (int64_t s = blockIdx.x; s < nseg; s += gridDim.x) {
		const int64_t t0 = seg_slice[s], t1 = seg_slice[s + 1], r0 = seg_rows[s];
		for (int64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) sl_row[t] = r0 + 32 * (t - t0);
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) sl_row[nslices] = seg_rows[nseg];
}

// one warp per slice: row lengths and the slice's entry count (32 x width)
__global__ void k_sell_width(const int64_t *offsets, const int64_t *sl_row, int64_t nslices,
	uint8_t *len, int64_t *count) {
	const int lane = threadIdx.x & 31;
	const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
	for (int64_t t = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; t <= nslices;
		 t += nw) {
		if (t == nslices) {
			if (lane == 0) count[t] = 0;
			continue;
		}
		const int64_t i = sl_row[t] + lane;
		int l = 0;
		if (i < sl_row[t + 1]) {
			l = int(offsets[i + 1] - offsets[i]);
			len[i] = uint8_t(l);
		}
		for (int o = 16; o > 0; o >>= 1) {
			const int v = __shfl_xor_sync(0xffffffffu, l, o);
			l = v > l ? v : l;
		}
		if (lane == 0) count[t] = 32 * int64_t(l);
	}
}

__global__ void k_sell_fill(const int64_t *offsets, const uint32_t *indices, const double *values,
	const int64_t *sl_row, const int64_t *sl_off, int64_t nslices, uint32_t *idx, double *val) {
	const int lane = threadIdx.x & 31;
	const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
	for (int64_t t = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; t < nslices;
		 t += nw) {
		const int64_t i = sl_row[t] + lane, e0 = sl_off[t];
		const int w = int((sl_off[t + 1] - e0) >> 5);
		const bool own = i < sl_row[t + 1];
		const int64_t kb = own ? offsets[i] : 0, l = own ? offsets[i + 1] - kb : 0;
		for (int q = 0; q < w; ++q) {
			const int64_t e = e0 + 32 * int64_t(q) + lane;
			idx[e] = q < l ? indices[kb + q] : 0u;
			val[e] = q < l ? values[kb + q] : 0.0;
		}
	}
}

struct alpb_batched_cg_s {
	alpb_spmv_plan_s plan;
	SegmentedTiles st;
	int64_t n = 0, nnz = 0, nseg = 0;
	const int64_t *offsets = nullptr;
	const uint32_t *indices = nullptr;
	const double *values = nullptr;
	double *work = nullptr;     // r, u0, u1, temp
	double *scratch = nullptr;  // own, own2
	BcgInst *inst = nullptr;
	int32_t *active = nullptr;
	GridSync *gs = nullptr;
	int grid = 0;
	bool list = false;          // active-tile list (nseg <= BCG_LIST_MAX)
	bool rows = false;          // sliced storage (rows of at most 32 nonzeroes)
	int64_t nslices = 0;
	int64_t *seg_slice = nullptr, *sl_row = nullptr, *sl_off = nullptr;
	uint32_t *sl_idx = nullptr;
	double *sl_val = nullptr;
	uint8_t *sl_len = nullptr;
	int64_t nslots = 0;         // partial slots of each kind (sliced solver)
	cudaGraphExec_t graph = nullptr;
	const double *g_b = nullptr;
	double *g_x = nullptr;
	int64_t g_max = 0;
	double g_tol = 0;
};

static int sell_build(alpb_batched_cg_s *h, const int64_t *seg_rows, cudaStream_t s) {
	const int64_t nseg = h->nseg;
	int64_t *cnt = nullptr;
	void *tmp = nullptr;
	size_t tb = 0;
	ALPB_CUDA(cudaMalloc(&h->seg_slice, size_t(nseg + 1) * 8));
	ALPB_CUDA(cudaMallocAsync(&cnt, size_t(nseg + 1) * 8, s));
	k_sell_slices<<<grid_for(nseg + 1, 256), 256, 0, s>>>(seg_rows, nseg, cnt);
	ALPB_LAUNCHED();
	ALPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, h->seg_slice, nseg + 1, s));
	ALPB_CUDA(cudaMallocAsync(&tmp, tb, s));
	ALPB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, h->seg_slice, nseg + 1, s));
	g_launches.fetch_add(1);
	ALPB_CUDA(cudaMemcpyAsync(&h->nslices, h->seg_slice + nseg, 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	ALPB_CUDA(cudaFreeAsync(cnt, s));
	ALPB_CUDA(cudaFreeAsync(tmp, s));
	const int64_t ns = h->nslices;
	ALPB_CUDA(cudaMalloc(&h->sl_row, size_t(ns + 1) * 8));
	ALPB_CUDA(cudaMalloc(&h->sl_off, size_t(ns + 1) * 8));
	ALPB_CUDA(cudaMalloc(&h->sl_len, size_t(h->n > 0 ? h->n : 1)));
	k_sell_rows<<<unsigned(nseg < 4096 ? nseg : 4096), 256, 0, s>>>(seg_rows, h->seg_slice, nseg,
		h->sl_row, ns);
	ALPB_LAUNCHED();
	ALPB_CUDA(cudaMallocAsync(&cnt, size_t(ns + 1) * 8, s));
	k_sell_width<<<grid_for((ns + 1) * 32, 256), 256, 0, s>>>(h->offsets, h->sl_row, ns, h->sl_len,
		cnt);
	ALPB_LAUNCHED();
	tb = 0;
	ALPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, h->sl_off, ns + 1, s));
	ALPB_CUDA(cudaMallocAsync(&tmp, tb, s));
	ALPB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, h->sl_off, ns + 1, s));
	g_launches.fetch_add(1);
	int64_t ne = 0;
	ALPB_CUDA(cudaMemcpyAsync(&ne, h->sl_off + ns, 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	ALPB_CUDA(cudaFreeAsync(cnt, s));
	ALPB_CUDA(cudaFreeAsync(tmp, s));
	ALPB_CUDA(cudaMalloc(&h->sl_idx, size_t(ne > 0 ? ne : 1) * 4));
	ALPB_CUDA(cudaMalloc(&h->sl_val, size_t(ne > 0 ? ne : 1) * 8));
	k_sell_fill<<<grid_for(ns * 32, 256), 256, 0, s>>>(h->offsets, h->indices, h->values, h->sl_row,
		h->sl_off, ns, h->sl_idx, h->sl_val);
	ALPB_LAUNCHED();
	ALPB_CUDA(cudaStreamSynchronize(s));
	return ALPB_SUCCESS;
}

__global__ void k_bcg_reset(GridSync *gs, int32_t *active, int32_t nseg) {
	gs->count = 0;
	gs->gen = 0;
	gs->err = 0;
	*active = nseg;
}

static int bcg_launch(alpb_batched_cg_s *h, const double *b, double *x, int64_t max_iter,
	double tol, cudaStream_t s) {
	// per-tile partials: as many as tiles or slices, whichever the solve uses
	const int64_t nt = h->plan.ntiles > h->nslices ? h->plan.ntiles : h->nslices;
	// kernels only (no host-memory copies), so the solve can be captured
	k_bcg_reset<<<1, 1, 0, s>>>(h->gs, h->active, int32_t(h->nseg));
	ALPB_LAUNCHED();
	BcgArgs a;
	a.mt = merge_tables(h->plan);
	a.mt.tile_d = h->st.tile_d;
	a.offsets = h->offsets;
	a.indices = h->indices;
	a.values = h->values;
	a.b = b;
	a.x = x;
	a.r = h->work;
	a.u0 = h->work + h->n;
	a.u1 = h->work + 2 * h->n;
	a.temp = h->work + 3 * h->n;
	a.own = h->scratch;
	a.own2 = h->scratch + nt;
	a.tile_seg = h->st.tile_seg;
	a.seg_tile = h->st.seg_tile;
	a.sl_row = h->sl_row;
	a.sl_off = h->sl_off;
	a.sl_idx = h->sl_idx;
	a.sl_val = h->sl_val;
	a.sl_len = h->sl_len;
	if (h->rows) {   // the slices are the tiles
		a.seg_tile = h->seg_slice;
		a.mt.ntiles = h->nslices;
	}
	a.inst = h->inst;
	a.nseg = h->nseg;
	a.max_iter = max_iter;
	a.tol = tol;
	a.active = h->active;
	a.gs = h->gs;
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(h->grid);
	cfg.blockDim = dim3(32 * BCG_WARPS);
	cfg.stream = s;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeCooperative;
	attr[0].val.cooperative = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	if (h->rows) {
		BcsArgs c;
		c.seg_rows = h->st.seg_rows;
		c.seg_slice = h->seg_slice;
		c.sl_off = h->sl_off;
		c.sl_idx = h->sl_idx;
		c.sl_val = h->sl_val;
		c.sl_len = h->sl_len;
		c.b = b;
		c.x = x;
		c.pair[0] = reinterpret_cast<double2 *>(h->work);
		c.pair[1] = reinterpret_cast<double2 *>(h->work + 2 * h->n);
		c.temp = h->work + 4 * h->n;
		c.slot_a = h->scratch;
		c.slot_b = h->scratch + h->nslots;
		c.inst = h->inst;
		c.nseg = h->nseg;
		c.max_iter = max_iter;
		c.tol = tol;
		c.gs = h->gs;
		cfg.blockDim = dim3(32 * BCS_WARPS);
		ALPB_CUDA(cudaLaunchKernelEx(&cfg, k_bcg_sliced, c));
	} else if (h->list) {
		ALPB_CUDA(cudaLaunchKernelEx(&cfg, k_batched_cg<true, false>, a));
	} else {
		ALPB_CUDA(cudaLaunchKernelEx(&cfg, k_batched_cg<false, false>, a));
	}
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

extern "C" {

int alpb_batched_cg_create(alpb_batched_cg *out, int64_t n, int64_t nnz, const int64_t *row_ptr,
	const uint32_t *col_idx, const double *values, int64_t nseg, const int64_t *seg_rows,
	void *stream) {
	ALPB_CHECK(out != nullptr, ALPB_ILLEGAL, "alpb_batched_cg_create: null handle");
	*out = nullptr;
	ALPB_CHECK(n > 0 && nnz >= 0 && nseg > 0 && nseg < (int64_t(1) << 31), ALPB_ILLEGAL,
		"alpb_batched_cg_create: bad sizes");
	ALPB_CHECK(n + nnz < (int64_t(1) << 31) * 1024, ALPB_OVERFLW, "alpb_batched_cg_create: too large");
	cudaStream_t s = as_stream(stream);
	auto *h = new alpb_batched_cg_s();
	h->n = n;
	h->nnz = nnz;
	h->nseg = nseg;
	h->offsets = row_ptr;
	h->indices = col_idx;
	h->values = values;
	h->plan.m = n;
	h->plan.nnz = nnz;
	h->plan.offsets = row_ptr;
	h->plan.sched = ALPB_SCHED_MERGE_PATH;
	int rc = merge_plan_segmented(&h->plan, row_ptr, nseg, seg_rows, &h->st, s);
	if (rc != ALPB_SUCCESS) {
		alpb_batched_cg_destroy(h);
		return rc;
	}
	int64_t nt = h->plan.ntiles;
	h->list = nseg <= BCG_LIST_MAX && nt < (int64_t(1) << 31);
	if (h->list && h->st.tile_d) {   // whole-row tiles: rows of at most 32 nonzeroes
		rc = sell_build(h, seg_rows, s);
		if (rc != ALPB_SUCCESS) {
			alpb_batched_cg_destroy(h);
			return rc;
		}
		h->rows = h->nslices < (int64_t(1) << 31);
		if (h->nslices > nt) nt = h->nslices;
	}
	if (h->rows)
		h->grid = solver_grid(k_bcg_sliced, 32 * BCS_WARPS, h->nslices, BCS_WARPS);
	else if (h->list)
		h->grid = solver_grid(k_batched_cg<true, false>, 32 * BCG_WARPS, nt, BCG_WARPS);
	else
		h->grid = solver_grid(k_batched_cg<false, false>, 32 * BCG_WARPS, nt, BCG_WARPS);
	if (h->grid <= 0) {
		alpb_batched_cg_destroy(h);
		set_error("alpb_batched_cg_create: no cooperative occupancy");
		return ALPB_PANIC;
	}
	// sliced solver: pairs (r, p) twice and A p; slots for every (warp,
	// instance) pair a run can make: at most one per warp plus one per instance
	h->nslots = h->rows ? int64_t(h->grid) * BCS_WARPS + nseg : 0;
	const int64_t nscratch = h->rows ? 2 * h->nslots : 2 * nt;
	if (cudaMalloc(&h->work, size_t((h->rows ? 5 : 4) * n) * 8) != cudaSuccess ||
		cudaMalloc(&h->scratch, size_t(nscratch) * 8) != cudaSuccess ||
		cudaMalloc(&h->inst, size_t(nseg) * sizeof(BcgInst)) != cudaSuccess ||
		cudaMalloc(&h->active, 8) != cudaSuccess || cudaMalloc(&h->gs, sizeof(GridSync)) != cudaSuccess) {
		cudaGetLastError();
		alpb_batched_cg_destroy(h);
		set_error("alpb_batched_cg_create: out of device memory");
		return ALPB_OUTOFMEM;
	}
	ALPB_CUDA(cudaMemsetAsync(h->inst, 0, size_t(nseg) * sizeof(BcgInst), s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	*out = h;
	return ALPB_SUCCESS;
}

int alpb_batched_cg_destroy(alpb_batched_cg h) {
	if (!h) return ALPB_SUCCESS;
	if (h->graph) cudaGraphExecDestroy(h->graph);
	segmented_free(&h->st);
	cudaFree(h->seg_slice);
	cudaFree(h->sl_row);
	cudaFree(h->sl_off);
	cudaFree(h->sl_idx);
	cudaFree(h->sl_val);
	cudaFree(h->sl_len);
	cudaFree(h->plan.tile_row);
	cudaFree(h->plan.head_first);
	cudaFree(h->plan.tail_first);
	cudaFree(h->plan.span_len);
	cudaFree(h->plan.counter);
	cudaFree(h->plan.head_val);
	cudaFree(h->plan.tail_val);
	cudaFree(h->plan.head_has);
	cudaFree(h->plan.tail_has);
	cudaFree(h->plan.ready);
	cudaFree(h->work);
	cudaFree(h->scratch);
	cudaFree(h->inst);
	cudaFree(h->active);
	cudaFree(h->gs);
	delete h;
	return ALPB_SUCCESS;
}

int alpb_batched_cg_solve(alpb_batched_cg h, const double *b, double *x, int64_t max_iter,
	double tol, void *stream) {
	ALPB_CHECK(h != nullptr, ALPB_ILLEGAL, "alpb_batched_cg_solve: null handle");
	ALPB_CHECK(tol > 0 && max_iter > 0, ALPB_ILLEGAL, "alpb_batched_cg_solve: bad tol/max_iter");
	return bcg_launch(h, b, x, max_iter, tol, as_stream(stream));
}

int alpb_batched_cg_capture(alpb_batched_cg h, const double *b, double *x, int64_t max_iter,
	double tol, void *stream) {
	ALPB_CHECK(h != nullptr, ALPB_ILLEGAL, "alpb_batched_cg_capture: null handle");
	ALPB_CHECK(tol > 0 && max_iter > 0, ALPB_ILLEGAL, "alpb_batched_cg_capture: bad tol/max_iter");
	cudaStream_t s = as_stream(stream);
	cudaStream_t cs;
	ALPB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
	cudaGraph_t g;
	ALPB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
	int rc = bcg_launch(h, b, x, max_iter, tol, cs);
	cudaError_t e = cudaStreamEndCapture(cs, &g);
	cudaStreamDestroy(cs);
	if (rc != ALPB_SUCCESS) return rc;
	ALPB_CUDA(e);
	if (h->graph) cudaGraphExecDestroy(h->graph);
	h->graph = nullptr;
	cudaError_t ie = cudaGraphInstantiate(&h->graph, g, 0);
	cudaGraphDestroy(g);
	ALPB_CUDA(ie);
	(void) s;
	return ALPB_SUCCESS;
}

int alpb_batched_cg_replay(alpb_batched_cg h, void *stream) {
	ALPB_CHECK(h != nullptr && h->graph != nullptr, ALPB_ILLEGAL,
		"alpb_batched_cg_replay: no captured solve");
	ALPB_CUDA(cudaGraphLaunch(h->graph, as_stream(stream)));
	g_launches.fetch_add(1);
	return ALPB_SUCCESS;
}

int alpb_batched_cg_results(alpb_batched_cg h, int64_t *iterations, double *residuals,
	int32_t *converged, void *stream) {
	ALPB_CHECK(h != nullptr, ALPB_ILLEGAL, "alpb_batched_cg_results: null handle");
	cudaStream_t s = as_stream(stream);
	std::vector<BcgInst> v(size_t(h->nseg));
	GridSync gs;
	ALPB_CUDA(cudaMemcpyAsync(v.data(), h->inst, v.size() * sizeof(BcgInst),
		cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaMemcpyAsync(&gs, h->gs, sizeof(GridSync), cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	ALPB_CHECK(gs.err == 0, ALPB_PANIC, "alpb_batched_cg: a grid barrier or tile wait timed out");
	int all = 1;
	for (size_t i = 0; i < v.size(); ++i) {
		if (iterations) iterations[i] = v[i].iterations;
		if (residuals) residuals[i] = v[i].rr;
		if (converged) converged[i] = v[i].converged;
		all &= v[i].converged;
	}
	return all ? ALPB_SUCCESS : ALPB_FAILED;
}

} // extern "C"
