// Merge-path tile engine shared by the standalone SpMV and the fused solvers.
//
// The merge list of a compressed storage is its m row-end items interleaved
// with its nnz nonzero items (row i's nonzeroes, then its row end).  Tile t
// owns the diagonals [t*TILE, (t+1)*TILE): at most TILE items, whatever the
// row lengths, so power-law rows cost the same as uniform ones (Merrill &
// Garland, SC'16).
//
// A row whose items all lie in one tile is finished inside that tile: the
// thread that consumes its row end calls Epi::row(r, sum, has).  A row that
// crosses tiles ("spanning") gets one partial per tile it touches, written
// to that tile's head or tail slot; each touching tile then bumps the row's
// arrival counter, and the last to arrive sums the slots in tile order and
// calls Epi::row_span.  No grid barrier and no second launch are needed, and
// every sum is formed in a fixed order: results are deterministic.
#pragma once
#include "common.cuh"
#include "spmv.cuh"

namespace alpb {

// Device view of a plan's merge tables (see alpb_spmv_plan_s).
struct MergeTables {
	int64_t m, nnz, ntiles;
	const int64_t *tile_row;   // [ntiles+1] rows consumed before each tile
	const int64_t *head_first; // [ntiles] first tile of the head row if it spans, else -1
	const int64_t *tail_first; // [ntiles] first tile of the tail row if it spans, else -1
	const int32_t *span_len;   // [ntiles] tiles covered by the spanning row starting here
	int32_t *counter;          // [ntiles] arrivals per spanning row (indexed by first tile)
	uint64_t *head_val;        // [ntiles] partial of the head row (ring value bits)
	uint64_t *tail_val;        // [ntiles] partial of the tail row
	uint8_t *head_has;
	uint8_t *tail_has;
	// [ntiles+1] first diagonal of each tile when tiles are cut per segment
	// (batched solves: no tile straddles two instances); null: t * MP_TILE
	const int64_t *tile_d = nullptr;
	// [ntiles] publication epochs of the tail partials (warp_tile_ordered)
	int32_t *ready = nullptr;
};

template <class T>
__device__ __forceinline__ void store_bits(uint64_t *p, T v) {
	*reinterpret_cast<T *>(p) = v;
}
template <class T>
__device__ __forceinline__ T load_bits(const uint64_t *p) {
	return *reinterpret_cast<const volatile T *>(p);
}

template <class R>
struct MergeSmem {
	typename R::T prod[MP_TILE];
	int32_t row_end[MP_TILE + 2];  // [k] = end of tile row k-1, relative to j0
	int32_t crow[MP_BLOCK];        // carry-out row of each thread (tile relative)
	typename R::T cval[MP_BLOCK];
	uint8_t chas[MP_BLOCK];
};

// Spanning row finisher: called by one thread after its tile's partial for
// row r is in its slot.  Returns true (and the full sum) for the last arrival.
template <class R>
__device__ __forceinline__ bool arrive(const MergeTables &mt, int64_t first, typename R::T &sum,
	bool &has) {
	using T = typename R::T;
	__threadfence();
	const int32_t n = mt.span_len[first];
	const int32_t prev = atomicAdd(mt.counter + first, 1);
	if (prev != n - 1) return false;
	__threadfence();
	mt.counter[first] = 0;  // ready for the next product with this plan
	T v = R::zero();
	bool h = false;
	for (int64_t k = first; k < first + n; ++k) {
		const bool is_last = (k == first + n - 1);
		const uint8_t kh = is_last ? ((volatile uint8_t *) mt.head_has)[k]
								   : ((volatile uint8_t *) mt.tail_has)[k];
		if (kh) {
			v = R::add(v, load_bits<T>(is_last ? mt.head_val + k : mt.tail_val + k));
			h = true;
		}
	}
	sum = v;
	has = h;
	return true;
}

// One tile of the merge path.  XL: functor `T operator()(uint32_t j)` giving
// the gathered input x_j.  Epi: `void row(int64_t r, T sum, bool has)` for a
// row finished inside the tile and `void row_span(int64_t first, int64_t r,
// T sum, bool has)` for a spanning row (first = its first tile), so that
// fused epilogues can attribute reduction terms to a fixed tile.
// `left` selects mul(x, a) (vxm) instead of mul(a, x) (mxv).
template <class R, class XL, class Epi>
__device__ __forceinline__ void merge_tile(int64_t t, const MergeTables &mt,
	const int64_t *__restrict__ offsets, const uint32_t *__restrict__ indices,
	const typename R::T *__restrict__ values, const XL &xl, Epi &epi, int left,
	MergeSmem<R> &sm) {
	using T = typename R::T;
	const int tid = threadIdx.x;
	const int64_t m = mt.m, nnz = mt.nnz;
	const int64_t i0 = mt.tile_row[t], i1 = mt.tile_row[t + 1];
	int64_t d0, d1;
	if (mt.tile_d) {
		d0 = mt.tile_d[t];
		d1 = mt.tile_d[t + 1];
	} else {
		d0 = t * MP_TILE;
		d1 = d0 + MP_TILE;
		if (d1 > m + nnz) d1 = m + nnz;
	}
	const int64_t j0 = d0 - i0, j1 = d1 - i1;
	const int nrows = int(i1 - i0);
	const int nnzt = int(j1 - j0);

	for (int k = tid; k <= nrows + 1; k += MP_BLOCK) {
		int64_t v;
		if (k == 0) v = offsets[i0];
		else {
			const int64_t r = i0 + k;
			v = r <= m ? offsets[r] : j1 + 1;
		}
		sm.row_end[k] = int32_t(v - j0);
	}
	{
		uint32_t col[MP_IPT];
		T a[MP_IPT];
#pragma unroll
		for (int u = 0; u < MP_IPT; ++u) {
			const int k = tid + u * MP_BLOCK;
			if (k < nnzt) {
				col[u] = __ldcs(indices + j0 + k);
				a[u] = values ? __ldcs(values + j0 + k) : R::one();
			}
		}
#pragma unroll
		for (int u = 0; u < MP_IPT; ++u) {
			const int k = tid + u * MP_BLOCK;
			if (k < nnzt) {
				const T xv = xl(col[u]);
				sm.prod[k] = left ? R::mull(xv, a[u]) : R::mulr(a[u], xv);
			}
		}
	}
	__syncthreads();

	const int items = nrows + nnzt;
	int dl = tid * MP_IPT;
	if (dl > items) dl = items;
	int ti, tj;
	{
		int lo = dl - nnzt > 0 ? dl - nnzt : 0, hi = dl < nrows ? dl : nrows;
		while (lo < hi) {
			const int pivot = (lo + hi) >> 1;
			if (sm.row_end[pivot + 1] <= dl - pivot - 1) lo = pivot + 1; else hi = pivot;
		}
		ti = lo;
		tj = dl - lo;
	}
	int dend = dl + MP_IPT;
	if (dend > items) dend = items;

	T acc = R::zero();
	bool has = false;
	int first_row = -1;
	T first_val = R::zero();
	bool first_has = false;
	for (int d = dl; d < dend; ++d) {
		if (tj < sm.row_end[ti + 1]) {
			acc = R::add(acc, sm.prod[tj]);
			has = true;
			++tj;
		} else {
			if (first_row < 0) {
				first_row = ti;
				first_val = acc;
				first_has = has;
			} else {
				epi.row(i0 + ti, acc, has);
			}
			acc = R::zero();
			has = false;
			++ti;
		}
	}
	sm.crow[tid] = ti;
	sm.cval[tid] = acc;
	sm.chas[tid] = has ? 1 : 0;
	__syncthreads();

	if (first_row >= 0) {
		T v = first_val;
		bool h = first_has;
		for (int s = tid - 1; s >= 0 && sm.crow[s] == first_row; --s) {
			if (sm.chas[s]) {
				v = R::add(v, sm.cval[s]);
				h = true;
			}
		}
		if (first_row == 0 && mt.head_first[t] >= 0) {
			// head row started in an earlier tile: park this tile's partial
			store_bits<T>(mt.head_val + t, v);
			mt.head_has[t] = h ? 1 : 0;
			T sum;
			bool hs;
			if (arrive<R>(mt, mt.head_first[t], sum, hs)) epi.row_span(mt.head_first[t], i0, sum, hs);
		} else {
			epi.row(i0 + first_row, v, h);
		}
	}
	if (tid == MP_BLOCK - 1 && mt.tail_first[t] >= 0) {
		T v = R::zero();
		bool h = false;
		for (int s = MP_BLOCK - 1; s >= 0 && sm.crow[s] == nrows; --s) {
			if (sm.chas[s]) {
				v = R::add(v, sm.cval[s]);
				h = true;
			}
		}
		store_bits<T>(mt.tail_val + t, v);
		mt.tail_has[t] = h ? 1 : 0;
		T sum;
		bool hs;
		if (arrive<R>(mt, mt.tail_first[t], sum, hs)) epi.row_span(mt.tail_first[t], i1, sum, hs);
	}
	__syncthreads();  // shared memory is reused by the next tile
}

// Gather of a plain input vector (read-only path, stays in L2 across tiles).
template <class T>
struct PlainX {
	const T *__restrict__ x;
	__device__ __forceinline__ T operator()(uint32_t j) const { return __ldg(x + j); }
};

// Table kernels (spmv.cu): tile starts by merge-path search, then the
// spanning-row tables.
// `tile` = merge items per tile.
__global__ void k_merge_tiles(const int64_t *offsets, int64_t m, int64_t nnz, int64_t ntiles,
	int64_t *tile_row, int64_t tile = MP_TILE);
__global__ void k_merge_tables(const int64_t *offsets, int64_t m, int64_t nnz, int64_t ntiles,
	const int64_t *tile_row, int64_t *head_first, int64_t *tail_first, int32_t *span_len,
	int64_t tile = MP_TILE);

// Segmented tables (batched solves): tiles are cut at segment boundaries.
struct SegmentedTiles {
	int64_t nseg = 0;
	int64_t *seg_rows = nullptr;  // [nseg+1] first row of each segment (device)
	int64_t *seg_tile = nullptr;  // [nseg+1] first tile of each segment (device)
	int64_t *tile_d = nullptr;    // [ntiles+1]
	int32_t *tile_seg = nullptr;  // [ntiles] segment of each tile
};
// Build a plan whose tiles never straddle segments (seg_rows on the device,
// nseg+1 entries, ascending from 0 to m).  Fills p's merge tables and `st`.
int merge_plan_segmented(alpb_spmv_plan_s *p, const int64_t *offsets, int64_t nseg,
	const int64_t *seg_rows, SegmentedTiles *st, cudaStream_t s);
void segmented_free(SegmentedTiles *st);

MergeTables merge_tables(const alpb_spmv_plan_s &p);

} // namespace alpb
