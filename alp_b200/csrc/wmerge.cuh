// Warp-granular merge-path tiles.
//
// Same merge list as merge.cuh (a tile owns a fixed number of consecutive
// merge items, whatever the row lengths), but one warp owns one tile of
// 32 x WM_IPT items and synchronises only with __syncwarp:
//   1. the tile's row ends and products a_ij (*) x_j are staged in the warp's
//      shared memory with coalesced, lane-strided loads (the epilogue may
//      prefetch what its rows need at the same time: Epi::begin_tile);
//   2. every lane walks WM_IPT consecutive merge items and finishes the rows
//      whose row end it meets;
//   3. the lanes' carries (the partial of the row each lane stops in) are
//      combined with a segmented inclusive scan over shuffles, keyed by row:
//      a lane's first finished row gets the carries of the lanes before it;
//   4. a row that crosses tiles leaves one partial per tile in the tile's
//      head or tail slot, and a second, tiny pass (k_wm_fixup) sums each
//      such row's slots in tile order.  No atomics and no fences.
// Every sum has a fixed order (in-lane order, scan tree, slot order): results
// are deterministic from run to run.
#pragma once
#include "merge.cuh"

#include <type_traits>

namespace alpb {

#ifndef ALPB_WM_IPT
#define ALPB_WM_IPT 8
#endif
constexpr int WM_IPT = ALPB_WM_IPT;    // merge items per lane
constexpr int WM_TILE = 32 * WM_IPT;   // merge items per warp tile
constexpr unsigned WM_FULL = 0xffffffffu;

// wm_core options
constexpr int WM_LOADS_FIRST = 1;
constexpr int WM_WALK_AHEAD = 2;

// Position of product k in shared memory.  The staging writes k = 32u + L
// (lane L) and the walk reads k ~ 8L + c; XOR-ing the low four bits with bits
// 3..6 makes both patterns hit sixteen distinct 8-byte bank pairs per
// half-warp (a bijection of k within each aligned block of 128 entries).
__device__ __forceinline__ int wm_pad(int k) { return k ^ ((k >> 3) & 15); }

template <class R>
struct WarpSmem {
	using End = int32_t;
	typename R::T prod[WM_TILE < 128 ? 128 : WM_TILE];
	End row_end[WM_TILE + 2];  // [k] = end of tile row k-1, relative to j0, clamped
};

// Compact variant (2.7 KB per warp for FP64 instead of 3 KB plus a separate
// y buffer): row ends fit 16 bits (they are clamped to [-1, WM_TILE + 1]),
// and the y values of the tile's rows share the product buffer, from its far
// end down: products occupy [0, nnzt rounded up to 16) (the swizzle stays
// inside aligned groups of 16) and y of row k sits at prod[WM_TILE + 15 - k];
// the two never meet since rows + nonzeroes of a tile are at most WM_TILE.
template <class R>
struct WarpSmemCompact {
	using End = int16_t;
	typename R::T prod[WM_TILE + 16];
	End row_end[WM_TILE + 2];
	__device__ __forceinline__ typename R::T &y(int k) { return prod[WM_TILE + 15 - k]; }
};

template <class T>
__device__ __forceinline__ T wm_shfl_up(T v, int off) {
	if constexpr (std::is_same<T, bool>::value) return __shfl_up_sync(WM_FULL, int(v), off) != 0;
	else return __shfl_up_sync(WM_FULL, v, off);
}
template <class T>
__device__ __forceinline__ T wm_shfl(T v, int src) {
	if constexpr (std::is_same<T, bool>::value) return __shfl_sync(WM_FULL, int(v), src) != 0;
	else return __shfl_sync(WM_FULL, v, src);
}
template <class T>
__device__ __forceinline__ T wm_shfl_xor(T v, int m) {
	if constexpr (std::is_same<T, bool>::value) return __shfl_xor_sync(WM_FULL, int(v), m) != 0;
	else return __shfl_xor_sync(WM_FULL, v, m);
}

// Value bits of a slot, read through L2 (slots are written by other SMs).
template <class T>
__device__ __forceinline__ T wm_load_slot(const uint64_t *p) {
	const unsigned long long b = __ldcg(reinterpret_cast<const unsigned long long *>(p));
	T v;
	memcpy(&v, &b, sizeof(T));
	return v;
}

// Shared body of a warp tile: stages the tile, walks it, scans the carries
// and calls epi.row for every row that ends in the tile -- except the head
// row when it started in an earlier tile (hf >= 0).  epi.begin_tile(i0,
// nrows, lane) runs first, on every lane, for the rows [i0, i0 + nrows) that
// end in the tile (its shared-memory writes are visible to epi.row).  Leaves in every lane:
// head_v/head_h (the partial of row i0 up to its end, in the lane whose first
// finished row is row 0) and sv/sh (lane 31: the partial of the tail row).
//
// Opts (WM_LOADS_FIRST | WM_WALK_AHEAD):
// WM_LOADS_FIRST issues the tile's loads (the offsets of its first 64 rows,
// its column indices and values, then epi.begin_tile's) before any
// shared-memory store, so that their round trips overlap; it holds 4 more
// registers while they are in flight, which a kernel at the 64-register
// limit cannot spare (the hot-column SpMV leaves it out).
// WM_WALK_AHEAD reads the walk's next product and next row end one step
// ahead (measured: the SpMV kernels gain 1-2 %, PageRank's loses 2 %).
template <class R, class XL, class Epi, class SM, int Opts = WM_LOADS_FIRST>
__device__ __forceinline__ void wm_core(int64_t t, const MergeTables &mt,
	const int64_t *__restrict__ offsets, const uint32_t *__restrict__ indices,
	const typename R::T *__restrict__ values, const XL &xl, Epi &epi, int left,
	SM &sm, int64_t i0, int64_t i1, int64_t hf, int &first_row,
	typename R::T &head_v, bool &head_h, typename R::T &sv, bool &sh) {
	using T = typename R::T;
	const int lane = threadIdx.x & 31;
	const int64_t m = mt.m, nnz = mt.nnz;
	int64_t d0, d1;
	if (mt.tile_d) {
		d0 = mt.tile_d[t];
		d1 = mt.tile_d[t + 1];
	} else {
		d0 = t * WM_TILE;
		d1 = d0 + WM_TILE;
		if (d1 > m + nnz) d1 = m + nnz;
	}
	const int64_t j0 = d0 - i0, j1 = d1 - i1;
	const int nrows = int(i1 - i0);
	const int nnzt = int(j1 - j0);
	if constexpr ((Opts & WM_LOADS_FIRST) != 0) {
		int64_t ro[2];
#pragma unroll
		for (int h = 0; h < 2; ++h) {
			const int k = lane + 32 * h;
			const int64_t r = i0 + k;
			ro[h] = k <= nrows + 1 && r <= m ? offsets[r] : j1 + 1;
		}
		uint32_t col[WM_IPT];
		T a[WM_IPT];
#pragma unroll
		for (int u = 0; u < WM_IPT; ++u) {
			const int k = lane + 32 * u;
			if (k < nnzt) {
				col[u] = __ldcs(indices + j0 + k);
				a[u] = values ? __ldcs(values + j0 + k) : R::one();
			}
		}
		epi.begin_tile(i0, nrows, lane);
		// row ends, relative to j0, clamped as below
#pragma unroll
		for (int h = 0; h < 2; ++h) {
			const int k = lane + 32 * h;
			if (k <= nrows + 1) {
				int64_t v = ro[h] - j0;
				if (v > WM_TILE + 1) v = WM_TILE + 1;
				if (v < -1) v = -1;
				sm.row_end[k] = static_cast<typename SM::End>(v);
			}
		}
		for (int k = lane + 64; k <= nrows + 1; k += 32) {
			const int64_t r = i0 + k;
			int64_t v = (r <= m ? offsets[r] : j1 + 1) - j0;
			if (v > WM_TILE + 1) v = WM_TILE + 1;
			if (v < -1) v = -1;
			sm.row_end[k] = static_cast<typename SM::End>(v);
		}
#pragma unroll
		for (int u = 0; u < WM_IPT; ++u) {
			const int k = lane + 32 * u;
			if (k < nnzt) {
				const T xv = xl(col[u]);
				sm.prod[wm_pad(k)] = left ? R::mull(xv, a[u]) : R::mulr(a[u], xv);
			}
		}
	} else {
		epi.begin_tile(i0, nrows, lane);

		// row ends, relative to j0; clamped to the tile (the walk compares them
		// with positions <= nnzt only)
		for (int k = lane; k <= nrows + 1; k += 32) {
			int64_t v;
			if (k == 0) v = offsets[i0] - j0;
			else {
				const int64_t r = i0 + k;
				v = (r <= m ? offsets[r] : j1 + 1) - j0;
			}
			if (v > WM_TILE + 1) v = WM_TILE + 1;
			if (v < -1) v = -1;
			sm.row_end[k] = static_cast<typename SM::End>(v);
		}
		{
			uint32_t col[WM_IPT];
			T a[WM_IPT];
#pragma unroll
			for (int u = 0; u < WM_IPT; ++u) {
				const int k = lane + 32 * u;
				if (k < nnzt) {
					col[u] = __ldcs(indices + j0 + k);
					a[u] = values ? __ldcs(values + j0 + k) : R::one();
				}
			}
#pragma unroll
			for (int u = 0; u < WM_IPT; ++u) {
				const int k = lane + 32 * u;
				if (k < nnzt) {
					const T xv = xl(col[u]);
					sm.prod[wm_pad(k)] = left ? R::mull(xv, a[u]) : R::mulr(a[u], xv);
				}
			}
		}
	}
	__syncwarp();

	// merge-path split of this lane's WM_IPT items
	const int items = nrows + nnzt;
	int dl = lane * WM_IPT;
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
	int dend = dl + WM_IPT;
	if (dend > items) dend = items;

	T acc = R::zero();
	bool has = false;
	first_row = -1;
	T first_val = R::zero();
	bool first_has = false;
	int re = sm.row_end[ti + 1];  // end of the row being walked
	if constexpr ((Opts & WM_WALK_AHEAD) != 0) {
		// the next product and the next row end are read one step ahead, so no
		// step waits on a shared-memory load issued by the step before (the reads
		// past the tile's last product or row are clamped into the arrays and
		// their values never used)
		int re2 = sm.row_end[ti + 2 <= nrows + 1 ? ti + 2 : nrows + 1];
		T pv = sm.prod[wm_pad(tj < WM_TILE ? tj : WM_TILE - 1)];
#pragma unroll
		for (int s = 0; s < WM_IPT; ++s) {
			if (dl + s < dend) {
				if (tj < re) {
					acc = R::add(acc, pv);
					has = true;
					++tj;
					pv = sm.prod[wm_pad(tj < WM_TILE ? tj : WM_TILE - 1)];
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
					re = re2;
					re2 = sm.row_end[ti + 2 <= nrows + 1 ? ti + 2 : nrows + 1];
				}
			}
		}
	} else {
		for (int d = dl; d < dend; ++d) {
			if (tj < re) {
				acc = R::add(acc, sm.prod[wm_pad(tj)]);
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
				re = sm.row_end[ti + 1];
			}
		}
	}

	// segmented inclusive scan of the carries, keyed by the row each lane
	// stops in (rows are non-decreasing over lanes)
	// (rows are non-decreasing over lanes, so the lanes that stop in this
	// lane's row are the run [seg0, lane]: one match replaces a shuffle of
	// the row per step, and the presence flags are OR-ed from one ballot)
	sv = acc;
	const int seg0 = __ffs(__match_any_sync(WM_FULL, ti)) - 1;
#pragma unroll
	for (int off = 1; off < 32; off <<= 1) {
		const T v = wm_shfl_up(sv, off);
		if (lane - off >= seg0) sv = R::add(v, sv);
	}
	{
		const unsigned upto = lane == 31 ? 0xffffffffu : (1u << (lane + 1)) - 1u;
		sh = (__ballot_sync(WM_FULL, has) & upto & ~((1u << seg0) - 1u)) != 0;
	}
	// carry into this lane: the scan of lane-1, whose stop row is this lane's
	// start row
	T cin = wm_shfl_up(sv, 1);
	bool cin_h = wm_shfl_up(sh, 1);
	if (lane == 0) {
		cin = R::zero();
		cin_h = false;
	}
	head_v = R::zero();
	head_h = false;
	if (first_row >= 0) {
		head_v = R::add(cin, first_val);
		head_h = cin_h || first_has;
		if (!(first_row == 0 && hf >= 0)) epi.row(i0 + first_row, head_v, head_h);
	}
	__syncwarp();  // the warp's shared memory is reused by its next tile
}

// Table entries of one warp tile (loaded one tile ahead by the persistent
// loops, so that their latency hides behind the previous tile's work).
struct WmMeta {
	int64_t i0, i1, hf, tf;
};
__device__ __forceinline__ WmMeta wm_meta(const MergeTables &mt, int64_t t) {
	WmMeta g{0, 0, -1, -1};
	if (t < mt.ntiles) {
		g.i0 = mt.tile_row[t];
		g.i1 = mt.tile_row[t + 1];
		g.hf = mt.head_first[t];
		g.tf = mt.tail_first[t];
	}
	return g;
}

// One warp tile t for the two-pass SpMV: rows that end in the tile are
// finished here (epi.row); a row crossing tiles leaves this tile's partial in
// head_val[t] (the row ends here) or tail_val[t] (it continues), and
// k_wm_fixup finishes it.  A spanning row always holds nonzeroes, so its
// partials need no presence flag: an empty partial is the additive identity.
template <class R, class XL, class Epi, class SM, int Opts = WM_LOADS_FIRST>
__device__ __forceinline__ void warp_tile(int64_t t, const WmMeta &g, const MergeTables &mt,
	const int64_t *__restrict__ offsets, const uint32_t *__restrict__ indices,
	const typename R::T *__restrict__ values, const XL &xl, Epi &epi, int left,
	SM &sm) {
	using T = typename R::T;
	const int lane = threadIdx.x & 31;
	int first_row;
	T head_v, sv;
	bool head_h, sh;
	wm_core<R, XL, Epi, SM, Opts>(t, mt, offsets, indices, values, xl, epi, left, sm, g.i0,
		g.i1, g.hf, first_row, head_v, head_h, sv, sh);
	if (g.hf >= 0 && first_row == 0) store_bits<T>(mt.head_val + t, head_v);
	if (g.tf >= 0 && lane == 31) store_bits<T>(mt.tail_val + t, sv);
}

__device__ __forceinline__ int wm_ld_acquire(const int32_t *p) {
	int32_t v;
	asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ void wm_st_release(int32_t *p, int32_t v) {
	asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Spin bound of a tile waiting for an earlier tile's tail partial (~0.5 s at
// the sleep granularity below; far beyond any wait between co-resident warps).
constexpr long long kWmSpinLimit = 1ll << 23;

// One warp tile t of a fused solver, with every row finished by a FIXED tile:
// a row crossing tiles is finished by the tile where it ends, which waits for
// the tail partials that the row's earlier tiles publish in mt.ready under
// `epoch` (larger than any value the array held before; it starts at zero).
// Epilogue terms therefore accumulate in a fixed order wherever the tiles
// run.  Requires every warp of the grid to be resident (a cooperative launch)
// and each warp to take its tiles in increasing order: a tile publishes its
// tail before it waits, and waits only on smaller tiles, so no wait can close
// a cycle.  Epi: begin_tile and row(r, sum, has), from any lane.  Returns
// false if a wait gave up or *err was set elsewhere (a timeout sets *err = 1;
// the caller leaves at its next grid barrier, which checks the same flag).
template <class R, class XL, class Epi, int Opts = WM_LOADS_FIRST>
__device__ __forceinline__ bool warp_tile_ordered(int64_t t, const WmMeta &g,
	const MergeTables &mt, const int64_t *__restrict__ offsets,
	const uint32_t *__restrict__ indices, const typename R::T *__restrict__ values,
	const XL &xl, Epi &epi, int left, WarpSmem<R> &sm, int32_t epoch, int *err) {
	using T = typename R::T;
	const int lane = threadIdx.x & 31;
	int first_row;
	T head_v, sv;
	bool head_h, sh;
	wm_core<R, XL, Epi, WarpSmem<R>, Opts>(t, mt, offsets, indices, values, xl, epi, left,
		sm, g.i0, g.i1, g.hf, first_row, head_v, head_h, sv, sh);
	if (g.tf >= 0 && lane == 31) {
		store_bits<T>(mt.tail_val + t, sv);
		wm_st_release(mt.ready + t, epoch);  // orders the store above before the flag
	}
	if (g.hf < 0) return true;
	T v = R::zero();
	bool ok = true;
	for (int64_t k = g.hf + lane; k < t && ok; k += 32) {
		long long spins = 0;
		while (wm_ld_acquire(mt.ready + k) < epoch) {
			if (++spins > kWmSpinLimit) {
				atomicExch(err, 1);
				ok = false;
				break;
			}
			if (*reinterpret_cast<volatile int *>(err)) {  // another wait gave up
				ok = false;
				break;
			}
			__nanosleep(64);
		}
		if (ok) v = R::add(v, wm_load_slot<T>(mt.tail_val + k));
	}
	if (!__all_sync(WM_FULL, ok)) return false;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		const T vo = wm_shfl_xor(v, o);
		v = R::add(v, vo);
	}
	if (first_row == 0) epi.row(g.i0, R::add(v, head_v), true);
	return true;
}

// v (+)= slots[k] for k = k0, k0+1, ..., k1-1, in that order, eight loads in
// flight (a row spanning many tiles then costs a few round trips, not one
// per tile).
template <class R>
__device__ __forceinline__ typename R::T wm_sum_slots(typename R::T v, const uint64_t *slots,
	int64_t k0, int64_t k1) {
	using T = typename R::T;
	int64_t k = k0;
	for (; k + 8 <= k1; k += 8) {
		T b[8];
#pragma unroll
		for (int u = 0; u < 8; ++u) b[u] = wm_load_slot<T>(slots + k + u);
#pragma unroll
		for (int u = 0; u < 8; ++u) v = R::add(v, b[u]);
	}
	for (; k < k1; ++k) v = R::add(v, wm_load_slot<T>(slots + k));
	return v;
}

// v (+)= slots[k] for k = k0, k0 + 32, k0 + 64, ... < k1, in that order,
// eight loads in flight (one lane's share of a row spanning many tiles).
template <class R>
__device__ __forceinline__ typename R::T wm_sum_slots32(typename R::T v, const uint64_t *slots,
	int64_t k0, int64_t k1) {
	using T = typename R::T;
	int64_t k = k0;
	for (; k + 7 * 32 < k1; k += 8 * 32) {
		T b[8];
#pragma unroll
		for (int u = 0; u < 8; ++u) b[u] = wm_load_slot<T>(slots + k + 32 * u);
#pragma unroll
		for (int u = 0; u < 8; ++u) v = R::add(v, b[u]);
	}
	for (; k < k1; k += 32) v = R::add(v, wm_load_slot<T>(slots + k));
	return v;
}

// Second pass: every row that crosses tiles, y_r = y_r (+) its slots summed
// in tile order (tail slots of its first..last-1 tiles, head slot of its last
// tile).  One lane per first tile for spans up to 32 tiles; the whole warp
// for longer ones.
template <class R, class Epi>
__global__ void __launch_bounds__(256) k_wm_fixup(MergeTables mt, Epi epi) {
	using T = typename R::T;
	const int lane = threadIdx.x & 31;
	const int64_t warp = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
	const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
	for (int64_t base = warp * 32; base < mt.ntiles; base += nwarps * 32) {
		const int64_t t = base + lane;
		const int32_t n = t < mt.ntiles ? mt.span_len[t] : 0;
		if (n > 0 && n <= 32) {
			T v = wm_sum_slots<R>(R::zero(), mt.tail_val, t, t + n - 1);
			v = R::add(v, wm_load_slot<T>(mt.head_val + t + n - 1));
			epi.row(mt.tile_row[t + 1], v, true);
		}
		unsigned long_rows = __ballot_sync(WM_FULL, n > 32);
		while (long_rows) {
			const int src = __ffs(long_rows) - 1;
			long_rows &= long_rows - 1;
			const int64_t f = base + src;
			const int32_t nn = __shfl_sync(WM_FULL, n, src);
			T v = wm_sum_slots32<R>(R::zero(), mt.tail_val, f + lane, f + nn - 1);
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) {
				const T vo = wm_shfl_xor(v, o);
				v = R::add(v, vo);
			}
			if (lane == 0) {
				v = R::add(v, wm_load_slot<T>(mt.head_val + f + nn - 1));
				epi.row(mt.tile_row[f + 1], v, true);
			}
		}
	}
}

} // namespace alpb
