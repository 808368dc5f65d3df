// Personalised PageRank and its adjoint (differentiable PageRank).
//
// ALP's simple_pagerank (algorithms/simple_pagerank.hpp:146-533) teleports
// uniformly and normalises by the out-degree count; this is its personalised
// form over a weighted graph, for up to 128 seeds at once.  With W the edge
// weights (row i -> column j), d_i = sum_j w_ij and v_s the one-hot vector of
// seed s:
//
//   forward   x_s = alpha M x_s + (alpha dangling(x_s) + 1 - alpha) v_s,
//             M_ji = w_ij / d_i, dangling(x) = sum of x over rows with d_i = 0,
//             by the power iteration of simple_pagerank: the input of each
//             product is pre-scaled by alpha / d_i (zero for dangling rows,
//             whose mass is summed apart, :281-289 and :324-357), the
//             teleport term is (alpha * dangling + 1 - alpha) (:390) and a
//             seed stops at L1 change <= conv (:440-490);
//   adjoint   lambda_s = alpha M^T lambda_s + alpha [i dangling] lambda_s[seed_s]
//                        + g_s,  g = dL/dx, by the same fixed-point iteration;
//   gradient  dL/dw_ij = alpha / d_i sum_s x_is (lambda_js - mu_is),
//             mu_s = M^T lambda_s   (implicit function theorem: no iterate of
//                                    the forward solve is stored).
// With unit weights d_i is the out-degree count of the reference, and the mean
// of the personalised vectors over all n seeds of a graph without dangling rows
// is simple_pagerank's vector.
//
// Vectors hold the S = nseeds values of a row side by side (row-major n x S).
// Products run on chunks of at most HP_CHUNK nonzeroes of one row of the
// compressed storage (CCS for the forward gather, CRS for the adjoint one): a
// warp loads a chunk's indices and weights in one coalesced access and its
// lanes, one or more per seed, gather 8*S contiguous bytes per nonzero.  Rows
// of several chunks leave per-chunk partials that a second launch sums in
// chunk order, and every per-seed sum is reduced in a fixed order, so results
// are deterministic.  A third launch (one block per seed) closes the
// iteration: residual, teleport or dangling term, convergence.
#include "common.cuh"

#include <cub/device/device_scan.cuh>

#include <cmath>
#include <vector>

namespace alpb {

constexpr int HP_CHUNK = 32;          // nonzeroes per chunk (one per lane)
constexpr int HP_WARPS = 8;           // warps per block of the gather kernels
constexpr int HP_MAX_SEEDS = 128;
constexpr int HP_FIN_THREADS = 256;
#ifndef ALPB_HP_MINB
#define ALPB_HP_MINB 4       // resident blocks per SM the gather kernels are built for
#endif
#ifndef ALPB_HP_BATCH
#define ALPB_HP_BATCH 4      // nonzeroes per lane group and gather batch (halved at 4+ seeds per lane)
#endif

// Chunk table of one compressed storage (CRS or CCS).  Chunk c covers
// nonzeroes [beg[c], beg[c+1]) of row row[c]; every row has at least one
// chunk (possibly empty).  slot[c] >= 0 names the partial of a chunk of a row
// of several chunks (the slots of one row are consecutive); multi lists those
// rows with their first slot and chunk count.  A row of more than HP_GROUP
// chunks (a power-law hub) has its slots summed in groups of HP_GROUP first
// (one warp per group), so no warp sums thousands of partials alone: mgroup
// names the row's first group (-1 without groups), group g covers slots
// [gslot[g], gslot[g] + glen[g]).
constexpr int HP_GROUP_CHUNKS = 32;

struct HpChunks {
	int64_t nchunks = 0, nmulti = 0, nslots = 0, ngroups = 0;
	int64_t *beg = nullptr;       // [nchunks + 1]
	uint32_t *row = nullptr;      // [nchunks]
	int32_t *slot = nullptr;      // [nchunks]
	uint32_t *mrow = nullptr;     // [nmulti]
	int32_t *mslot = nullptr;     // [nmulti]
	int32_t *mcount = nullptr;    // [nmulti]
	int32_t *mgroup = nullptr;    // [nmulti]
	int32_t *gslot = nullptr;     // [ngroups]
	int32_t *glen = nullptr;      // [ngroups]
};

static void chunks_free(HpChunks *c) {
	cudaFree(c->beg);
	cudaFree(c->row);
	cudaFree(c->slot);
	cudaFree(c->mrow);
	cudaFree(c->mslot);
	cudaFree(c->mcount);
	cudaFree(c->mgroup);
	cudaFree(c->gslot);
	cudaFree(c->glen);
	*c = HpChunks{};
}

// per row: chunk count, slot count and multi flag of rows of several chunks,
// group count of rows of more than HP_GROUP_CHUNKS chunks
__global__ void k_hp_count(const int64_t *offsets, int64_t n, int64_t *nch, int64_t *nsl,
	int64_t *nmu, int64_t *ngr) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i <= n;
		 i += int64_t(gridDim.x) * blockDim.x) {
		if (i == n) {
			nch[i] = nsl[i] = nmu[i] = ngr[i] = 0;
			continue;
		}
		const int64_t len = offsets[i + 1] - offsets[i];
		int64_t c = (len + HP_CHUNK - 1) / HP_CHUNK;
		if (c < 1) c = 1;
		nch[i] = c;
		nsl[i] = c > 1 ? c : 0;
		nmu[i] = c > 1 ? 1 : 0;
		ngr[i] = c > HP_GROUP_CHUNKS ? (c + HP_GROUP_CHUNKS - 1) / HP_GROUP_CHUNKS : 0;
	}
}

__global__ void k_hp_fill(const int64_t *offsets, int64_t n, const int64_t *first,
	const int64_t *slot0, const int64_t *mpos, const int64_t *gfirst, HpChunks t) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x) {
		const int64_t c0 = first[i], c1 = first[i + 1];
		const bool multi = c1 - c0 > 1;
		for (int64_t c = c0; c < c1; ++c) {
			t.beg[c] = offsets[i] + (c - c0) * HP_CHUNK;
			t.row[c] = uint32_t(i);
			t.slot[c] = multi ? int32_t(slot0[i] + (c - c0)) : -1;
		}
		if (multi) {
			const int64_t p = mpos[i];
			t.mrow[p] = uint32_t(i);
			t.mslot[p] = int32_t(slot0[i]);
			t.mcount[p] = int32_t(c1 - c0);
			const int64_t g0 = gfirst[i], g1 = gfirst[i + 1];
			t.mgroup[p] = g1 > g0 ? int32_t(g0) : -1;
			for (int64_t g = g0; g < g1; ++g) {
				const int64_t k0 = (g - g0) * HP_GROUP_CHUNKS;
				const int64_t k1 = k0 + HP_GROUP_CHUNKS < c1 - c0 ? k0 + HP_GROUP_CHUNKS : c1 - c0;
				t.gslot[g] = int32_t(slot0[i] + k0);
				t.glen[g] = int32_t(k1 - k0);
			}
		}
		if (i == n - 1) t.beg[c1] = offsets[n];
	}
}

template <class T>
static int exclusive_scan(const T *in, T *out, int64_t count, cudaStream_t s) {
	size_t bytes = 0;
	ALPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, count, s));
	void *tmp = nullptr;
	ALPB_CUDA(cudaMallocAsync(&tmp, bytes, s));
	ALPB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, count, s));
	g_launches.fetch_add(1);
	ALPB_CUDA(cudaFreeAsync(tmp, s));
	return ALPB_SUCCESS;
}

static int chunks_build(HpChunks *t, const int64_t *offsets, int64_t n, cudaStream_t s) {
	int64_t *buf = nullptr;   // nch, nsl, nmu, ngr and their scans: 8 x (n + 1)
	ALPB_CUDA(cudaMallocAsync(&buf, size_t(8) * (n + 1) * 8, s));
	int64_t *nch = buf, *nsl = buf + (n + 1), *nmu = buf + 2 * (n + 1), *ngr = buf + 3 * (n + 1);
	int64_t *first = buf + 4 * (n + 1), *slot0 = buf + 5 * (n + 1), *mpos = buf + 6 * (n + 1);
	int64_t *gfirst = buf + 7 * (n + 1);
	k_hp_count<<<grid_for(n + 1, 256), 256, 0, s>>>(offsets, n, nch, nsl, nmu, ngr);
	ALPB_LAUNCHED();
	int rc = exclusive_scan(nch, first, n + 1, s);
	rc = rc ? rc : exclusive_scan(nsl, slot0, n + 1, s);
	rc = rc ? rc : exclusive_scan(nmu, mpos, n + 1, s);
	rc = rc ? rc : exclusive_scan(ngr, gfirst, n + 1, s);
	if (rc) {
		cudaFreeAsync(buf, s);
		return rc;
	}
	int64_t tot[4];
	ALPB_CUDA(cudaMemcpyAsync(&tot[0], first + n, 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaMemcpyAsync(&tot[1], slot0 + n, 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaMemcpyAsync(&tot[2], mpos + n, 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaMemcpyAsync(&tot[3], gfirst + n, 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	t->nchunks = tot[0];
	t->nslots = tot[1];
	t->nmulti = tot[2];
	t->ngroups = tot[3];
	ALPB_CHECK(t->nslots < (int64_t(1) << 31), ALPB_OVERFLW, "ppr: too many chunk partials");
	if (cudaMalloc(&t->beg, size_t(t->nchunks + 1) * 8) != cudaSuccess ||
		cudaMalloc(&t->row, size_t(t->nchunks) * 4) != cudaSuccess ||
		cudaMalloc(&t->slot, size_t(t->nchunks) * 4) != cudaSuccess ||
		cudaMalloc(&t->mrow, size_t(t->nmulti + 1) * 4) != cudaSuccess ||
		cudaMalloc(&t->mslot, size_t(t->nmulti + 1) * 4) != cudaSuccess ||
		cudaMalloc(&t->mcount, size_t(t->nmulti + 1) * 4) != cudaSuccess ||
		cudaMalloc(&t->mgroup, size_t(t->nmulti + 1) * 4) != cudaSuccess ||
		cudaMalloc(&t->gslot, size_t(t->ngroups + 1) * 4) != cudaSuccess ||
		cudaMalloc(&t->glen, size_t(t->ngroups + 1) * 4) != cudaSuccess) {
		cudaGetLastError();
		cudaFreeAsync(buf, s);
		set_error("ppr: out of device memory for the chunk tables");
		return ALPB_OUTOFMEM;
	}
	k_hp_fill<<<grid_for(n, 256), 256, 0, s>>>(offsets, n, first, slot0, mpos, gfirst, *t);
	ALPB_LAUNCHED();
	ALPB_CUDA(cudaFreeAsync(buf, s));
	return ALPB_SUCCESS;
}


// ------------------------------------------------------------ the passes --
enum HpMode { HP_FWD = 0, HP_ADJ = 1, HP_MU = 2 };

// Per-seed state on the device, [S] each.
struct HpSeeds {
	const int64_t *seed;
	double *term;       // forward: teleport term; adjoint: alpha * lambda[seed]
	double *res;        // residual of the last finished iteration
	int32_t *active;
	int64_t *iters;
	int32_t *n_active;  // seeds still iterating
};

struct HpArgs {
	// the chunked storage this pass gathers over
	const int64_t *beg;
	const uint32_t *crow;
	const int32_t *cslot;
	int64_t nchunks;
	const uint32_t *mrow;
	const int32_t *mslot, *mcount, *mgroup;
	int64_t nmulti;
	const int32_t *gslot, *glen;
	int64_t ngroups;
	double *gpart;      // [ngroups][S] group partials of hub rows
	const uint32_t *idx;
	const double *val;
	// vectors (n x S)
	const double *in;   // forward: scaled input; adjoint and mu: lambda
	double *out;        // forward: next scaled input; adjoint: next lambda
	double *x;          // forward: updated in place; mu: read
	const double *g;    // adjoint: dL/dx
	const double *rowscale;  // forward: alpha / d (0 dangling); adjoint, mu: 1 / d (0 dangling)
	double *part;       // [nslots][S] chunk partials
	double *bp;         // [blocks][2S] block partials (residual, dangling)
	double *c;          // mu: per row sum_s x_is mu_is
	HpSeeds sd;
	int64_t n;
	int S;
	double alpha;
};

// Seed layout of a warp: 32 / G lane groups of G lanes; lane gl of a group
// handles seeds gl + G q, q < SPL.  Groups split a chunk's nonzeroes.
template <int G, int SPL>
struct HpLanes {
	int lane, gsub, gl;
	__device__ __forceinline__ HpLanes() {
		lane = threadIdx.x & 31;
		gsub = lane / G;
		gl = lane % G;
	}
	__device__ __forceinline__ int seed(int q) const { return gl + G * q; }
	__device__ __forceinline__ bool lead() const { return gsub == 0; }
};

// Row epilogue in two halves: hp_epi_load fetches the operands of row r at
// the start of its chunk (they do not depend on the gather, so their latency
// hides behind it), hp_epi_apply finishes the row once the sums are in.
template <int SPL>
struct HpEpiIn {
	double rs;
	double v0[SPL];   // forward: old x; adjoint: current lambda; mu: x
	double v1[SPL];   // adjoint: dL/dx
};

template <int MODE, int G, int SPL>
__device__ __forceinline__ void hp_epi_load(const HpArgs &a, const HpLanes<G, SPL> &L, int64_t r,
	HpEpiIn<SPL> &e) {
	const int S = a.S;
	e.rs = __ldg(a.rowscale + r);
#pragma unroll
	for (int q = 0; q < SPL; ++q) {
		const int s = L.seed(q);
		const bool own = L.lead() && s < S;
		const int64_t o = r * S + s;
		e.v0[q] = 0.0;
		e.v1[q] = 0.0;
		if (own) {
			if (MODE == HP_FWD || MODE == HP_MU) e.v0[q] = __ldcs(a.x + o);
			if (MODE == HP_ADJ) {
				e.v0[q] = __ldg(a.in + o);   // the gathered vector: keep its L2 priority
				e.v1[q] = __ldcs(a.g + o);
			}
		}
	}
}

template <int MODE, int G, int SPL>
__device__ __forceinline__ void hp_epi_apply(const HpArgs &a, const HpLanes<G, SPL> &L,
	int64_t r, const double (&acc)[SPL], const HpEpiIn<SPL> &e, const int64_t (&seedrow)[SPL],
	const double (&term)[SPL], const bool (&act)[SPL], double (&res)[SPL], double (&dng)[SPL]) {
	const int S = a.S;
	const double rs = e.rs;
	if (MODE == HP_FWD) {
#pragma unroll
		for (int q = 0; q < SPL; ++q) {
			const int s = L.seed(q);
			if (!(L.lead() && s < S && act[q])) continue;
			const int64_t o = r * S + s;
			const double old = e.v0[q];
			const double nw = acc[q] + (r == seedrow[q] ? term[q] : 0.0);
			__stcs(a.x + o, nw);
			res[q] += old > nw ? old - nw : nw - old;
			if (rs == 0.0) {
				__stcs(a.out + o, 0.0);
				dng[q] += nw;
			} else {
				__stcs(a.out + o, nw * rs);
			}
		}
	} else if (MODE == HP_ADJ) {
#pragma unroll
		for (int q = 0; q < SPL; ++q) {
			const int s = L.seed(q);
			if (!(L.lead() && s < S)) continue;
			const int64_t o = r * S + s;
			const double cur = e.v0[q];
			if (act[q]) {
				const double mu = acc[q] * rs;
				const double nw = a.alpha * mu + (rs == 0.0 ? term[q] : 0.0) + e.v1[q];
				res[q] += cur > nw ? cur - nw : nw - cur;
				__stcs(a.out + o, nw);
			} else {
				__stcs(a.out + o, cur);
			}
		}
	} else {  // HP_MU: c_r = sum_s x_rs mu_rs
		double p = 0.0;
#pragma unroll
		for (int q = 0; q < SPL; ++q) {
			const int s = L.seed(q);
			if (L.lead() && s < S) p += e.v0[q] * (acc[q] * rs);
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
		if (L.lane == 0) a.c[r] = p;
	}
}

// Reduce the lead lanes' per-seed residual and dangling sums of a block into
// bp[block][0..S) and bp[block][S..2S), in a fixed order.
template <int G, int SPL>
__device__ __forceinline__ void hp_block_partials(const HpArgs &a, const HpLanes<G, SPL> &L,
	const double (&res)[SPL], const double (&dng)[SPL], int64_t block, double *red) {
	const int S = a.S, w = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
#pragma unroll
	for (int q = 0; q < SPL; ++q) {
		const int s = L.seed(q);
		if (L.lead() && s < S) {
			red[w * 2 * S + s] = res[q];
			red[w * 2 * S + S + s] = dng[q];
		}
	}
	__syncthreads();
	for (int t = threadIdx.x; t < 2 * S; t += blockDim.x) {
		double v = 0.0;
		for (int k = 0; k < nwarps; ++k) v += red[k * 2 * S + t];
		a.bp[block * 2 * S + t] = v;
	}
}

template <int G, int SPL>
__device__ __forceinline__ void hp_load_seeds(const HpArgs &a, const HpLanes<G, SPL> &L,
	int64_t (&seedrow)[SPL], double (&term)[SPL], bool (&act)[SPL]) {
#pragma unroll
	for (int q = 0; q < SPL; ++q) {
		const int s = L.seed(q);
		const bool ok = s < a.S;
		seedrow[q] = ok ? a.sd.seed[s] : -1;
		term[q] = ok ? a.sd.term[s] : 0.0;
		act[q] = ok && a.sd.active[s] != 0;
	}
}

// Chunk descriptor of the chunk loop (warp-uniform).
struct HpMeta {
	int64_t b, r;
	int len;
	int32_t slot;
};

__device__ __forceinline__ HpMeta hp_meta(const HpArgs &a, int64_t c) {
	HpMeta m{0, 0, 0, -1};
	if (c < a.nchunks) {
		m.b = __ldg(a.beg + c);
		m.len = int(__ldg(a.beg + c + 1) - m.b);
		m.r = __ldg(a.crow + c);
		m.slot = __ldg(a.cslot + c);
	}
	return m;
}

// Main gather: one warp per chunk, chunks strided over the grid's warps.
// Lane k holds nonzero k of the chunk (index and weight); each lane group
// walks the chunk's nonzeroes in batches (stride 32 / G, warp-uniform trip
// count so the broadcasts stay converged), issuing every gather of a batch
// before its multiply-adds.  The next chunk's descriptor and the current
// row's epilogue operands are in flight during the gathers.
template <int MODE, int G, int SPL>
__global__ void __launch_bounds__(32 * HP_WARPS, ALPB_HP_MINB) k_hp_chunks(HpArgs a) {
	constexpr int STEP = 32 / G;
	constexpr int B = SPL >= 4 ? ALPB_HP_BATCH / 2 : ALPB_HP_BATCH;
	__shared__ double red[HP_WARPS * 2 * HP_MAX_SEEDS];
	if (MODE != HP_MU && *a.sd.n_active == 0) return;
	const HpLanes<G, SPL> L;
	const int S = a.S;
	int64_t seedrow[SPL];
	double term[SPL];
	bool act[SPL];
	hp_load_seeds(a, L, seedrow, term, act);
	double res[SPL], dng[SPL];
#pragma unroll
	for (int q = 0; q < SPL; ++q) res[q] = dng[q] = 0.0;
	const int64_t nw = int64_t(gridDim.x) * HP_WARPS;
	int64_t c = int64_t(blockIdx.x) * HP_WARPS + (threadIdx.x >> 5);
	HpMeta m = hp_meta(a, c);
	uint32_t myi = 0;
	double myw = 0.0;
	if (L.lane < m.len) {
		myi = __ldg(a.idx + m.b + L.lane);
		myw = __ldg(a.val + m.b + L.lane);
	}
	for (; c < a.nchunks; c += nw) {
		const HpMeta mn = hp_meta(a, c + nw);
		HpEpiIn<SPL> e;
		if (m.slot < 0) hp_epi_load<MODE>(a, L, m.r, e);
		double acc[SPL];
#pragma unroll
		for (int q = 0; q < SPL; ++q) acc[q] = 0.0;
		for (int t0 = 0; t0 < m.len; t0 += B * STEP) {
			double v[B][SPL], wv[B];
#pragma unroll
			for (int u = 0; u < B; ++u) {
				const int t = t0 + u * STEP + L.gsub;
				const uint32_t i = __shfl_sync(0xffffffffu, myi, t & 31);
				wv[u] = __shfl_sync(0xffffffffu, myw, t & 31);
				const double *src = a.in + int64_t(i) * S;
#pragma unroll
				for (int q = 0; q < SPL; ++q) {
					const int s = L.seed(q);
					v[u][q] = (t < m.len && s < S) ? __ldg(src + s) : 0.0;
				}
			}
#pragma unroll
			for (int u = 0; u < B; ++u) {
#pragma unroll
				for (int q = 0; q < SPL; ++q) acc[q] = fma(wv[u], v[u][q], acc[q]);
			}
		}
		uint32_t ni = 0;
		double nwt = 0.0;
		if (L.lane < mn.len) {
			ni = __ldg(a.idx + mn.b + L.lane);
			nwt = __ldg(a.val + mn.b + L.lane);
		}
#pragma unroll
		for (int o = G; o < 32; o <<= 1) {
#pragma unroll
			for (int q = 0; q < SPL; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
		}
		if (m.slot >= 0) {
#pragma unroll
			for (int q = 0; q < SPL; ++q) {
				const int s = L.seed(q);
				if (L.lead() && s < S) __stcg(a.part + int64_t(m.slot) * S + s, acc[q]);
			}
		} else {
			hp_epi_apply<MODE>(a, L, m.r, acc, e, seedrow, term, act, res, dng);
		}
		m = mn;
		myi = ni;
		myw = nwt;
	}
	if (MODE != HP_MU) hp_block_partials(a, L, res, dng, blockIdx.x, red);
}

// Groups of HP_GROUP_CHUNKS consecutive chunk partials of a hub row: one warp
// per group sums them in chunk order (all the group's loads issued first).
template <int G, int SPL>
__global__ void __launch_bounds__(32 * HP_WARPS) k_hp_group(HpArgs a) {
	const HpLanes<G, SPL> L;
	const int S = a.S;
	const int64_t nw = int64_t(gridDim.x) * HP_WARPS;
	for (int64_t g = int64_t(blockIdx.x) * HP_WARPS + (threadIdx.x >> 5); g < a.ngroups; g += nw) {
		const int64_t s0 = __ldg(a.gslot + g);
		const int len = __ldg(a.glen + g);
		if (!L.lead()) continue;
#pragma unroll
		for (int q = 0; q < SPL; ++q) {
			const int s = L.seed(q);
			if (s >= S) continue;
			double v[HP_GROUP_CHUNKS];
#pragma unroll
			for (int k = 0; k < HP_GROUP_CHUNKS; ++k)
				v[k] = k < len ? __ldcg(a.part + (s0 + k) * S + s) : 0.0;
			double acc = 0.0;
#pragma unroll
			for (int k = 0; k < HP_GROUP_CHUNKS; ++k)
				if (k < len) acc += v[k];
			__stcg(a.gpart + g * S + s, acc);
		}
	}
}

// Rows of several chunks: one warp per row sums its chunk partials (or, for
// a hub row, its group partials) in order and runs the row epilogue.  Block partials go after the main kernel's
// (block index offset bp_base).
template <int MODE, int G, int SPL>
__global__ void __launch_bounds__(32 * HP_WARPS) k_hp_multi(HpArgs a, int64_t bp_base) {
	__shared__ double red[HP_WARPS * 2 * HP_MAX_SEEDS];
	if (MODE != HP_MU && *a.sd.n_active == 0) return;
	const HpLanes<G, SPL> L;
	const int S = a.S;
	int64_t seedrow[SPL];
	double term[SPL];
	bool act[SPL];
	hp_load_seeds(a, L, seedrow, term, act);
	double res[SPL], dng[SPL];
#pragma unroll
	for (int q = 0; q < SPL; ++q) res[q] = dng[q] = 0.0;
	const int64_t nw = int64_t(gridDim.x) * HP_WARPS;
	for (int64_t m = int64_t(blockIdx.x) * HP_WARPS + (threadIdx.x >> 5); m < a.nmulti; m += nw) {
		const int64_t r = __ldg(a.mrow + m);
		const int32_t g0 = __ldg(a.mgroup + m);
		const int mc = __ldg(a.mcount + m);
		// partials to sum: the row's groups, else its chunk slots
		const double *src = g0 >= 0 ? a.gpart + int64_t(g0) * S : a.part + int64_t(__ldg(a.mslot + m)) * S;
		const int cnt = g0 >= 0 ? (mc + HP_GROUP_CHUNKS - 1) / HP_GROUP_CHUNKS : mc;
		HpEpiIn<SPL> e;
		hp_epi_load<MODE>(a, L, r, e);
		double acc[SPL];
#pragma unroll
		for (int q = 0; q < SPL; ++q) acc[q] = 0.0;
		if (L.lead()) {
#pragma unroll 4
			for (int k = 0; k < cnt; ++k) {
				const double *p = src + int64_t(k) * S;
#pragma unroll
				for (int q = 0; q < SPL; ++q) {
					const int s = L.seed(q);
					if (s < S) acc[q] += __ldcg(p + s);
				}
			}
		}
		hp_epi_apply<MODE>(a, L, r, acc, e, seedrow, term, act, res, dng);
	}
	if (MODE != HP_MU) hp_block_partials(a, L, res, dng, bp_base + blockIdx.x, red);
}

// Close an iteration: one block per seed sums the block partials in block
// order.  kind 0: forward iteration `iter`; 1: adjoint iteration `iter`;
// 2: forward set-up (teleport term of the initial guess); 3: adjoint set-up.
// `lam` is the adjoint iterate the next iteration reads.
__global__ void __launch_bounds__(HP_FIN_THREADS) k_hp_finish(HpSeeds sd, const double *bp,
	int64_t nblocks, int S, int kind, int64_t iter, int64_t max_iter, double conv, double alpha,
	const double *lam) {
	__shared__ double r1[HP_FIN_THREADS], r2[HP_FIN_THREADS];
	const int s = blockIdx.x;
	if ((kind == 0 || kind == 1) && *sd.n_active == 0) return;
	double res = 0.0, dng = 0.0;
	if (kind != 3) {
		for (int64_t b = threadIdx.x; b < nblocks; b += blockDim.x) {
			res += bp[b * 2 * S + s];
			dng += bp[b * 2 * S + S + s];
		}
	}
	r1[threadIdx.x] = res;
	r2[threadIdx.x] = dng;
	__syncthreads();
	for (int o = HP_FIN_THREADS / 2; o > 0; o >>= 1) {
		if (threadIdx.x < o) {
			r1[threadIdx.x] += r1[threadIdx.x + o];
			r2[threadIdx.x] += r2[threadIdx.x + o];
		}
		__syncthreads();
	}
	if (threadIdx.x != 0) return;
	res = r1[0];
	dng = r2[0];
	if (kind >= 2) {
		sd.term[s] = kind == 2 ? alpha * dng + 1 - alpha : alpha * lam[sd.seed[s] * S + s];
		sd.res[s] = 0.0;
		sd.iters[s] = 0;
		sd.active[s] = 1;
		atomicAdd(sd.n_active, 1);
		return;
	}
	if (!sd.active[s]) return;
	sd.res[s] = res;
	sd.iters[s] = iter;
	sd.term[s] = kind == 0 ? alpha * dng + 1 - alpha : alpha * lam[sd.seed[s] * S + s];
	if ((conv != 0.0 && res <= conv) || iter >= max_iter) {
		sd.active[s] = 0;
		atomicSub(sd.n_active, 1);
	}
}

// Forward set-up: initial guess (1/n unless given), its scaled input and the
// dangling mass.  One warp per row, lanes over seeds.
template <int SPL>
__global__ void __launch_bounds__(32 * HP_WARPS) k_hp_fwd_init(HpArgs a, int init_given) {
	__shared__ double red[HP_WARPS * 2 * HP_MAX_SEEDS];
	const HpLanes<32, SPL> L;
	const int S = a.S;
	double res[SPL], dng[SPL];
#pragma unroll
	for (int q = 0; q < SPL; ++q) res[q] = dng[q] = 0.0;
	const double x0 = 1.0 / double(a.n);
	const int64_t nw = int64_t(gridDim.x) * HP_WARPS;
	for (int64_t r = int64_t(blockIdx.x) * HP_WARPS + (threadIdx.x >> 5); r < a.n; r += nw) {
		const double rs = __ldg(a.rowscale + r);
#pragma unroll
		for (int q = 0; q < SPL; ++q) {
			const int s = L.seed(q);
			if (s >= S) continue;
			const int64_t o = r * S + s;
			const double x = init_given ? a.x[o] : x0;
			a.x[o] = x;
			if (rs == 0.0) {
				a.out[o] = 0.0;
				dng[q] += x;
			} else {
				a.out[o] = x * rs;
			}
		}
	}
	hp_block_partials(a, L, res, dng, blockIdx.x, red);
}

// Gradient with respect to the stored weights (CRS order):
//   grad_ij = alpha / d_i (sum_s x_is lambda_js - c_i),  c_i = sum_s x_is mu_is.
// One warp per chunk, lanes over seeds; the per-nonzero seed sums of 8
// nonzeroes are reduced together by a butterfly that halves the values held
// per lane at each step (9 shuffles for 8 sums).
template <int SPL>
__global__ void __launch_bounds__(32 * HP_WARPS) k_hp_grad(HpArgs a, const double *lam,
	double *grad) {
	const HpLanes<32, SPL> L;
	const int S = a.S, lane = L.lane;
	const int64_t nw = int64_t(gridDim.x) * HP_WARPS;
	for (int64_t c = int64_t(blockIdx.x) * HP_WARPS + (threadIdx.x >> 5); c < a.nchunks; c += nw) {
		const int64_t b = __ldg(a.beg + c);
		const int len = int(__ldg(a.beg + c + 1) - b);
		const int64_t r = __ldg(a.crow + c);
		const double inv_d = __ldg(a.rowscale + r);
		if (inv_d == 0.0) {   // dangling row: no stored weight moves x
			if (lane < len) grad[b + lane] = 0.0;
			continue;
		}
		double xr[SPL];
#pragma unroll
		for (int q = 0; q < SPL; ++q) {
			const int s = L.seed(q);
			xr[q] = s < S ? __ldg(a.x + r * S + s) : 0.0;
		}
		const double cr = __ldg(a.c + r);
		const double scale = a.alpha * inv_d;
		const uint32_t myi = lane < len ? __ldg(a.idx + b + lane) : 0u;
		for (int t0 = 0; t0 < len; t0 += 8) {
			double p[8];
#pragma unroll
			for (int u = 0; u < 8; ++u) {
				const int t = t0 + u;
				const uint32_t j = __shfl_sync(0xffffffffu, myi, t & 31);
				double v = 0.0;
				if (t < len) {
					const double *src = lam + int64_t(j) * S;
#pragma unroll
					for (int q = 0; q < SPL; ++q) {
						const int s = L.seed(q);
						if (s < S) v = fma(xr[q], __ldg(src + s), v);
					}
				}
				p[u] = v;
			}
			const bool hi = lane & 16, mid = lane & 8, lo = lane & 4;
#pragma unroll
			for (int u = 0; u < 4; ++u) {
				const double send = hi ? p[u] : p[u + 4];
				const double keep = hi ? p[u + 4] : p[u];
				p[u] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
			}
#pragma unroll
			for (int u = 0; u < 2; ++u) {
				const double send = mid ? p[u] : p[u + 2];
				const double keep = mid ? p[u + 2] : p[u];
				p[u] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
			}
			{
				const double send = lo ? p[0] : p[1];
				const double keep = lo ? p[1] : p[0];
				p[0] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
			}
			p[0] += __shfl_xor_sync(0xffffffffu, p[0], 2);
			p[0] += __shfl_xor_sync(0xffffffffu, p[0], 1);
			const int t = t0 + (hi ? 4 : 0) + (mid ? 2 : 0) + (lo ? 1 : 0);
			if ((lane & 3) == 0 && t < len) grad[b + t] = scale * (p[0] - cr);
		}
	}
}

// Weighted out-degrees: inv_d = 1 / sum_j w_ij (0 for a dangling row); flags
// a negative or non-finite weight.
__global__ void k_hp_degrees(const int64_t *ptr, const double *w, int64_t n, double *deg,
	double *inv_d, int *bad) {
	const int lane = threadIdx.x & 31;
	const int64_t nw = int64_t(gridDim.x) * (blockDim.x >> 5);
	for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nw) {
		const int64_t b = ptr[i], e = ptr[i + 1];
		double d = 0.0;
		bool neg = false;
		for (int64_t k = b + lane; k < e; k += 32) {
			const double v = w[k];
			neg |= !(v >= 0.0) || isinf(v);
			d += v;
		}
		for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
		if (__any_sync(0xffffffffu, neg) && lane == 0) *bad = 1;
		if (lane == 0) {
			deg[i] = d;
			inv_d[i] = d > 0.0 ? 1.0 / d : 0.0;
		}
	}
}

// alpha / d_i, zero for a dangling row (simple_pagerank.hpp:281-289)
__global__ void k_hp_rs(const double *deg, int64_t n, double alpha, double *rs) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x) {
		const double d = deg[i];
		rs[i] = d > 0.0 ? alpha / d : 0.0;
	}
}

__global__ void k_hp_permute(const double *w, const uint32_t *perm, int64_t nnz, double *out) {
	for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < nnz;
		 k += int64_t(gridDim.x) * blockDim.x)
		out[k] = w[perm[k]];
}

__global__ void k_hp_iota(uint32_t *p, int64_t n) {
	for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
		 k += int64_t(gridDim.x) * blockDim.x)
		p[k] = uint32_t(k);
}

}  // namespace alpb

using namespace alpb;

struct alpb_ppr_s {
	int64_t n = 0, nnz = 0;
	int S = 0;
	const int64_t *crs_ptr = nullptr;   // the caller's CRS, held by reference
	const uint32_t *crs_idx = nullptr;
	const double *w = nullptr;
	int64_t *ccs_ptr = nullptr;         // its transpose, with CRS positions
	uint32_t *ccs_idx = nullptr, *perm = nullptr;
	double *ccs_w = nullptr;
	double *deg = nullptr, *inv_d = nullptr, *rs = nullptr, *c = nullptr;
	HpChunks crs, ccs;
	double *y[2] = {nullptr, nullptr};
	double *part = nullptr, *bp = nullptr, *gpart = nullptr;
	int64_t *seed = nullptr, *iters = nullptr;
	double *term = nullptr, *res = nullptr;
	int32_t *active = nullptr, *n_active = nullptr, *h_active = nullptr;
	int *bad = nullptr;
	double alpha = 0.0;
	bool solved = false;
};

namespace {

HpSeeds seeds_of(alpb_ppr h) {
	return HpSeeds{h->seed, h->term, h->res, h->active, h->iters, h->n_active};
}

HpArgs args_over(alpb_ppr h, bool ccs) {
	HpArgs a{};
	const HpChunks &t = ccs ? h->ccs : h->crs;
	a.beg = t.beg;
	a.crow = t.row;
	a.cslot = t.slot;
	a.nchunks = t.nchunks;
	a.mrow = t.mrow;
	a.mslot = t.mslot;
	a.mcount = t.mcount;
	a.mgroup = t.mgroup;
	a.nmulti = t.nmulti;
	a.gslot = t.gslot;
	a.glen = t.glen;
	a.ngroups = t.ngroups;
	a.gpart = h->gpart;
	a.idx = ccs ? h->ccs_idx : h->crs_idx;
	a.val = ccs ? h->ccs_w : h->w;
	a.part = h->part;
	a.bp = h->bp;
	a.c = h->c;
	a.sd = seeds_of(h);
	a.n = h->n;
	a.S = h->S;
	a.alpha = h->alpha;
	return a;
}

template <int MODE, int G, int SPL>
int hp_launch(const HpArgs &a, cudaStream_t s, int64_t *nblocks) {
	const unsigned gm = grid_for(a.nchunks * 32, 32 * HP_WARPS);
	k_hp_chunks<MODE, G, SPL><<<gm, 32 * HP_WARPS, 0, s>>>(a);
	ALPB_LAUNCHED();
	int64_t nb = gm;
	if (a.ngroups > 0) {
		k_hp_group<G, SPL><<<grid_for(a.ngroups * 32, 32 * HP_WARPS), 32 * HP_WARPS, 0, s>>>(a);
		ALPB_LAUNCHED();
	}
	if (a.nmulti > 0) {
		const unsigned gx = grid_for(a.nmulti * 32, 32 * HP_WARPS);
		k_hp_multi<MODE, G, SPL><<<gx, 32 * HP_WARPS, 0, s>>>(a, gm);
		ALPB_LAUNCHED();
		nb += gx;
	}
	*nblocks = nb;
	return ALPB_SUCCESS;
}

// one gather pass over the chunks of a storage, lane layout chosen by S
template <int MODE>
int hp_pass(const HpArgs &a, cudaStream_t s, int64_t *nblocks) {
	if (a.S <= 8) return hp_launch<MODE, 8, 1>(a, s, nblocks);
	if (a.S <= 16) return hp_launch<MODE, 16, 1>(a, s, nblocks);
	if (a.S <= 32) return hp_launch<MODE, 32, 1>(a, s, nblocks);
	if (a.S <= 64) return hp_launch<MODE, 32, 2>(a, s, nblocks);
	return hp_launch<MODE, 32, 4>(a, s, nblocks);
}

int hp_fwd_init(const HpArgs &a, int init_given, cudaStream_t s, int64_t *nblocks) {
	const unsigned g = grid_for(a.n * 32, 32 * HP_WARPS);
	if (a.S <= 32) k_hp_fwd_init<1><<<g, 32 * HP_WARPS, 0, s>>>(a, init_given);
	else if (a.S <= 64) k_hp_fwd_init<2><<<g, 32 * HP_WARPS, 0, s>>>(a, init_given);
	else k_hp_fwd_init<4><<<g, 32 * HP_WARPS, 0, s>>>(a, init_given);
	ALPB_LAUNCHED();
	*nblocks = g;
	return ALPB_SUCCESS;
}

int hp_grad(const HpArgs &a, const double *lam, double *grad, cudaStream_t s) {
	const unsigned g = grid_for(a.nchunks * 32, 32 * HP_WARPS);
	if (a.S <= 32) k_hp_grad<1><<<g, 32 * HP_WARPS, 0, s>>>(a, lam, grad);
	else if (a.S <= 64) k_hp_grad<2><<<g, 32 * HP_WARPS, 0, s>>>(a, lam, grad);
	else k_hp_grad<4><<<g, 32 * HP_WARPS, 0, s>>>(a, lam, grad);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int hp_finish(alpb_ppr h, int64_t nblocks, int kind, int64_t iter, int64_t max_iter, double conv,
	const double *lam, cudaStream_t s) {
	k_hp_finish<<<h->S, HP_FIN_THREADS, 0, s>>>(seeds_of(h), h->bp, nblocks, h->S, kind, iter,
		max_iter, conv, h->alpha, lam);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

// true once every seed has stopped (reads the device count)
int hp_all_stopped(alpb_ppr h, cudaStream_t s, bool *stopped) {
	ALPB_CUDA(cudaMemcpyAsync(h->h_active, h->n_active, 4, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	*stopped = *h->h_active == 0;
	return ALPB_SUCCESS;
}

// per-seed iteration counts and residuals to the caller; the largest count
int hp_results(alpb_ppr h, int64_t *iterations, double *residuals, double conv, int64_t *last,
	cudaStream_t s) {
	std::vector<int64_t> it(h->S);
	std::vector<double> res(h->S);
	ALPB_CUDA(cudaMemcpyAsync(it.data(), h->iters, size_t(h->S) * 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaMemcpyAsync(res.data(), h->res, size_t(h->S) * 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	int64_t mx = 0;
	bool ok = true;
	for (int q = 0; q < h->S; ++q) {
		if (iterations) iterations[q] = it[q];
		if (residuals) residuals[q] = res[q];
		mx = it[q] > mx ? it[q] : mx;
		if (conv != 0.0 && !(res[q] <= conv)) ok = false;
	}
	*last = mx;
	return ok ? ALPB_SUCCESS : ALPB_FAILED;
}

int hp_weights(alpb_ppr h, cudaStream_t s) {
	if (h->nnz > 0) {
		k_hp_permute<<<grid_for(h->nnz, 256), 256, 0, s>>>(h->w, h->perm, h->nnz, h->ccs_w);
		ALPB_LAUNCHED();
	}
	ALPB_CUDA(cudaMemsetAsync(h->bad, 0, sizeof(int), s));
	k_hp_degrees<<<grid_for(h->n * 32, 256), 256, 0, s>>>(h->crs_ptr, h->w, h->n, h->deg, h->inv_d,
		h->bad);
	ALPB_LAUNCHED();
	int bad = 0;
	ALPB_CUDA(cudaMemcpyAsync(&bad, h->bad, sizeof(int), cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	ALPB_CHECK(!bad, ALPB_ILLEGAL, "ppr: edge weights must be finite and non-negative");
	return ALPB_SUCCESS;
}

}  // namespace

extern "C" {

int alpb_ppr_destroy(alpb_ppr h) {
	if (!h) return ALPB_SUCCESS;
	cudaFree(h->ccs_ptr);
	cudaFree(h->ccs_idx);
	cudaFree(h->perm);
	cudaFree(h->ccs_w);
	cudaFree(h->deg);
	cudaFree(h->inv_d);
	cudaFree(h->rs);
	cudaFree(h->c);
	chunks_free(&h->crs);
	chunks_free(&h->ccs);
	cudaFree(h->y[0]);
	cudaFree(h->y[1]);
	cudaFree(h->part);
	cudaFree(h->gpart);
	cudaFree(h->bp);
	cudaFree(h->seed);
	cudaFree(h->iters);
	cudaFree(h->term);
	cudaFree(h->res);
	cudaFree(h->active);
	cudaFree(h->n_active);
	cudaFree(h->bad);
	if (h->h_active) cudaFreeHost(h->h_active);
	delete h;
	return ALPB_SUCCESS;
}

int alpb_ppr_create(alpb_ppr *out, int64_t n, int64_t nnz, const int64_t *row_ptr,
	const uint32_t *col_idx, const double *weights, int nseeds, void *stream) {
	ALPB_CHECK(out != nullptr, ALPB_ILLEGAL, "alpb_ppr_create: null handle");
	*out = nullptr;
	ALPB_CHECK(n > 0 && nnz >= 0, ALPB_ILLEGAL, "alpb_ppr_create: bad sizes");
	ALPB_CHECK(n <= int64_t(UINT32_MAX) && nnz < (int64_t(1) << 31), ALPB_OVERFLW,
		"alpb_ppr_create: graph too large");
	ALPB_CHECK(nseeds >= 1 && nseeds <= HP_MAX_SEEDS, ALPB_UNSUPPORTED,
		"alpb_ppr_create: nseeds must be in [1, %d]", HP_MAX_SEEDS);
	ALPB_CHECK(row_ptr && (nnz == 0 || (col_idx && weights)), ALPB_ILLEGAL,
		"alpb_ppr_create: null storage");
	cudaStream_t s = as_stream(stream);
	auto *h = new alpb_ppr_s();
	h->n = n;
	h->nnz = nnz;
	h->S = nseeds;
	h->crs_ptr = row_ptr;
	h->crs_idx = col_idx;
	h->w = weights;
	const size_t vec = size_t(n) * size_t(nseeds) * 8;
	const size_t nz = size_t(nnz > 0 ? nnz : 1);
	const size_t bp = size_t(2) * size_t(sm_count()) * 8 * 2 * HP_MAX_SEEDS * 8;
	bool ok = cudaMalloc(&h->ccs_ptr, size_t(n + 1) * 8) == cudaSuccess &&
		cudaMalloc(&h->ccs_idx, nz * 4) == cudaSuccess &&
		cudaMalloc(&h->perm, nz * 4) == cudaSuccess &&
		cudaMalloc(&h->ccs_w, nz * 8) == cudaSuccess &&
		cudaMalloc(&h->deg, size_t(n) * 8) == cudaSuccess &&
		cudaMalloc(&h->inv_d, size_t(n) * 8) == cudaSuccess &&
		cudaMalloc(&h->rs, size_t(n) * 8) == cudaSuccess &&
		cudaMalloc(&h->c, size_t(n) * 8) == cudaSuccess &&
		cudaMalloc(&h->y[0], vec) == cudaSuccess && cudaMalloc(&h->y[1], vec) == cudaSuccess &&
		cudaMalloc(&h->bp, bp) == cudaSuccess &&
		cudaMalloc(&h->seed, HP_MAX_SEEDS * 8) == cudaSuccess &&
		cudaMalloc(&h->iters, HP_MAX_SEEDS * 8) == cudaSuccess &&
		cudaMalloc(&h->term, HP_MAX_SEEDS * 8) == cudaSuccess &&
		cudaMalloc(&h->res, HP_MAX_SEEDS * 8) == cudaSuccess &&
		cudaMalloc(&h->active, HP_MAX_SEEDS * 4) == cudaSuccess &&
		cudaMalloc(&h->n_active, 4) == cudaSuccess && cudaMalloc(&h->bad, 4) == cudaSuccess &&
		cudaMallocHost(&h->h_active, 4) == cudaSuccess;
	if (!ok) {
		cudaGetLastError();
		alpb_ppr_destroy(h);
		set_error("alpb_ppr_create: out of device memory");
		return ALPB_OUTOFMEM;
	}
	int rc = ALPB_SUCCESS;
	if (nnz > 0) {   // CCS with the CRS position of every entry
		uint32_t *iota = nullptr;
		if (cudaMallocAsync(&iota, size_t(nnz) * 4, s) != cudaSuccess) {
			cudaGetLastError();
			alpb_ppr_destroy(h);
			set_error("alpb_ppr_create: out of device memory");
			return ALPB_OUTOFMEM;
		}
		k_hp_iota<<<grid_for(nnz, 256), 256, 0, s>>>(iota, nnz);
		g_launches.fetch_add(1);
		rc = alpb_crs_transpose(n, n, nnz, row_ptr, col_idx, iota, ALPB_UINT32, h->ccs_ptr,
			h->ccs_idx, h->perm, stream);
		cudaFreeAsync(iota, s);
	} else if (cudaMemsetAsync(h->ccs_ptr, 0, size_t(n + 1) * 8, s) != cudaSuccess) {
		rc = ALPB_PANIC;
	}
	rc = rc ? rc : chunks_build(&h->crs, row_ptr, n, s);
	rc = rc ? rc : chunks_build(&h->ccs, h->ccs_ptr, n, s);
	if (rc == ALPB_SUCCESS) {
		const int64_t slots = h->crs.nslots > h->ccs.nslots ? h->crs.nslots : h->ccs.nslots;
		const int64_t groups = h->crs.ngroups > h->ccs.ngroups ? h->crs.ngroups : h->ccs.ngroups;
		if (cudaMalloc(&h->part, size_t(slots > 0 ? slots : 1) * nseeds * 8) != cudaSuccess ||
			cudaMalloc(&h->gpart, size_t(groups > 0 ? groups : 1) * nseeds * 8) != cudaSuccess) {
			cudaGetLastError();
			set_error("alpb_ppr_create: out of device memory");
			rc = ALPB_OUTOFMEM;
		}
	}
	rc = rc ? rc : hp_weights(h, s);
	if (rc != ALPB_SUCCESS) {
		alpb_ppr_destroy(h);
		return rc;
	}
	*out = h;
	return ALPB_SUCCESS;
}

int alpb_ppr_set_weights(alpb_ppr h, const double *weights, void *stream) {
	ALPB_CHECK(h != nullptr, ALPB_ILLEGAL, "alpb_ppr_set_weights: null handle");
	ALPB_CHECK(weights || h->nnz == 0, ALPB_ILLEGAL, "alpb_ppr_set_weights: null weights");
	const double *old = h->w;
	h->w = weights;
	const int rc = hp_weights(h, as_stream(stream));
	if (rc == ALPB_ILLEGAL) {   // rejected weights: keep the previous ones
		h->w = old;
		const int rc2 = hp_weights(h, as_stream(stream));
		if (rc2 != ALPB_SUCCESS) return rc2;
		set_error("ppr: edge weights must be finite and non-negative");
	}
	return rc;
}

int alpb_ppr_solve(alpb_ppr h, const int64_t *seeds, double alpha, double conv, int64_t max_iter,
	double *x, int init_given, int64_t *iterations, double *residuals, void *stream) {
	ALPB_CHECK(h != nullptr && seeds && x, ALPB_ILLEGAL, "alpb_ppr_solve: null argument");
	ALPB_CHECK(alpha > 0 && alpha < 1, ALPB_ILLEGAL, "alpb_ppr_solve: alpha must be in (0, 1)");
	ALPB_CHECK(max_iter > 0 && conv >= 0, ALPB_ILLEGAL, "alpb_ppr_solve: bad max_iter/conv");
	for (int q = 0; q < h->S; ++q)
		ALPB_CHECK(seeds[q] >= 0 && seeds[q] < h->n, ALPB_MISMATCH,
			"alpb_ppr_solve: seed %d out of range", q);
	cudaStream_t s = as_stream(stream);
	ALPB_CUDA(cudaMemcpyAsync(h->seed, seeds, size_t(h->S) * 8, cudaMemcpyHostToDevice, s));
	h->alpha = alpha;
	h->solved = false;
	k_hp_rs<<<grid_for(h->n, 256), 256, 0, s>>>(h->deg, h->n, alpha, h->rs);
	ALPB_LAUNCHED();
	ALPB_CUDA(cudaMemsetAsync(h->n_active, 0, 4, s));
	HpArgs a = args_over(h, true);
	a.rowscale = h->rs;
	a.x = x;
	a.out = h->y[0];
	int64_t nb = 0;
	int rc = hp_fwd_init(a, init_given, s, &nb);
	rc = rc ? rc : hp_finish(h, nb, 2, 0, max_iter, conv, nullptr, s);
	for (int64_t k = 1; rc == ALPB_SUCCESS && k <= max_iter; ++k) {
		a.in = h->y[(k - 1) & 1];
		a.out = h->y[k & 1];
		rc = hp_pass<HP_FWD>(a, s, &nb);
		rc = rc ? rc : hp_finish(h, nb, 0, k, max_iter, conv, nullptr, s);
		if (rc == ALPB_SUCCESS && (k % 8 == 0 || k == max_iter)) {
			bool stopped = false;
			rc = hp_all_stopped(h, s, &stopped);
			if (stopped) break;
		}
	}
	if (rc != ALPB_SUCCESS) return rc;
	int64_t last = 0;
	rc = hp_results(h, iterations, residuals, conv, &last, s);
	h->solved = rc == ALPB_SUCCESS || rc == ALPB_FAILED;
	return rc;
}

int alpb_ppr_adjoint(alpb_ppr h, const double *dl_dx, double *lambda, double conv,
	int64_t max_iter, int64_t *iterations, double *residuals, void *stream) {
	ALPB_CHECK(h != nullptr && dl_dx && lambda, ALPB_ILLEGAL, "alpb_ppr_adjoint: null argument");
	ALPB_CHECK(h->solved, ALPB_ILLEGAL, "alpb_ppr_adjoint: no forward solve on this handle");
	ALPB_CHECK(dl_dx != lambda, ALPB_OVERLAP, "alpb_ppr_adjoint: dl_dx and lambda overlap");
	ALPB_CHECK(max_iter > 0 && conv >= 0, ALPB_ILLEGAL, "alpb_ppr_adjoint: bad max_iter/conv");
	cudaStream_t s = as_stream(stream);
	const size_t vec = size_t(h->n) * size_t(h->S) * 8;
	double *buf[2] = {lambda, h->y[0]};
	ALPB_CUDA(cudaMemcpyAsync(lambda, dl_dx, vec, cudaMemcpyDeviceToDevice, s));
	ALPB_CUDA(cudaMemsetAsync(h->n_active, 0, 4, s));
	int rc = hp_finish(h, 0, 3, 0, max_iter, conv, lambda, s);
	HpArgs a = args_over(h, false);
	a.rowscale = h->inv_d;
	a.g = dl_dx;
	for (int64_t k = 1; rc == ALPB_SUCCESS && k <= max_iter; ++k) {
		a.in = buf[(k - 1) & 1];
		a.out = buf[k & 1];
		int64_t nb = 0;
		rc = hp_pass<HP_ADJ>(a, s, &nb);
		rc = rc ? rc : hp_finish(h, nb, 1, k, max_iter, conv, buf[k & 1], s);
		if (rc == ALPB_SUCCESS && (k % 8 == 0 || k == max_iter)) {
			bool stopped = false;
			rc = hp_all_stopped(h, s, &stopped);
			if (stopped) break;
		}
	}
	if (rc != ALPB_SUCCESS) return rc;
	int64_t last = 0;
	rc = hp_results(h, iterations, residuals, conv, &last, s);
	if (last & 1) {   // the last iteration wrote the internal buffer
		ALPB_CUDA(cudaMemcpyAsync(lambda, h->y[0], vec, cudaMemcpyDeviceToDevice, s));
		ALPB_CUDA(cudaStreamSynchronize(s));
	}
	return rc;
}

int alpb_ppr_grad_weights(alpb_ppr h, const double *x, const double *lambda, double *grad,
	void *stream) {
	ALPB_CHECK(h != nullptr && x && lambda && (grad || h->nnz == 0), ALPB_ILLEGAL,
		"alpb_ppr_grad_weights: null argument");
	ALPB_CHECK(h->solved, ALPB_ILLEGAL, "alpb_ppr_grad_weights: no forward solve on this handle");
	cudaStream_t s = as_stream(stream);
	HpArgs a = args_over(h, false);
	a.rowscale = h->inv_d;
	a.in = lambda;
	a.x = const_cast<double *>(x);
	int64_t nb = 0;
	int rc = hp_pass<HP_MU>(a, s, &nb);
	if (rc == ALPB_SUCCESS && h->nnz > 0) rc = hp_grad(a, lambda, grad, s);
	return rc;
}

int alpb_ppr_info(alpb_ppr h, int64_t *chunks_ccs, int64_t *multi_ccs, int64_t *chunks_crs,
	int64_t *multi_crs) {
	ALPB_CHECK(h != nullptr, ALPB_ILLEGAL, "alpb_ppr_info: null handle");
	if (chunks_ccs) *chunks_ccs = h->ccs.nchunks;
	if (multi_ccs) *multi_ccs = h->ccs.nmulti;
	if (chunks_crs) *chunks_crs = h->crs.nchunks;
	if (multi_crs) *multi_crs = h->crs.nmulti;
	return ALPB_SUCCESS;
}

}  // extern "C"
