// Fused HPCG: algorithms::hpcg (hpcg/hpcg.hpp:97-223), its multigrid V-cycle
// (hpcg/multigrid_v_cycle.hpp:67-246) and the multi-colour Gauss-Seidel
// smoother (hpcg/red_black_gauss_seidel.hpp:55-123) as device kernels, for
// the system build_hpcg_system makes (hpcg/system_building_utils.hpp:84-150):
// the 3-D 27-point box stencil on every level, levels coarsened by 2 per
// dimension, injection as the coarsening matrix, static colours (row index
// modulo the colour count).
//
// Several right-hand sides are solved together: vectors hold the nrhs values
// of a row side by side (row-major), so every pass over a matrix serves all
// of them.  Each right-hand side keeps its own CG scalars and its own
// convergence test, exactly as separate runs of the algorithm would.
//
// Kernels (all FP64, each row's sum in CRS order):
//   k_hpcg_rows<NRHS, Op>  one kernel for every row-wise product: the SpMM
//                          A p, a colour step of the smoother (x_i = (r_i -
//                          (A x)_i + x_i d) / d on the rows of one colour),
//                          the restriction (r_c = r_f - A z at injected fine
//                          rows only) and the prolongation (z_f += z_c)
//   k_hpcg_dot / k_hpcg_finish  per-right-hand-side dot products in a fixed
//                          order, and the CG scalar updates on the device
//   k_hpcg_axpy...         the CG vector updates
#include "common.cuh"

#include <cmath>
#include <vector>

namespace alpb {

constexpr int HG_GROUP = 8;     // lanes per matrix row
constexpr int HG_BLOCK = 256;

// Row-wise product engine: a group of 8 lanes per row; lane q handles the
// right-hand side q % NRHS and the nonzeroes s, s + S, ... of the row, with
// s = q / NRHS and S = 8 / NRHS; the S partial sums are combined by an xor
// tree.  With NRHS = 8 every lane walks its row in CRS order.
template <int NRHS, class Op>
__global__ void __launch_bounds__(HG_BLOCK)
k_hpcg_rows(const int64_t *__restrict__ offsets, const uint32_t *__restrict__ indices,
	const double *__restrict__ values, const double *__restrict__ x, int64_t count, Op op) {
	constexpr int S = HG_GROUP / NRHS;
	constexpr int GPW = 32 / HG_GROUP;  // row groups per warp
	const int q = threadIdx.x & (HG_GROUP - 1);
	const int k = q % NRHS, s = q / NRHS;
	const int g = (threadIdx.x & 31) / HG_GROUP;
	const int64_t warp = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
	const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
	// the loop bound is the same for the whole warp, so every lane reaches
	// every shuffle below
	for (int64_t wb = warp * GPW; wb < count; wb += nwarps * GPW) {
		const int64_t idx = wb + g;
		const bool valid = idx < count;
		double acc = 0.0;
		int64_t row = 0;
		if (valid) {
			row = op.row(idx);
			const int64_t b = offsets[row], e = offsets[row + 1];
			for (int64_t j = b + s; j < e; j += S)
				acc += values[j] * x[int64_t(indices[j]) * NRHS + k];
		}
#pragma unroll
		for (int o = NRHS; o < HG_GROUP; o <<= 1) {
			const double w = __shfl_xor_sync(0xffffffffu, acc, o);
			acc += w;
		}
		if (valid && s == 0) op.finish(idx, row, k, acc);
	}
}

// ------------------------------------------------------- row operations --
// y = 0 + A x on every row (set( y, 0 ); mxv( y, A, x ))
template <int NRHS>
struct HgSpmm {
	double *y;
	__device__ __forceinline__ int64_t row(int64_t i) const { return i; }
	__device__ __forceinline__ void finish(int64_t, int64_t r, int k, double acc) const {
		y[r * NRHS + k] = 0.0 + acc;
	}
};

// One colour step of the smoother on rows c, c + K, c + 2K, ... (the rows
// whose index is c modulo K), red_black_gauss_seidel.hpp:63-86:
//   temp = 0 + A[mask] x;  x[mask] = (r - temp + x d) / d.
// Fused (temp never stored) when no two neighbours share a colour, so that
// no row of the colour reads another's new value; otherwise `temp` receives
// the products and k_hpcg_color_update applies them.
template <int NRHS>
struct HgColor {
	const double *r;
	double *x;
	double *temp;  // null: fused
	double d;
	int64_t c, K;
	__device__ __forceinline__ int64_t row(int64_t i) const { return c + i * K; }
	__device__ __forceinline__ void finish(int64_t, int64_t row, int k, double acc) const {
		const double t = 0.0 + acc;
		const int64_t at = row * NRHS + k;
		if (temp) {
			temp[at] = t;
		} else {
			const double v = r[at] - t + x[at] * d;
			x[at] = v / d;
		}
	}
};

template <int NRHS>
__global__ void k_hpcg_color_update(const double *r, const double *temp, double *x, double d,
	int64_t c, int64_t K, int64_t count) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count * NRHS;
		 i += int64_t(gridDim.x) * blockDim.x) {
		const int64_t at = (c + (i / NRHS) * K) * NRHS + i % NRHS;
		const double v = r[at] - temp[at] + x[at] * d;
		x[at] = v / d;
	}
}

// Fine row of coarse point c under injection: coarse (cx, cy, cz) takes the
// fine point (2cx, 2cy, 2cz) (coarsener_generator_iterator,
// ndim_matrix_builders.hpp:412-541; x varies fastest).
struct HgInject {
	int64_t cnx, cny, fnx, fny;
	__device__ __forceinline__ int64_t operator()(int64_t c) const {
		const int64_t cx = c % cnx, cy = (c / cnx) % cny, cz = c / (cnx * cny);
		return 2 * cx + 2 * cy * fnx + 2 * cz * fnx * fny;
	}
};

// Restriction, compute_coarsening (multigrid_v_cycle.hpp:67-86): with
// Ax = 0 + A z, r_c = 0 + 1 (r_f - Ax) at the injected rows; the product is
// formed only where the injection reads it.
template <int NRHS>
struct HgRestrict {
	const double *r_f;
	double *r_c;
	HgInject inj;
	__device__ __forceinline__ int64_t row(int64_t c) const { return inj(c); }
	__device__ __forceinline__ void finish(int64_t c, int64_t f, int k, double acc) const {
		const double ax = 0.0 + acc;
		r_c[c * NRHS + k] = 0.0 + 1.0 * (r_f[f * NRHS + k] - ax);
	}
};

// Prolongation, compute_prolongation (multigrid_v_cycle.hpp:88-103):
// z_f += 0 + 1 z_c at the injected rows (the other rows add zero).
template <int NRHS>
__global__ void k_hpcg_prolong(double *z_f, const double *z_c, HgInject inj, int64_t count) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count * NRHS;
		 i += int64_t(gridDim.x) * blockDim.x) {
		const int64_t c = i / NRHS;
		const int k = int(i % NRHS);
		const int64_t at = inj(c) * NRHS + k;
		z_f[at] = z_f[at] + (0.0 + 1.0 * z_c[i]);
	}
}

// ------------------------------------------------------------ CG pieces --
// Per-right-hand-side dot products x_k . y_k: block partials, then one block
// sums them in block order (fixed order: deterministic).
template <int NRHS>
__global__ void __launch_bounds__(HG_BLOCK)
k_hpcg_dot(const double *__restrict__ x, const double *__restrict__ y, int64_t n,
	double *partials) {
	__shared__ double sm[HG_BLOCK];
	// thread t handles right-hand side t % NRHS (HG_BLOCK is a multiple of NRHS)
	double acc = 0.0;
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n * NRHS;
		 i += int64_t(gridDim.x) * blockDim.x)
		acc += x[i] * y[i];
	sm[threadIdx.x] = acc;
	__syncthreads();
	for (int w = HG_BLOCK / 2; w >= NRHS; w >>= 1) {
		if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
		__syncthreads();
	}
	if (threadIdx.x < NRHS) partials[blockIdx.x * NRHS + threadIdx.x] = sm[threadIdx.x];
}

// out[k] = 0 + sum over blocks of partials[., k]
template <int NRHS>
__global__ void k_hpcg_dot_finish(const double *partials, int nblocks, double *out) {
	const int k = threadIdx.x;
	if (k >= NRHS) return;
	double v = 0.0;
	for (int b = 0; b < nblocks; ++b) v += partials[b * NRHS + k];
	out[k] = 0.0 + v;
}

// Device-side CG state of one right-hand side.
struct HgScalars {
	double norm0, norm, rz, rz_old, pap, alpha, beta;
	int64_t iterations;
	int32_t active;
	int32_t pad;
};

template <int NRHS>
__global__ void k_hpcg_axpby(double *out, const double *a, const double *b, const HgScalars *sc,
	int which, int64_t n) {
	// which 0: out = b - a   (r = b - Ap, eWiseApply with minus)
	//       1: out = beta a + b  (Ap = beta p + z, eWiseMulAdd into a cleared vector)
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n * NRHS;
		 i += int64_t(gridDim.x) * blockDim.x) {
		const int k = int(i % NRHS);
		if (which == 0) out[i] = b[i] - a[i];
		else out[i] = sc[k].active ? sc[k].beta * a[i] + b[i] : a[i];  // finished: p kept
	}
}

// x += alpha p; r += -alpha Ap (eWiseMul with the ring, hpcg.hpp:206-207)
template <int NRHS>
__global__ void k_hpcg_update(double *x, double *r, const double *p, const double *ap,
	const HgScalars *sc, int64_t n) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n * NRHS;
		 i += int64_t(gridDim.x) * blockDim.x) {
		const int k = int(i % NRHS);
		if (!sc[k].active) continue;
		const double al = sc[k].alpha;
		x[i] = x[i] + al * p[i];
		r[i] = r[i] + (-al) * ap[i];
	}
}

// Scalar steps, one thread per right-hand side.  step 0: after r.r of the
// initial residual; 1: after r.z; 2: after p.Ap; 3: after the new r.r.
template <int NRHS>
__global__ void k_hpcg_scalars(HgScalars *sc, const double *dot, int step, int64_t iter,
	int64_t max_iter, double tol) {
	const int k = threadIdx.x;
	if (k >= NRHS) return;
	HgScalars &s = sc[k];
	switch (step) {
	case 0:
		s.norm0 = sqrt(dot[k]);
		s.norm = s.norm0;
		s.iterations = 0;
		s.active = 1;
		s.rz = 0.0;
		break;
	case 1:
		if (!s.active) return;
		s.rz_old = s.rz;
		s.rz = dot[k];
		s.beta = iter == 0 ? 0.0 : s.rz / s.rz_old;
		break;
	case 2:
		if (!s.active) return;
		s.pap = dot[k];
		s.alpha = s.rz / s.pap;
		break;
	case 3:
		if (!s.active) return;
		s.norm = sqrt(dot[k]);
		s.iterations = iter + 1;
		// do { ... } while( iter < max && norm / norm0 > tol )  (hpcg.hpp:209)
		if (!(s.iterations < max_iter && s.norm / s.norm0 > tol)) s.active = 0;
		break;
	}
}

}  // namespace alpb

namespace alpb {

// 1 where two neighbouring rows share a colour (row index modulo K).
__global__ void k_hpcg_color_conflicts(const int64_t *offsets, const uint32_t *indices, int64_t n,
	int64_t K, int32_t *flag) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x)
		for (int64_t j = offsets[i]; j < offsets[i + 1]; ++j) {
			const int64_t c = indices[j];
			if (c != i && (c % K) == (i % K)) atomicExch(flag, 1);
		}
}

// ------------------------------------------------- recognising a system --
// Checks of a caller's level against this handle's (alpb_hpcg_match_level);
// each sets *bad on the first difference it sees.
__global__ void k_hg_words_differ(const uint32_t *a, const uint32_t *b, int64_t words,
	int32_t *bad) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < words;
		 i += int64_t(gridDim.x) * blockDim.x)
		if (a[i] != b[i]) {
			*bad = 1;
			return;
		}
}

// every entry assigned and equal to the handle's diagonal value
__global__ void k_hg_check_diag(const double *d, const uint8_t *flags, int64_t n, double diag,
	int32_t *bad) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x)
		if ((flags && !flags[i]) || d[i] != diag) {
			*bad = 1;
			return;
		}
}

// colour c of `colors`: assigned (and true) exactly at the rows i = c mod colors
// (build_static_color_masks, hpcg/matrix_building_utils.hpp:131-165)
__global__ void k_hg_check_mask(const uint8_t *vals, const uint8_t *flags, int64_t n,
	int64_t colors, int64_t c, int32_t *bad) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x) {
		const bool want = i % colors == c;
		const bool has = flags ? flags[i] != 0 : true;
		if (has != want || (has && vals[i] == 0)) {
			*bad = 1;
			return;
		}
	}
}

// the injection coarsener of build_ndims_coarsener_matrix: coarse row c holds
// one 1 at fine column inj(c)
__global__ void k_hg_check_coarsening(const int64_t *off, const uint32_t *idx, const double *val,
	int64_t nc, int64_t fine_n, int64_t cnx, int64_t cny, int64_t fnx, int64_t fny,
	int32_t *bad) {
	for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c <= nc;
		 c += int64_t(gridDim.x) * blockDim.x) {
		if (off[c] != c) {
			*bad = 1;
			return;
		}
		if (c == nc) continue;
		const int64_t cx = c % cnx, cy = (c / cnx) % cny, cz = c / (cnx * cny);
		const int64_t f = 2 * cx + 2 * cy * fnx + 2 * cz * fnx * fny;
		if (f >= fine_n || int64_t(idx[c]) != f || val[c] != 1.0) {
			*bad = 1;
			return;
		}
	}
}

struct HgLevel {
	int64_t nx = 0, ny = 0, nz = 0, n = 0, nnz = 0;
	int64_t *offsets = nullptr;
	uint32_t *indices = nullptr;
	double *values = nullptr;
	double *r = nullptr, *z = nullptr, *temp = nullptr;  // n * nrhs each
	bool fused = true;
};

}  // namespace alpb

using namespace alpb;

struct alpb_hpcg_s {
	std::vector<HgLevel> levels;   // [0] is the finest (the system itself)
	int nrhs = 1;
	int64_t colors = 27;
	double diag = 26.0;
	double *p = nullptr, *ap = nullptr;  // CG vectors of the finest level
	double *partials = nullptr, *dots = nullptr;
	HgScalars *scalars = nullptr;
	int dot_blocks = 0;
};

namespace alpb {

template <int NRHS, class Op>
static int hg_rows(const HgLevel &L, const double *x, int64_t count, const Op &op, cudaStream_t s) {
	if (count <= 0) return ALPB_SUCCESS;
	k_hpcg_rows<NRHS, Op><<<grid_for(count * HG_GROUP, HG_BLOCK), HG_BLOCK, 0, s>>>(L.offsets,
		L.indices, L.values, x, count, op);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

// red_black_gauss_seidel: colours forward, then backward (:96-117)
template <int NRHS>
static int hg_smoother(alpb_hpcg_s *h, HgLevel &L, cudaStream_t s) {
	const int64_t K = h->colors;
	for (int pass = 0; pass < 2; ++pass)
		for (int64_t q = 0; q < K; ++q) {
			const int64_t c = pass == 0 ? q : K - 1 - q;
			const int64_t count = c < L.n ? (L.n - 1 - c) / K + 1 : 0;
			HgColor<NRHS> op{L.r, L.z, L.fused ? nullptr : L.temp, h->diag, c, K};
			int rc = hg_rows<NRHS>(L, L.z, count, op, s);
			if (rc != ALPB_SUCCESS) return rc;
			if (!L.fused && count > 0) {
				k_hpcg_color_update<NRHS><<<grid_for(count * NRHS, 256), 256, 0, s>>>(L.r, L.temp,
					L.z, h->diag, c, K, count);
				ALPB_LAUNCHED();
			}
		}
	return ALPB_SUCCESS;
}

// multi_grid (multigrid_v_cycle.hpp:193-246): z = 0; smooth; restrict the
// residual; recurse; prolong; smooth.  The coarsest level smooths once.
template <int NRHS>
static int hg_vcycle(alpb_hpcg_s *h, size_t l, int64_t pre, int64_t post, cudaStream_t s) {
	HgLevel &L = h->levels[l];
	ALPB_CUDA(cudaMemsetAsync(L.z, 0, size_t(L.n) * NRHS * 8, s));
	int rc = ALPB_SUCCESS;
	if (l + 1 == h->levels.size()) return hg_smoother<NRHS>(h, L, s);
	for (int64_t i = 0; i < pre && rc == ALPB_SUCCESS; ++i) rc = hg_smoother<NRHS>(h, L, s);
	if (rc != ALPB_SUCCESS) return rc;
	HgLevel &Cl = h->levels[l + 1];
	const HgInject inj{Cl.nx, Cl.ny, L.nx, L.ny};
	rc = hg_rows<NRHS>(L, L.z, Cl.n, HgRestrict<NRHS>{L.r, Cl.r, inj}, s);
	if (rc != ALPB_SUCCESS) return rc;
	rc = hg_vcycle<NRHS>(h, l + 1, pre, post, s);
	if (rc != ALPB_SUCCESS) return rc;
	k_hpcg_prolong<NRHS><<<grid_for(Cl.n * NRHS, 256), 256, 0, s>>>(L.z, Cl.z, inj, Cl.n);
	ALPB_LAUNCHED();
	for (int64_t i = 0; i < post && rc == ALPB_SUCCESS; ++i) rc = hg_smoother<NRHS>(h, L, s);
	return rc;
}

template <int NRHS>
static int hg_dot(alpb_hpcg_s *h, const double *x, const double *y, int64_t n, cudaStream_t s) {
	k_hpcg_dot<NRHS><<<h->dot_blocks, HG_BLOCK, 0, s>>>(x, y, n, h->partials);
	ALPB_LAUNCHED();
	k_hpcg_dot_finish<NRHS><<<1, 32, 0, s>>>(h->partials, h->dot_blocks, h->dots);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

// algorithms::hpcg (hpcg.hpp:97-223) for NRHS right-hand sides at once
template <int NRHS>
static int hg_solve(alpb_hpcg_s *h, const double *b, double *x, bool precondition, int64_t pre,
	int64_t post, int64_t max_iter, double tol, int64_t *iterations, double *residuals,
	cudaStream_t s) {
	HgLevel &L = h->levels[0];
	const int64_t n = L.n;
	const unsigned g = grid_for(n * NRHS, 256);
	// Ap = 0; r = 0; p = x; Ap = A x; r = b - Ap; norm = sqrt(r.r)
	ALPB_CUDA(cudaMemcpyAsync(h->p, x, size_t(n) * NRHS * 8, cudaMemcpyDeviceToDevice, s));
	int rc = hg_rows<NRHS>(L, x, n, HgSpmm<NRHS>{h->ap}, s);
	if (rc != ALPB_SUCCESS) return rc;
	k_hpcg_axpby<NRHS><<<g, 256, 0, s>>>(L.r, h->ap, b, h->scalars, 0, n);
	ALPB_LAUNCHED();
	hg_dot<NRHS>(h, L.r, L.r, n, s);
	k_hpcg_scalars<NRHS><<<1, 32, 0, s>>>(h->scalars, h->dots, 0, 0, max_iter, tol);
	ALPB_LAUNCHED();
	HgScalars hs[NRHS];
	for (int64_t iter = 0;; ++iter) {
		if (precondition) {
			rc = hg_vcycle<NRHS>(h, 0, pre, post, s);
			if (rc != ALPB_SUCCESS) return rc;
		} else {
			ALPB_CUDA(cudaMemcpyAsync(L.z, L.r, size_t(n) * NRHS * 8, cudaMemcpyDeviceToDevice, s));
		}
		// r.z, beta; p = z (first iteration) or p = beta p + z
		hg_dot<NRHS>(h, L.r, L.z, n, s);
		k_hpcg_scalars<NRHS><<<1, 32, 0, s>>>(h->scalars, h->dots, 1, iter, max_iter, tol);
		ALPB_LAUNCHED();
		if (iter == 0) {
			ALPB_CUDA(cudaMemcpyAsync(h->p, L.z, size_t(n) * NRHS * 8, cudaMemcpyDeviceToDevice, s));
		} else {
			// into Ap, then swapped with p (hpcg.hpp:193-196)
			k_hpcg_axpby<NRHS><<<g, 256, 0, s>>>(h->ap, h->p, L.z, h->scalars, 1, n);
			ALPB_LAUNCHED();
			double *t = h->p;
			h->p = h->ap;
			h->ap = t;
		}
		// Ap = A p; alpha = r.z / p.Ap; x += alpha p; r -= alpha Ap; norm
		rc = hg_rows<NRHS>(L, h->p, n, HgSpmm<NRHS>{h->ap}, s);
		if (rc != ALPB_SUCCESS) return rc;
		hg_dot<NRHS>(h, h->ap, h->p, n, s);
		k_hpcg_scalars<NRHS><<<1, 32, 0, s>>>(h->scalars, h->dots, 2, iter, max_iter, tol);
		ALPB_LAUNCHED();
		k_hpcg_update<NRHS><<<g, 256, 0, s>>>(x, L.r, h->p, h->ap, h->scalars, n);
		ALPB_LAUNCHED();
		hg_dot<NRHS>(h, L.r, L.r, n, s);
		k_hpcg_scalars<NRHS><<<1, 32, 0, s>>>(h->scalars, h->dots, 3, iter, max_iter, tol);
		ALPB_LAUNCHED();
		ALPB_CUDA(cudaMemcpyAsync(hs, h->scalars, sizeof(hs), cudaMemcpyDeviceToHost, s));
		ALPB_CUDA(cudaStreamSynchronize(s));
		bool any = false;
		for (int k = 0; k < NRHS; ++k) any = any || hs[k].active;
		if (!any) break;
	}
	for (int k = 0; k < NRHS; ++k) {
		if (iterations) iterations[k] = hs[k].iterations;
		if (residuals) residuals[k] = hs[k].norm;
	}
	return ALPB_SUCCESS;
}

}  // namespace alpb

extern "C" {

int alpb_hpcg_destroy(alpb_hpcg h) {
	if (!h) return ALPB_SUCCESS;
	for (HgLevel &L : h->levels) {
		cudaFree(L.offsets);
		cudaFree(L.indices);
		cudaFree(L.values);
		cudaFree(L.r);
		cudaFree(L.z);
		cudaFree(L.temp);
	}
	cudaFree(h->p);
	cudaFree(h->ap);
	cudaFree(h->partials);
	cudaFree(h->dots);
	cudaFree(h->scalars);
	delete h;
	return ALPB_SUCCESS;
}

int alpb_hpcg_create(alpb_hpcg *out, int64_t nx, int64_t ny, int64_t nz, double diag,
	double off, int64_t colors, int64_t min_size, int64_t max_levels, int nrhs, void *stream) {
	ALPB_CHECK(out != nullptr, ALPB_ILLEGAL, "alpb_hpcg_create: null handle");
	*out = nullptr;
	ALPB_CHECK(nx > 0 && ny > 0 && nz > 0 && colors > 0 && min_size > 0 && max_levels >= 0,
		ALPB_ILLEGAL, "alpb_hpcg_create: bad sizes");
	ALPB_CHECK(nrhs == 1 || nrhs == 2 || nrhs == 4 || nrhs == 8, ALPB_UNSUPPORTED,
		"alpb_hpcg_create: %d right-hand sides (1, 2, 4 or 8)", nrhs);
	ALPB_CHECK(diag != 0.0, ALPB_ILLEGAL, "alpb_hpcg_create: zero diagonal");
	ALPB_CHECK(nx * ny * nz >= colors, ALPB_ILLEGAL,
		"alpb_hpcg_create: fewer rows than colours");  // build_static_color_masks
	cudaStream_t s = as_stream(stream);
	auto *h = new alpb_hpcg_s();
	h->nrhs = nrhs;
	h->colors = colors;
	h->diag = diag;
	// levels as build_hpcg_system makes them (system_building_utils.hpp:107-147)
	std::vector<int64_t> dims = {nx, ny, nz};
	int64_t min_coarse = std::min(nx, std::min(ny, nz)) / 2;
	h->levels.push_back(HgLevel{});
	h->levels.back().nx = nx;
	h->levels.back().ny = ny;
	h->levels.back().nz = nz;
	int64_t level = 0;
	while (min_coarse >= min_size && level < max_levels) {
		HgLevel c;
		c.nx = h->levels.back().nx / 2;
		c.ny = h->levels.back().ny / 2;
		c.nz = h->levels.back().nz / 2;
		if (c.nx * 2 != h->levels.back().nx || c.ny * 2 != h->levels.back().ny ||
			c.nz * 2 != h->levels.back().nz) {
			alpb_hpcg_destroy(h);
			set_error("alpb_hpcg_create: level sizes must halve exactly");
			return ALPB_ILLEGAL;
		}
		h->levels.push_back(c);
		min_coarse /= 2;
		++level;
	}
	int32_t *flag = nullptr;
	int rc = ALPB_SUCCESS;
	if (cudaMallocAsync(&flag, 4, s) != cudaSuccess) {
		alpb_hpcg_destroy(h);
		set_error("alpb_hpcg_create: out of device memory");
		return ALPB_OUTOFMEM;
	}
	for (HgLevel &L : h->levels) {
		L.n = L.nx * L.ny * L.nz;
		int64_t sizes[4] = {L.nx, L.ny, L.nz, 0};
		if (cudaMalloc(&L.offsets, size_t(L.n + 1) * 8) != cudaSuccess) {
			cudaGetLastError();
			rc = ALPB_OUTOFMEM;
			set_error("alpb_hpcg_create: out of device memory");
			break;
		}
		// first call: row offsets and the nonzero count
		rc = alpb_gen_stencil_crs(3, sizes, diag, off, 1, L.offsets, nullptr, nullptr, &L.nnz,
			stream);
		if (rc != ALPB_SUCCESS) break;
		const size_t vbytes = size_t(L.n) * nrhs * 8;
		if (cudaMalloc(&L.indices, size_t(L.nnz) * 4) != cudaSuccess ||
			cudaMalloc(&L.values, size_t(L.nnz) * 8) != cudaSuccess ||
			cudaMalloc(&L.r, vbytes) != cudaSuccess || cudaMalloc(&L.z, vbytes) != cudaSuccess) {
			cudaGetLastError();
			rc = ALPB_OUTOFMEM;
			set_error("alpb_hpcg_create: out of device memory");
			break;
		}
		rc = alpb_gen_stencil_crs(3, sizes, diag, off, 1, L.offsets, L.indices, L.values, &L.nnz,
			stream);
		if (rc != ALPB_SUCCESS) break;
		// the smoother fuses a colour's product and update when no two
		// neighbours share a colour
		int32_t conflict = 0;
		if (cudaMemsetAsync(flag, 0, 4, s) != cudaSuccess) { rc = ALPB_PANIC; break; }
		k_hpcg_color_conflicts<<<grid_for(L.n, 256), 256, 0, s>>>(L.offsets, L.indices, L.n,
			colors, flag);
		ALPB_LAUNCHED();
		if (cudaMemcpyAsync(&conflict, flag, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
			cudaStreamSynchronize(s) != cudaSuccess) {
			rc = ALPB_PANIC;
			set_error("alpb_hpcg_create: colour check failed");
			break;
		}
		L.fused = conflict == 0;
		if (!L.fused && cudaMalloc(&L.temp, vbytes) != cudaSuccess) {
			cudaGetLastError();
			rc = ALPB_OUTOFMEM;
			set_error("alpb_hpcg_create: out of device memory");
			break;
		}
	}
	cudaFreeAsync(flag, s);
	const int64_t n0 = h->levels[0].n;
	if (rc == ALPB_SUCCESS) {
		h->dot_blocks = int(grid_for(n0 * nrhs, HG_BLOCK, 2));
		if (cudaMalloc(&h->p, size_t(n0) * nrhs * 8) != cudaSuccess ||
			cudaMalloc(&h->ap, size_t(n0) * nrhs * 8) != cudaSuccess ||
			cudaMalloc(&h->partials, size_t(h->dot_blocks) * nrhs * 8) != cudaSuccess ||
			cudaMalloc(&h->dots, size_t(nrhs) * 8) != cudaSuccess ||
			cudaMalloc(&h->scalars, size_t(nrhs) * sizeof(HgScalars)) != cudaSuccess) {
			cudaGetLastError();
			rc = ALPB_OUTOFMEM;
			set_error("alpb_hpcg_create: out of device memory");
		}
	}
	if (rc != ALPB_SUCCESS) {
		alpb_hpcg_destroy(h);
		return rc;
	}
	*out = h;
	return ALPB_SUCCESS;
}

int alpb_hpcg_info(alpb_hpcg h, int64_t *levels, int64_t *n_finest, int64_t *nnz_finest,
	int *fused_smoother) {
	ALPB_CHECK(h != nullptr, ALPB_ILLEGAL, "alpb_hpcg_info: null handle");
	if (levels) *levels = int64_t(h->levels.size());
	if (n_finest) *n_finest = h->levels[0].n;
	if (nnz_finest) *nnz_finest = h->levels[0].nnz;
	if (fused_smoother) {
		int all = 1;
		for (const HgLevel &L : h->levels) all &= L.fused ? 1 : 0;
		*fused_smoother = all;
	}
	return ALPB_SUCCESS;
}

int alpb_hpcg_matrix(alpb_hpcg h, int64_t level, const int64_t **offsets,
	const uint32_t **indices, const double **values, int64_t *n, int64_t *nnz) {
	ALPB_CHECK(h != nullptr && level >= 0 && level < int64_t(h->levels.size()), ALPB_ILLEGAL,
		"alpb_hpcg_matrix: no level %lld", (long long) level);
	const HgLevel &L = h->levels[size_t(level)];
	if (offsets) *offsets = L.offsets;
	if (indices) *indices = L.indices;
	if (values) *values = L.values;
	if (n) *n = L.n;
	if (nnz) *nnz = L.nnz;
	return ALPB_SUCCESS;
}

int alpb_hpcg_solve(alpb_hpcg h, const double *b, double *x, int with_preconditioning,
	int64_t presmoother_steps, int64_t postsmoother_steps, int64_t max_iterations,
	double tolerance, int64_t *iterations, double *residuals, void *stream) {
	ALPB_CHECK(h != nullptr && b != nullptr && x != nullptr, ALPB_ILLEGAL,
		"alpb_hpcg_solve: null argument");
	ALPB_CHECK(max_iterations > 0 && presmoother_steps >= 0 && postsmoother_steps >= 0,
		ALPB_ILLEGAL, "alpb_hpcg_solve: bad iteration counts");
	cudaStream_t s = as_stream(stream);
	const bool pc = with_preconditioning != 0;
	switch (h->nrhs) {
	case 1: return hg_solve<1>(h, b, x, pc, presmoother_steps, postsmoother_steps, max_iterations,
		tolerance, iterations, residuals, s);
	case 2: return hg_solve<2>(h, b, x, pc, presmoother_steps, postsmoother_steps, max_iterations,
		tolerance, iterations, residuals, s);
	case 4: return hg_solve<4>(h, b, x, pc, presmoother_steps, postsmoother_steps, max_iterations,
		tolerance, iterations, residuals, s);
	default: return hg_solve<8>(h, b, x, pc, presmoother_steps, postsmoother_steps,
		max_iterations, tolerance, iterations, residuals, s);
	}
}

int alpb_hpcg_match_level(alpb_hpcg h, int64_t level, int64_t n, int64_t nnz,
	const int64_t *offsets, const uint32_t *indices, const double *values, const double *diagonal,
	const uint8_t *diagonal_flags, int64_t colors, const uint8_t *const *mask_values,
	const uint8_t *const *mask_flags, int64_t coarse_nnz, const int64_t *coarse_offsets,
	const uint32_t *coarse_indices, const double *coarse_values, int *matches, void *stream) {
	ALPB_CHECK(h != nullptr && matches != nullptr, ALPB_ILLEGAL,
		"alpb_hpcg_match_level: null argument");
	*matches = 0;
	if (level < 0 || level >= int64_t(h->levels.size())) return ALPB_SUCCESS;
	const HgLevel &L = h->levels[size_t(level)];
	if (n != L.n || nnz != L.nnz || colors != h->colors || !offsets || (nnz && (!indices ||
			!values)) || !diagonal || (colors && (!mask_values || !mask_flags)))
		return ALPB_SUCCESS;
	if (level > 0 && (coarse_nnz != L.n || !coarse_offsets || !coarse_indices || !coarse_values))
		return ALPB_SUCCESS;
	cudaStream_t s = as_stream(stream);
	int32_t *bad = nullptr;
	ALPB_CUDA(cudaMallocAsync(&bad, 4, s));
	ALPB_CUDA(cudaMemsetAsync(bad, 0, 4, s));
	const void *const pa[3] = {offsets, indices, values};
	const void *const pb[3] = {L.offsets, L.indices, L.values};
	const int64_t nw[3] = {2 * (n + 1), nnz, 2 * nnz};   // 4-byte words
	for (int k = 0; k < 3; ++k) {
		if (nw[k] == 0) continue;
		k_hg_words_differ<<<grid_for(nw[k], 256, 2), 256, 0, s>>>(
			static_cast<const uint32_t *>(pa[k]), static_cast<const uint32_t *>(pb[k]), nw[k], bad);
		ALPB_LAUNCHED();
	}
	k_hg_check_diag<<<grid_for(n, 256, 2), 256, 0, s>>>(diagonal, diagonal_flags, n, h->diag,
		bad);
	ALPB_LAUNCHED();
	for (int64_t c = 0; c < colors; ++c) {
		k_hg_check_mask<<<grid_for(n, 256, 2), 256, 0, s>>>(mask_values[c], mask_flags[c], n,
			colors, c, bad);
		ALPB_LAUNCHED();
	}
	if (level > 0) {
		const HgLevel &F = h->levels[size_t(level - 1)];
		k_hg_check_coarsening<<<grid_for(L.n + 1, 256, 2), 256, 0, s>>>(coarse_offsets,
			coarse_indices, coarse_values, L.n, F.n, L.nx, L.ny, F.nx, F.ny, bad);
		ALPB_LAUNCHED();
	}
	int32_t hb = 1;
	ALPB_CUDA(cudaMemcpyAsync(&hb, bad, 4, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaFreeAsync(bad, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	*matches = hb == 0 ? 1 : 0;
	return ALPB_SUCCESS;
}

}  // extern "C"
