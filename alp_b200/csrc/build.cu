// Synthetic generators and device-side matrix construction.
//
// buildMatrixUnique of the reference (include/graphblas/reference/matrix.hpp:
// 1854-1951) is a two-pass counting sort that places the nonzeroes of a row in
// the REVERSE of their input order (decrementing fill, :1921-1930) and builds
// CRS and CCS together.  Here the same result is produced with a stable radix
// sort by row (CUB) followed by an in-segment reversal, all on the device.
#include "common.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <cub/device/device_scan.cuh>

namespace alpb {

// ------------------------------------------------------------ generators --
__global__ void k_hash_u64(uint64_t *out, int64_t n, uint64_t seed, uint64_t sid) {
	for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
		 k += int64_t(gridDim.x) * blockDim.x)
		out[k] = hash3(seed, sid, uint64_t(k));
}

__global__ void k_gen_values(void *out, int type, int64_t n, uint64_t seed, uint64_t sid,
	int32_t lo, int32_t hi, double p) {
	for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
		 k += int64_t(gridDim.x) * blockDim.x) {
		const uint64_t h = hash3(seed, sid, uint64_t(k));
		switch (type) {
		case ALPB_FP64: reinterpret_cast<double *>(out)[k] = u01(h); break;
		case ALPB_INT32:
			reinterpret_cast<int32_t *>(out)[k] =
				lo + int32_t(h % uint64_t(int64_t(hi) - int64_t(lo) + 1));
			break;
		case ALPB_BOOL: reinterpret_cast<uint8_t *>(out)[k] = u01(h) < p ? 1 : 0; break;
		default: break;
		}
	}
}

// R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004): each of `scale` levels picks a
// quadrant with probabilities a, b, c, d from one hash draw; level 0 sets the
// most significant bit.  Integer thresholds make CPU and GPU agree exactly.
__global__ void k_rmat(uint64_t *keys, int64_t n, int scale, uint64_t ta, uint64_t tab,
	uint64_t tabc, uint64_t seed) {
	for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
		 e += int64_t(gridDim.x) * blockDim.x) {
		uint64_t r = 0, c = 0;
		for (int l = 0; l < scale; ++l) {
			const uint64_t h = hash3(seed, uint64_t(e), uint64_t(l));
			const uint64_t rb = h >= tab ? 1u : 0u;
			const uint64_t cb = (h >= ta && h < tab) || h >= tabc ? 1u : 0u;
			r = (r << 1) | rb;
			c = (c << 1) | cb;
		}
		keys[e] = (r << 32) | c;
	}
}

__global__ void k_row_ptr_from_keys(const uint64_t *keys, int64_t nnz, int64_t m, int64_t *row_ptr) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i <= m;
		 i += int64_t(gridDim.x) * blockDim.x) {
		// lower_bound of (i << 32)
		const uint64_t target = uint64_t(i) << 32;
		int64_t lo = 0, hi = nnz;
		while (lo < hi) {
			const int64_t mid = (lo + hi) >> 1;
			if (keys[mid] < target) lo = mid + 1; else hi = mid;
		}
		row_ptr[i] = lo;
	}
}

__global__ void k_col_from_keys(const uint64_t *keys, int64_t nnz, uint32_t *col) {
	for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < nnz;
		 k += int64_t(gridDim.x) * blockDim.x)
		col[k] = uint32_t(keys[k] & 0xffffffffu);
}

// row of each nonzero by upper_bound over the offsets
__device__ __forceinline__ int64_t row_of(const int64_t *row_ptr, int64_t m, int64_t k) {
	int64_t lo = 0, hi = m;  // find largest i with row_ptr[i] <= k
	while (lo < hi) {
		const int64_t mid = (lo + hi + 1) >> 1;
		if (row_ptr[mid] <= k) lo = mid; else hi = mid - 1;
	}
	return lo;
}

__global__ void k_edge_values(void *vals, int type, const int64_t *row_ptr, const uint32_t *col,
	int64_t m, int64_t nnz, uint64_t seed, int32_t lo, int32_t hi) {
	for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < nnz;
		 k += int64_t(gridDim.x) * blockDim.x) {
		const int64_t i = row_of(row_ptr, m, k);
		const uint64_t key = (uint64_t(i) << 32) | col[k];
		const uint64_t h = hash3(seed, key, 0x5eedull);
		if (type == ALPB_FP64)
			reinterpret_cast<double *>(vals)[k] = u01(h);
		else if (type == ALPB_INT32)
			reinterpret_cast<int32_t *>(vals)[k] =
				lo + int32_t(h % uint64_t(int64_t(hi) - int64_t(lo) + 1));
		else if (type == ALPB_BOOL)
			reinterpret_cast<uint8_t *>(vals)[k] = 1;
	}
}

// ------------------------------------------------------------- COO build --
__global__ void k_check_coords(const uint32_t *I, const uint32_t *J, int64_t nnz, int64_t m,
	int64_t n, int *bad) {
	for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < nnz;
		 k += int64_t(gridDim.x) * blockDim.x)
		if (int64_t(I[k]) >= m || int64_t(J[k]) >= n) *bad = 1;
}

__global__ void k_iota_u32(uint32_t *v, int64_t n) {
	for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
		 k += int64_t(gridDim.x) * blockDim.x)
		v[k] = uint32_t(k);
}

__global__ void k_row_ptr_from_sorted_rows(const uint32_t *rows, int64_t nnz, int64_t m,
	int64_t *row_ptr) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i <= m;
		 i += int64_t(gridDim.x) * blockDim.x) {
		int64_t lo = 0, hi = nnz;
		while (lo < hi) {
			const int64_t mid = (lo + hi) >> 1;
			if (int64_t(rows[mid]) < i) lo = mid + 1; else hi = mid;
		}
		row_ptr[i] = lo;
	}
}

// Scatter in reverse order inside each row: sorted position p of row i goes to
// row_ptr[i] + row_ptr[i+1] - 1 - p.
__global__ void k_scatter_reversed(const uint32_t *sorted_rows, const uint32_t *perm,
	const int64_t *row_ptr, const uint32_t *J, const void *vals, int vsize, int reverse,
	int64_t nnz, uint32_t *col, void *out_vals) {
	for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < nnz;
		 p += int64_t(gridDim.x) * blockDim.x) {
		const uint32_t i = sorted_rows[p];
		const int64_t dst = reverse ? row_ptr[i] + row_ptr[i + 1] - 1 - p : p;
		const uint32_t src = perm[p];
		col[dst] = J[src];
		if (vsize == 8)
			reinterpret_cast<double *>(out_vals)[dst] = reinterpret_cast<const double *>(vals)[src];
		else if (vsize == 4)
			reinterpret_cast<int32_t *>(out_vals)[dst] = reinterpret_cast<const int32_t *>(vals)[src];
		else if (vsize == 1)
			reinterpret_cast<uint8_t *>(out_vals)[dst] = reinterpret_cast<const uint8_t *>(vals)[src];
	}
}

__global__ void k_expand_rows(const int64_t *row_ptr, int64_t m, uint32_t *rows) {
	// warp per row
	const int lane = threadIdx.x & 31;
	for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < m;
		 i += (int64_t(gridDim.x) * blockDim.x) >> 5)
		for (int64_t k = row_ptr[i] + lane; k < row_ptr[i + 1]; k += 32) rows[k] = uint32_t(i);
}

// ---------------------------------------------------------- stencils --
struct Grid {
	int dims;
	int64_t s[4];
};

__device__ __forceinline__ int64_t stencil_row_nnz(const Grid g, int64_t row) {
	int64_t cnt = 1, r = row;
	for (int d = 0; d < g.dims; ++d) {
		const int64_t c = r % g.s[d];
		r /= g.s[d];
		const int64_t lo = c > 0 ? c - 1 : 0;
		const int64_t hi = c + 1 < g.s[d] ? c + 1 : g.s[d] - 1;
		cnt *= hi - lo + 1;
	}
	return cnt;
}

__global__ void k_stencil_counts(Grid g, int64_t m, int64_t *counts) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m;
		 i += int64_t(gridDim.x) * blockDim.x)
		counts[i] = stencil_row_nnz(g, i);
}

// columns of a row in increasing order: dimension 0 fastest, as the iterator
// of hpcg/ndim_matrix_builders.hpp:288-338 visits them
__global__ void k_stencil_fill(Grid g, int64_t m, const int64_t *row_ptr, double diag,
	double off, int ref_order, uint32_t *col, double *val) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m;
		 i += int64_t(gridDim.x) * blockDim.x) {
		int64_t c[4], lo[4], hi[4], cur[4], stride[4];
		int64_t r = i, st = 1;
		for (int d = 0; d < g.dims; ++d) {
			c[d] = r % g.s[d];
			r /= g.s[d];
			lo[d] = c[d] > 0 ? c[d] - 1 : 0;
			hi[d] = c[d] + 1 < g.s[d] ? c[d] + 1 : g.s[d] - 1;
			cur[d] = lo[d];
			stride[d] = st;
			st *= g.s[d];
		}
		const int64_t begin = row_ptr[i], end = row_ptr[i + 1];
		for (int64_t t = 0; t < end - begin; ++t) {
			int64_t j = 0;
			for (int d = 0; d < g.dims; ++d) j += cur[d] * stride[d];
			const int64_t dst = ref_order ? end - 1 - t : begin + t;
			col[dst] = uint32_t(j);
			if (val) val[dst] = (j == i) ? diag : off;
			for (int d = 0; d < g.dims; ++d) {  // odometer, dimension 0 fastest
				if (cur[d] < hi[d]) { ++cur[d]; break; }
				cur[d] = lo[d];
			}
		}
	}
}

__global__ void k_poisson2d(int64_t L, double shift, int64_t *row_ptr, uint32_t *col, double *val) {
	const int64_t m = L * L;
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m;
		 i += int64_t(gridDim.x) * blockDim.x) {
		const int64_t x = i % L, y = i / L;
		// offset of row i in closed form: a grid line y has 4L-2 nonzeroes at
		// the two boundary lines and 5L-2 inside; within line y, each earlier
		// point x' contributes 1 + [x'>0] + 1 + [y>0] + [y<L-1].
		const int64_t py = (y > 0) + (y < L - 1);
		int64_t start = y == 0 ? 0 : (4 * L - 2) + (y - 1) * (5 * L - 2);
		start += x * (3 + py) - (x > 0 ? 1 : 0);
		if (i == m - 1) row_ptr[m] = start + 1 + (x > 0) + (x < L - 1) + py;
		row_ptr[i] = start;
		int64_t p = start;
		if (y > 0) { col[p] = uint32_t(i - L); val[p++] = -1.0; }
		if (x > 0) { col[p] = uint32_t(i - 1); val[p++] = -1.0; }
		col[p] = uint32_t(i); val[p++] = 4.0 + shift;
		if (x < L - 1) { col[p] = uint32_t(i + 1); val[p++] = -1.0; }
		if (y < L - 1) { col[p] = uint32_t(i + L); val[p++] = -1.0; }
	}
}

// block-diagonal batch of 5-point Poisson systems
__global__ void k_poisson2d_batch(int64_t nseg, const int64_t *Ls, const double *shifts,
	const int64_t *seg_rows, const int64_t *seg_nnz, int64_t total, int64_t *row_ptr,
	uint32_t *col, double *val) {
	for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total;
		 g += int64_t(gridDim.x) * blockDim.x) {
		int64_t lo = 0, hi = nseg - 1;  // instance: last s with seg_rows[s] <= g
		while (lo < hi) {
			const int64_t mid = (lo + hi + 1) >> 1;
			if (seg_rows[mid] <= g) lo = mid; else hi = mid - 1;
		}
		const int64_t s = lo, L = Ls[s], r0 = seg_rows[s], i = g - r0;
		const int64_t x = i % L, y = i / L;
		const int64_t py = (y > 0) + (y < L - 1);
		int64_t start = y == 0 ? 0 : (4 * L - 2) + (y - 1) * (5 * L - 2);
		start += x * (3 + py) - (x > 0 ? 1 : 0);
		start += seg_nnz[s];
		row_ptr[g] = start;
		if (g == total - 1) row_ptr[total] = start + 1 + (x > 0) + (x < L - 1) + py;
		int64_t p = start;
		if (y > 0) { col[p] = uint32_t(g - L); val[p++] = -1.0; }
		if (x > 0) { col[p] = uint32_t(g - 1); val[p++] = -1.0; }
		col[p] = uint32_t(g); val[p++] = 4.0 + shifts[s];
		if (x < L - 1) { col[p] = uint32_t(g + 1); val[p++] = -1.0; }
		if (y < L - 1) { col[p] = uint32_t(g + L); val[p++] = -1.0; }
	}
}

// Symmetric, strictly diagonally dominant values on a CRS pattern: the
// off-diagonal (i, j) takes -(lo + (hi - lo) u) with u hashed from the
// unordered pair, so A = A^T; the diagonal takes factor * sum_j |a_ij|.
__global__ void k_sym_dd_values(const int64_t *row_ptr, const uint32_t *col, int64_t m,
	uint64_t seed, double lo, double hi, double factor, double *val) {
	const int lane = threadIdx.x & 31;
	for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < m;
		 i += (int64_t(gridDim.x) * blockDim.x) >> 5) {
		double sum = 0.0;
		for (int64_t k = row_ptr[i] + lane; k < row_ptr[i + 1]; k += 32) {
			const uint64_t j = col[k];
			if (int64_t(j) == i) continue;
			const uint64_t a = uint64_t(i) < j ? uint64_t(i) : j, b = uint64_t(i) < j ? j : uint64_t(i);
			const double v = -(lo + (hi - lo) * u01(hash3(seed, (a << 32) | b, 0x5e11ull)));
			val[k] = v;
			sum += -v;
		}
		for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
		sum = __shfl_sync(0xffffffffu, sum, 0);
		for (int64_t k = row_ptr[i] + lane; k < row_ptr[i + 1]; k += 32)
			if (int64_t(col[k]) == i) val[k] = factor * sum;
	}
}

// Box-Muller (Box & Muller, Ann. Math. Statist. 29, 1958) on two hash draws
__global__ void k_gen_normal(double *out, int64_t n, uint64_t seed, uint64_t sid) {
	for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
		 k += int64_t(gridDim.x) * blockDim.x) {
		const double u1 = 1.0 - u01(hash3(seed, sid, uint64_t(2 * k)));  // (0, 1]
		const double u2 = u01(hash3(seed, sid, uint64_t(2 * k + 1)));
		out[k] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
	}
}

} // namespace alpb

using namespace alpb;

static uint64_t threshold_u64(double p) {
	if (p <= 0.0) return 0;
	if (p >= 1.0) return ~uint64_t(0);
	return uint64_t(p * 18446744073709551616.0);
}

extern "C" {

int alpb_gen_hash_u64(uint64_t *out, int64_t count, uint64_t seed, uint64_t sid, void *stream) {
	if (count <= 0) return ALPB_SUCCESS;
	k_hash_u64<<<grid_for(count, 256), 256, 0, as_stream(stream)>>>(out, count, seed, sid);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_gen_values(void *out, int type, int64_t count, uint64_t seed, uint64_t sid, int32_t lo,
	int32_t hi, double p, void *stream) {
	ALPB_CHECK(type == ALPB_FP64 || type == ALPB_INT32 || type == ALPB_BOOL, ALPB_UNSUPPORTED,
		"alpb_gen_values: type %d", type);
	ALPB_CHECK(hi >= lo, ALPB_ILLEGAL, "alpb_gen_values: hi < lo");
	if (count <= 0) return ALPB_SUCCESS;
	k_gen_values<<<grid_for(count, 256), 256, 0, as_stream(stream)>>>(out, type, count, seed, sid,
		lo, hi, p);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_gen_rmat_keys(uint64_t *keys, int64_t n, int scale, double a, double b, double c,
	uint64_t seed, void *stream) {
	ALPB_CHECK(scale >= 1 && scale <= 31, ALPB_ILLEGAL, "alpb_gen_rmat_keys: scale %d", scale);
	ALPB_CHECK(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0, ALPB_ILLEGAL,
		"alpb_gen_rmat_keys: bad probabilities");
	if (n <= 0) return ALPB_SUCCESS;
	k_rmat<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(keys, n, scale, threshold_u64(a),
		threshold_u64(a + b), threshold_u64(a + b + c), seed);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_gen_edge_values(void *values, int type, const int64_t *row_ptr, const uint32_t *col,
	int64_t m, int64_t nnz, uint64_t seed, int32_t lo, int32_t hi, void *stream) {
	ALPB_CHECK(type == ALPB_FP64 || type == ALPB_INT32 || type == ALPB_BOOL, ALPB_UNSUPPORTED,
		"alpb_gen_edge_values: type %d", type);
	if (nnz <= 0) return ALPB_SUCCESS;
	k_edge_values<<<grid_for(nnz, 256), 256, 0, as_stream(stream)>>>(values, type, row_ptr, col, m,
		nnz, seed, lo, hi);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_keys_sort_unique(uint64_t *keys, int64_t n, int64_t *n_unique, void *stream) {
	ALPB_CHECK(n_unique != nullptr, ALPB_ILLEGAL, "alpb_keys_sort_unique: null n_unique");
	*n_unique = 0;
	if (n <= 0) return ALPB_SUCCESS;
	ALPB_CHECK(n < (int64_t(1) << 31), ALPB_OVERFLW, "alpb_keys_sort_unique: n too large for one sort");
	cudaStream_t s = as_stream(stream);
	uint64_t *alt = nullptr;
	int64_t *d_cnt = nullptr;
	void *tmp = nullptr;
	size_t tmp_sort = 0, tmp_uniq = 0;
	ALPB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_sort, keys, keys, int(n), 0, 64, s));
	ALPB_CUDA(cub::DeviceSelect::Unique(nullptr, tmp_uniq, keys, keys, d_cnt, int(n), s));
	const size_t tmp_bytes = tmp_sort > tmp_uniq ? tmp_sort : tmp_uniq;
	ALPB_CUDA(cudaMallocAsync(&alt, size_t(n) * 8, s));
	ALPB_CUDA(cudaMallocAsync(&tmp, tmp_bytes, s));
	ALPB_CUDA(cudaMallocAsync(&d_cnt, 8, s));
	cub::DoubleBuffer<uint64_t> db(keys, alt);
	size_t t1 = tmp_bytes;
	ALPB_CUDA(cub::DeviceRadixSort::SortKeys(tmp, t1, db, int(n), 0, 64, s));
	g_launches.fetch_add(1);
	uint64_t *sorted = db.Current();
	uint64_t *other = sorted == keys ? alt : keys;
	size_t t2 = tmp_bytes;
	ALPB_CUDA(cub::DeviceSelect::Unique(tmp, t2, sorted, other, d_cnt, int(n), s));
	g_launches.fetch_add(1);
	int64_t cnt = 0;
	ALPB_CUDA(cudaMemcpyAsync(&cnt, d_cnt, 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	if (other != keys) ALPB_CUDA(cudaMemcpyAsync(keys, other, size_t(cnt) * 8, cudaMemcpyDeviceToDevice, s));
	ALPB_CUDA(cudaFreeAsync(alt, s));
	ALPB_CUDA(cudaFreeAsync(tmp, s));
	ALPB_CUDA(cudaFreeAsync(d_cnt, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	*n_unique = cnt;
	return ALPB_SUCCESS;
}

int alpb_crs_from_sorted_keys(const uint64_t *keys, int64_t nnz, int64_t m, int64_t *row_ptr,
	uint32_t *col_idx, void *stream) {
	ALPB_CHECK(m >= 0 && nnz >= 0, ALPB_ILLEGAL, "alpb_crs_from_sorted_keys: negative size");
	cudaStream_t s = as_stream(stream);
	k_row_ptr_from_keys<<<grid_for(m + 1, 256), 256, 0, s>>>(keys, nnz, m, row_ptr);
	ALPB_LAUNCHED();
	if (nnz > 0) {
		k_col_from_keys<<<grid_for(nnz, 256), 256, 0, s>>>(keys, nnz, col_idx);
		ALPB_LAUNCHED();
	}
	return ALPB_SUCCESS;
}

// shared by coo_to_crs and crs_transpose: stable sort of (row key, position)
static int sorted_build(int64_t m, int64_t nnz, const uint32_t *rows_in, const uint32_t *J,
	const void *values, int type, int reverse, int64_t *row_ptr, uint32_t *col_idx,
	void *out_values, cudaStream_t s) {
	const size_t vs = type_size(type);
	ALPB_CHECK(type == ALPB_VOID || vs > 0, ALPB_UNSUPPORTED, "build: value type %d", type);
	ALPB_CHECK(vs == 0 || (values && out_values), ALPB_ILLEGAL, "build: null values");
	ALPB_CHECK(nnz < (int64_t(1) << 31), ALPB_OVERFLW, "build: nnz too large for one sort");
	if (nnz == 0) {
		ALPB_CUDA(cudaMemsetAsync(row_ptr, 0, size_t(m + 1) * 8, s));
		return ALPB_SUCCESS;
	}
	uint32_t *keys_out = nullptr, *perm_in = nullptr, *perm_out = nullptr;
	void *tmp = nullptr;
	size_t tmp_bytes = 0;
	int end_bit = 1;
	while (end_bit < 32 && (int64_t(1) << end_bit) < m) ++end_bit;
	ALPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, rows_in, keys_out, perm_in,
		perm_out, int(nnz), 0, end_bit, s));
	ALPB_CUDA(cudaMallocAsync(&keys_out, size_t(nnz) * 4, s));
	ALPB_CUDA(cudaMallocAsync(&perm_in, size_t(nnz) * 4, s));
	ALPB_CUDA(cudaMallocAsync(&perm_out, size_t(nnz) * 4, s));
	ALPB_CUDA(cudaMallocAsync(&tmp, tmp_bytes, s));
	k_iota_u32<<<grid_for(nnz, 256), 256, 0, s>>>(perm_in, nnz);
	ALPB_LAUNCHED();
	ALPB_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, rows_in, keys_out, perm_in, perm_out,
		int(nnz), 0, end_bit, s));
	g_launches.fetch_add(1);
	k_row_ptr_from_sorted_rows<<<grid_for(m + 1, 256), 256, 0, s>>>(keys_out, nnz, m, row_ptr);
	ALPB_LAUNCHED();
	k_scatter_reversed<<<grid_for(nnz, 256), 256, 0, s>>>(keys_out, perm_out, row_ptr, J, values,
		int(vs), reverse, nnz, col_idx, out_values);
	ALPB_LAUNCHED();
	ALPB_CUDA(cudaFreeAsync(keys_out, s));
	ALPB_CUDA(cudaFreeAsync(perm_in, s));
	ALPB_CUDA(cudaFreeAsync(perm_out, s));
	ALPB_CUDA(cudaFreeAsync(tmp, s));
	return ALPB_SUCCESS;
}

int alpb_coo_to_crs(int64_t m, int64_t n, int64_t nnz, const uint32_t *I, const uint32_t *J,
	const void *values, int type, int64_t *row_ptr, uint32_t *col_idx, void *out_values,
	void *stream) {
	ALPB_CHECK(m >= 0 && n >= 0 && nnz >= 0, ALPB_ILLEGAL, "alpb_coo_to_crs: negative size");
	ALPB_CHECK(m <= int64_t(UINT32_MAX) && n <= int64_t(UINT32_MAX), ALPB_OVERFLW,
		"alpb_coo_to_crs: dimensions exceed uint32 indices");
	cudaStream_t s = as_stream(stream);
	if (nnz > 0) {
		int *bad = nullptr;
		int hbad = 0;
		ALPB_CUDA(cudaMallocAsync(&bad, 4, s));
		ALPB_CUDA(cudaMemsetAsync(bad, 0, 4, s));
		k_check_coords<<<grid_for(nnz, 256), 256, 0, s>>>(I, J, nnz, m, n, bad);
		ALPB_LAUNCHED();
		ALPB_CUDA(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, s));
		ALPB_CUDA(cudaFreeAsync(bad, s));
		ALPB_CUDA(cudaStreamSynchronize(s));
		ALPB_CHECK(!hbad, ALPB_MISMATCH, "alpb_coo_to_crs: coordinate out of range");
	}
	return sorted_build(m, nnz, I, J, values, type, 1, row_ptr, col_idx, out_values, s);
}

int alpb_crs_transpose(int64_t m, int64_t n, int64_t nnz, const int64_t *row_ptr,
	const uint32_t *col_idx, const void *values, int type, int64_t *col_ptr, uint32_t *row_idx,
	void *t_values, void *stream) {
	ALPB_CHECK(m >= 0 && n >= 0 && nnz >= 0, ALPB_ILLEGAL, "alpb_crs_transpose: negative size");
	cudaStream_t s = as_stream(stream);
	if (nnz == 0) {
		ALPB_CUDA(cudaMemsetAsync(col_ptr, 0, size_t(n + 1) * 8, s));
		return ALPB_SUCCESS;
	}
	uint32_t *rows = nullptr;
	ALPB_CUDA(cudaMallocAsync(&rows, size_t(nnz) * 4, s));
	k_expand_rows<<<grid_for(m * 32, 256), 256, 0, s>>>(row_ptr, m, rows);
	ALPB_LAUNCHED();
	// keys = column index, payload = row; stable, so rows stay increasing
	int rc = sorted_build(n, nnz, col_idx, rows, values, type, 0, col_ptr, row_idx, t_values, s);
	ALPB_CUDA(cudaFreeAsync(rows, s));
	return rc;
}

int alpb_gen_stencil_crs(int dims, const int64_t *sizes, double diag, double off, int ref_order,
	int64_t *row_ptr, uint32_t *col_idx, double *values, int64_t *nnz, void *stream) {
	ALPB_CHECK(dims >= 1 && dims <= 4, ALPB_UNSUPPORTED, "alpb_gen_stencil_crs: dims %d", dims);
	ALPB_CHECK(sizes && row_ptr && nnz, ALPB_ILLEGAL, "alpb_gen_stencil_crs: null argument");
	Grid g;
	g.dims = dims;
	int64_t m = 1;
	for (int d = 0; d < dims; ++d) {
		ALPB_CHECK(sizes[d] >= 3, ALPB_ILLEGAL, "alpb_gen_stencil_crs: size < 2*halo+1");
		g.s[d] = sizes[d];
		m *= sizes[d];
	}
	ALPB_CHECK(m <= int64_t(UINT32_MAX), ALPB_OVERFLW, "alpb_gen_stencil_crs: too many rows");
	cudaStream_t s = as_stream(stream);
	if (col_idx == nullptr) {
		// counts -> exclusive scan into row_ptr
		int64_t *counts = nullptr;
		void *tmp = nullptr;
		size_t tb = 0;
		ALPB_CUDA(cudaMallocAsync(&counts, size_t(m + 1) * 8, s));
		ALPB_CUDA(cudaMemsetAsync(counts + m, 0, 8, s));
		k_stencil_counts<<<grid_for(m, 256), 256, 0, s>>>(g, m, counts);
		ALPB_LAUNCHED();
		ALPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, counts, row_ptr, m + 1, s));
		ALPB_CUDA(cudaMallocAsync(&tmp, tb, s));
		ALPB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, counts, row_ptr, m + 1, s));
		g_launches.fetch_add(1);
		ALPB_CUDA(cudaMemcpyAsync(nnz, row_ptr + m, 8, cudaMemcpyDeviceToHost, s));
		ALPB_CUDA(cudaFreeAsync(counts, s));
		ALPB_CUDA(cudaFreeAsync(tmp, s));
		ALPB_CUDA(cudaStreamSynchronize(s));
		return ALPB_SUCCESS;
	}
	k_stencil_fill<<<grid_for(m, 256), 256, 0, s>>>(g, m, row_ptr, diag, off, ref_order, col_idx,
		values);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_gen_poisson2d_batch(int64_t nseg, const int64_t *L, const double *shift,
	const int64_t *seg_rows, const int64_t *seg_nnz, int64_t total_rows, int64_t *row_ptr,
	uint32_t *col_idx, double *values, void *stream) {
	ALPB_CHECK(nseg > 0 && total_rows > 0, ALPB_ILLEGAL, "alpb_gen_poisson2d_batch: empty batch");
	ALPB_CHECK(total_rows <= int64_t(UINT32_MAX), ALPB_OVERFLW,
		"alpb_gen_poisson2d_batch: too many rows for uint32 indices");
	k_poisson2d_batch<<<grid_for(total_rows, 256), 256, 0, as_stream(stream)>>>(nseg, L, shift,
		seg_rows, seg_nnz, total_rows, row_ptr, col_idx, values);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_gen_sym_dd_values(const int64_t *row_ptr, const uint32_t *col_idx, int64_t m,
	uint64_t seed, double lo, double hi, double diag_factor, double *values, void *stream) {
	ALPB_CHECK(m >= 0 && hi >= lo, ALPB_ILLEGAL, "alpb_gen_sym_dd_values: bad arguments");
	if (m == 0) return ALPB_SUCCESS;
	k_sym_dd_values<<<grid_for(m * 32, 256), 256, 0, as_stream(stream)>>>(row_ptr, col_idx, m, seed,
		lo, hi, diag_factor, values);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_gen_normal(double *out, int64_t count, uint64_t seed, uint64_t sid, void *stream) {
	if (count <= 0) return ALPB_SUCCESS;
	k_gen_normal<<<grid_for(count, 256), 256, 0, as_stream(stream)>>>(out, count, seed, sid);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_gen_poisson2d_crs(int64_t L, double shift, int64_t *row_ptr, uint32_t *col_idx,
	double *values, void *stream) {
	ALPB_CHECK(L >= 2, ALPB_ILLEGAL, "alpb_gen_poisson2d_crs: L < 2");
	k_poisson2d<<<grid_for(L * L, 256), 256, 0, as_stream(stream)>>>(L, shift, row_ptr, col_idx,
		values);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

} // extern "C"
