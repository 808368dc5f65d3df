// Generic element-wise vector primitive with ALP's sparse semantics: the
// device side of grb::set, grb::foldl / grb::foldr (vector forms),
// grb::eWiseApply and grb::eWiseMul / eWiseMulAdd of the C++ backend
// (reference/blas1.hpp, reference/io.hpp).
//
// Every operand is (values, assigned flags) with flags == nullptr meaning
// dense, or a scalar.  Values are read into double and the result is cast
// back to the output type (the ALP operator domains seen by the kernels are
// double, int32, int64 and bool; integers up to 2^53 round-trip exactly).
#include "common.cuh"

#include <vector>

namespace alpb {

__device__ __forceinline__ double ld_val(const void *p, int type, int64_t i) {
	switch (type) {
	case ALPB_FP64: return reinterpret_cast<const double *>(p)[i];
	case ALPB_INT32: return double(reinterpret_cast<const int32_t *>(p)[i]);
	case ALPB_BOOL: return reinterpret_cast<const uint8_t *>(p)[i] ? 1.0 : 0.0;
	case ALPB_INT64: return double(reinterpret_cast<const int64_t *>(p)[i]);
	case ALPB_UINT32: return double(reinterpret_cast<const uint32_t *>(p)[i]);
	case ALPB_UINT8: return double(reinterpret_cast<const uint8_t *>(p)[i]);
	case ALPB_INT8: return double(reinterpret_cast<const int8_t *>(p)[i]);
	}
	return 0.0;
}
__device__ __forceinline__ void st_val(void *p, int type, int64_t i, double v) {
	switch (type) {
	case ALPB_FP64: reinterpret_cast<double *>(p)[i] = v; break;
	case ALPB_INT32: reinterpret_cast<int32_t *>(p)[i] = int32_t(int64_t(v)); break;
	case ALPB_BOOL: reinterpret_cast<uint8_t *>(p)[i] = v != 0.0 ? 1 : 0; break;
	case ALPB_INT64: reinterpret_cast<int64_t *>(p)[i] = int64_t(v); break;
	case ALPB_UINT32: reinterpret_cast<uint32_t *>(p)[i] = uint32_t(int64_t(v)); break;
	case ALPB_UINT8: reinterpret_cast<uint8_t *>(p)[i] = uint8_t(int64_t(v)); break;
	case ALPB_INT8: reinterpret_cast<int8_t *>(p)[i] = int8_t(int64_t(v)); break;
	}
}
__device__ __forceinline__ double opd(int op, double a, double b) {
	switch (op) {
	case ALPB_OP_ADD: return a + b;
	case ALPB_OP_SUB: return a - b;
	case ALPB_OP_MUL: return a * b;
	case ALPB_OP_DIV: return a / b;
	case ALPB_OP_MIN: return a < b ? a : b;
	case ALPB_OP_MAX: return a > b ? a : b;
	case ALPB_OP_ABS_DIFF: return a > b ? a - b : b - a;
	case ALPB_OP_LEFT_ASSIGN: return a;
	case ALPB_OP_RIGHT_ASSIGN: return b;
	case ALPB_OP_LOR: return (a != 0.0 || b != 0.0) ? 1.0 : 0.0;
	case ALPB_OP_LAND: return (a != 0.0 && b != 0.0) ? 1.0 : 0.0;
	case ALPB_OP_LEFT_ASSIGN_IF: return a;  // callers test opd_skips first
	case ALPB_OP_EQUAL: return a == b ? 1.0 : 0.0;
	case ALPB_OP_NOT_EQUAL: return a != b ? 1.0 : 0.0;
	case ALPB_OP_LESS: return a < b ? 1.0 : 0.0;
	case ALPB_OP_LEQ: return a <= b ? 1.0 : 0.0;
	case ALPB_OP_GREATER: return a > b ? 1.0 : 0.0;
	case ALPB_OP_GEQ: return a >= b ? 1.0 : 0.0;
	}
	return 0.0;
}
// True where op leaves its output unchanged (left_assign_if with b false).
__device__ __forceinline__ bool opd_skips(int op, double b) {
	return op == ALPB_OP_LEFT_ASSIGN_IF && b == 0.0;
}

struct VecArgs {
	int kind, op, monoid;
	double identity;
	uint32_t descr;
	int64_t n;
	void *z;
	int zt;
	uint8_t *za;
	int64_t *znnz;
	const void *m;
	const uint8_t *ma;
	int mt;
	int masked;
	const void *x;
	int xt;
	const uint8_t *xa;
	double alpha;
	const void *y;
	int yt;
	const uint8_t *ya;
	double beta;
	int mul_op;
};

__global__ void k_vec(VecArgs a) {
	int64_t newly = 0;
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < a.n;
		 i += int64_t(gridDim.x) * blockDim.x) {
		if (a.masked && !eval_mask(a.m, a.ma, a.mt, a.descr, i)) continue;
		const bool zh = a.za == nullptr || a.za[i] != 0;
		const bool xh = a.x == nullptr || a.xa == nullptr || a.xa[i] != 0;
		const bool yh = a.y == nullptr || a.ya == nullptr || a.ya[i] != 0;
		const double xv = a.x ? (xh ? ld_val(a.x, a.xt, i) : 0.0) : a.alpha;
		const double yv = a.y ? (yh ? ld_val(a.y, a.yt, i) : 0.0) : a.beta;
		bool write = false, assign = false;
		double out = 0.0;
		switch (a.kind) {
		case ALPB_VEC_SET:  // z_i = x_i (or i under use_index) where x is present
			if (xh) {
				out = (a.descr & ALPB_DESC_USE_INDEX) ? double(i) : xv;
				write = true;
				assign = true;
			}
			break;
		case ALPB_VEC_FOLDL:  // z_i = z_i op x_i
		case ALPB_VEC_FOLDR:  // z_i = x_i op z_i
			if (!xh) break;
			if (zh) {
				const double zv = ld_val(a.z, a.zt, i);
				if (opd_skips(a.op, a.kind == ALPB_VEC_FOLDL ? xv : zv)) break;
				out = a.kind == ALPB_VEC_FOLDL ? opd(a.op, zv, xv) : opd(a.op, xv, zv);
				write = true;
			} else if (a.monoid) {
				// monoid fold into an absent entry: identity op x_i (a scalar x
				// reaches every absent entry, reference/blas1.hpp:957-981)
				out = a.kind == ALPB_VEC_FOLDL ? opd(a.op, a.identity, xv) : opd(a.op, xv, a.identity);
				write = true;
				assign = true;
			}
			break;
		case ALPB_VEC_APPLY:  // z_i = x_i op y_i: operator = intersection, monoid = union
			if (xh && yh) {
				if (opd_skips(a.op, yv)) break;
				out = opd(a.op, xv, yv);
				write = true;
				assign = true;
			}
			else if (a.monoid && (xh || yh)) {
				out = xh ? opd(a.op, xv, a.identity) : opd(a.op, a.identity, yv);
				write = true;
				assign = true;
			}
			break;
		case ALPB_VEC_MULADD: {  // z_i = z_i (+) (x_i (*) y_i) over the ring
			if (!(xh && yh) || opd_skips(a.mul_op, yv)) break;
			const double prod = opd(a.mul_op, xv, yv);
			if (zh) out = opd(a.op, ld_val(a.z, a.zt, i), prod);
			else { out = prod; assign = true; }
			write = true;
			break;
		}
		}
		if (write) st_val(a.z, a.zt, i, out);
		if (assign && a.za && !a.za[i]) {
			a.za[i] = 1;
			++newly;
		}
	}
	if (a.znnz) {
		for (int o = 16; o > 0; o >>= 1) newly += __shfl_down_sync(0xffffffffu, newly, o);
		if ((threadIdx.x & 31) == 0 && newly)
			atomicAdd((unsigned long long *) a.znnz, (unsigned long long) newly);
	}
}

// eWiseApply replaces the output: entries that end up without a value are
// removed first (z := empty, then assigned where the result exists)
__global__ void k_vec_clear_flags(uint8_t *za, int64_t n) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x)
		za[i] = 0;
}

__global__ void k_count_assigned(const uint8_t *a, int64_t n, int64_t *cnt) {
	int64_t c = 0;
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x)
		c += a[i] ? 1 : 0;
	for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
	if ((threadIdx.x & 31) == 0 && c) atomicAdd((unsigned long long *) cnt, (unsigned long long) c);
}

// Typed reduction: partial[b] = (+)_i x_i (*) y_i over i where x, y (and the
// mask) are present; y == nullptr means "no second operand" (plain fold).
__global__ void k_vec_dot(int add_op, double ident, int mul_op, int64_t n, const void *x, int xt,
	const uint8_t *xa, const void *y, int yt, const uint8_t *ya, const void *m,
	const uint8_t *ma, int mt, int masked, uint32_t descr, double *partials) {
	__shared__ double sm[32];
	double acc = ident;
	bool any = false;
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x) {
		if (xa && !xa[i]) continue;
		if (y && ya && !ya[i]) continue;
		if (masked && !eval_mask(m, ma, mt, descr, i)) continue;
		const double xv = ld_val(x, xt, i);
		const double yv = y ? ld_val(y, yt, i) : 0.0;
		if (y && opd_skips(mul_op, yv)) continue;
		const double t = y ? opd(mul_op, xv, yv) : xv;
		acc = any ? opd(add_op, acc, t) : opd(add_op, ident, t);
		any = true;
	}
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	for (int o = 16; o > 0; o >>= 1) acc = opd(add_op, acc, __shfl_down_sync(0xffffffffu, acc, o));
	if (lane == 0) sm[wid] = acc;
	__syncthreads();
	if (wid == 0) {
		double w = lane < int(blockDim.x >> 5) ? sm[lane] : ident;
		for (int o = 16; o > 0; o >>= 1) w = opd(add_op, w, __shfl_down_sync(0xffffffffu, w, o));
		if (lane == 0) partials[blockIdx.x] = w;
	}
}

} // namespace alpb

using namespace alpb;

extern "C" {

int alpb_vec_reduce(double *result, int add_op, double identity, int mul_op, uint32_t descr,
	int64_t n, const void *x, int x_type, const uint8_t *x_assigned, const void *y, int y_type,
	const uint8_t *y_assigned, const void *mask, const uint8_t *mask_assigned, int mask_type,
	int masked, void *stream) {
	ALPB_CHECK(result != nullptr, ALPB_ILLEGAL, "alpb_vec_reduce: null result");
	ALPB_CHECK(add_op >= ALPB_OP_ADD && add_op <= ALPB_OP_LAND && mul_op >= ALPB_OP_ADD &&
		mul_op <= ALPB_OP_GEQ, ALPB_UNSUPPORTED, "alpb_vec_reduce: ops %d %d", add_op,
		mul_op);
	if (n <= 0) return n == 0 ? ALPB_SUCCESS : ALPB_ILLEGAL;
	cudaStream_t s = as_stream(stream);
	int64_t g64 = (n + 256 * 8 - 1) / (256 * 8);
	if (g64 > int64_t(sm_count()) * 4) g64 = int64_t(sm_count()) * 4;
	const int g = int(g64 < 1 ? 1 : g64);
	double *part = nullptr;
	ALPB_CUDA(cudaMallocAsync(&part, size_t(g) * 8, s));
	k_vec_dot<<<g, 256, 0, s>>>(add_op, identity, mul_op, n, x, x_type, x_assigned, y, y_type,
		y_assigned, mask, mask_assigned, mask == nullptr ? ALPB_VOID : mask_type, masked, descr, part);
	ALPB_LAUNCHED();
	std::vector<double> h(static_cast<size_t>(g));
	ALPB_CUDA(cudaMemcpyAsync(h.data(), part, size_t(g) * 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaFreeAsync(part, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	double acc = *result;  // the reference folds into the given scalar
	for (int b = 0; b < g; ++b) {
		const double v = h[size_t(b)];
		switch (add_op) {
		case ALPB_OP_ADD: acc = acc + v; break;
		case ALPB_OP_MUL: acc = acc * v; break;
		case ALPB_OP_MIN: acc = acc < v ? acc : v; break;
		case ALPB_OP_MAX: acc = acc > v ? acc : v; break;
		case ALPB_OP_LOR: acc = (acc != 0 || v != 0) ? 1 : 0; break;
		case ALPB_OP_LAND: acc = (acc != 0 && v != 0) ? 1 : 0; break;
		default: acc = v; break;
		}
	}
	*result = acc;
	return ALPB_SUCCESS;
}

int alpb_vec_op(int kind, int op, int monoid, double identity, int mul_op, uint32_t descr,
	int64_t n, void *z, int z_type, uint8_t *z_assigned, int64_t *z_nnz,
	const void *mask, const uint8_t *mask_assigned, int mask_type, int masked,
	const void *x, int x_type, const uint8_t *x_assigned, double alpha,
	const void *y, int y_type, const uint8_t *y_assigned, double beta, void *stream) {
	ALPB_CHECK(kind >= ALPB_VEC_SET && kind <= ALPB_VEC_MULADD, ALPB_ILLEGAL,
		"alpb_vec_op: kind %d", kind);
	ALPB_CHECK(op >= ALPB_OP_ADD && op <= ALPB_OP_GEQ, ALPB_UNSUPPORTED,
		"alpb_vec_op: op %d", op);
	ALPB_CHECK(type_size(z_type) > 0, ALPB_UNSUPPORTED, "alpb_vec_op: output type %d", z_type);
	ALPB_CHECK(z_assigned == nullptr || z_nnz != nullptr, ALPB_ILLEGAL,
		"alpb_vec_op: sparse output needs its nnz counter");
	if (n <= 0) return n == 0 ? ALPB_SUCCESS : ALPB_ILLEGAL;
	cudaStream_t s = as_stream(stream);
	if (kind == ALPB_VEC_APPLY && z_assigned) {
		k_vec_clear_flags<<<grid_for(n, 256), 256, 0, s>>>(z_assigned, n);
		ALPB_LAUNCHED();
		ALPB_CUDA(cudaMemsetAsync(z_nnz, 0, 8, s));
	}
	VecArgs a;
	a.kind = kind;
	a.op = op;
	a.monoid = monoid;
	a.identity = identity;
	a.descr = descr;
	a.n = n;
	a.z = z;
	a.zt = z_type;
	a.za = z_assigned;
	a.znnz = z_nnz;
	a.m = mask;
	a.ma = mask_assigned;
	a.mt = mask == nullptr ? ALPB_VOID : mask_type;
	a.masked = masked;
	a.x = x;
	a.xt = x_type;
	a.xa = x_assigned;
	a.alpha = alpha;
	a.y = y;
	a.yt = y_type;
	a.ya = y_assigned;
	a.beta = beta;
	a.mul_op = mul_op;
	k_vec<<<grid_for(n, 256), 256, 0, s>>>(a);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_count_assigned(const uint8_t *assigned, int64_t n, int64_t *count, void *stream) {
	ALPB_CHECK(count != nullptr, ALPB_ILLEGAL, "alpb_count_assigned: null count");
	*count = 0;
	if (n <= 0) return ALPB_SUCCESS;
	cudaStream_t s = as_stream(stream);
	int64_t *d = nullptr;
	ALPB_CUDA(cudaMallocAsync(&d, 8, s));
	ALPB_CUDA(cudaMemsetAsync(d, 0, 8, s));
	k_count_assigned<<<grid_for(n, 256), 256, 0, s>>>(assigned, n, d);
	ALPB_LAUNCHED();
	ALPB_CUDA(cudaMemcpyAsync(count, d, 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaFreeAsync(d, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	return ALPB_SUCCESS;
}

} // extern "C"
