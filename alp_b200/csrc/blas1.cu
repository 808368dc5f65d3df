// Level-1 primitives on dense FP64 vectors (and the sparse dot), replacing
// the reference's dot (reference/blas1.hpp:9262-9681), eWiseApply
// (:2966-5343), eWiseMul / eWiseMulAdd (:6347-6770, :8610-9172), foldl /
// foldr (:1069-2897) and set (reference/io.hpp).
//
// Reductions are deterministic: a fixed grid (a function of n and the SM
// count only) forms block partials in a fixed order, and one block sums them.
#include "common.cuh"
#include "persist.cuh"

namespace alpb {

__device__ __forceinline__ double apply_op(int op, double a, double b) {
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
	case ALPB_OP_EQUAL: return a == b ? 1.0 : 0.0;
	case ALPB_OP_NOT_EQUAL: return a != b ? 1.0 : 0.0;
	case ALPB_OP_LESS: return a < b ? 1.0 : 0.0;
	case ALPB_OP_LEQ: return a <= b ? 1.0 : 0.0;
	case ALPB_OP_GREATER: return a > b ? 1.0 : 0.0;
	case ALPB_OP_GEQ: return a >= b ? 1.0 : 0.0;
	}
	return 0.0;
}
__device__ __forceinline__ double op_identity(int op) {
	switch (op) {
	case ALPB_OP_ADD: return 0.0;
	case ALPB_OP_MUL: return 1.0;
	case ALPB_OP_MIN: return __longlong_as_double(0x7ff0000000000000ll);   // +inf
	case ALPB_OP_MAX: return __longlong_as_double((long long) 0xfff0000000000000ull);  // -inf
	case ALPB_OP_LOR: return 0.0;
	case ALPB_OP_LAND: return 1.0;
	}
	return 0.0;
}
static bool is_monoid(int op) {
	return op == ALPB_OP_ADD || op == ALPB_OP_MUL || op == ALPB_OP_MIN || op == ALPB_OP_MAX ||
		op == ALPB_OP_LOR || op == ALPB_OP_LAND;
}
static bool valid_op(int op) {
	return (op >= ALPB_OP_ADD && op <= ALPB_OP_LAND) ||
		(op >= ALPB_OP_EQUAL && op <= ALPB_OP_GEQ);
}

constexpr int RB = 256;  // reduction block

__device__ __forceinline__ double block_reduce_op(int op, double v, double *sm) {
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	for (int o = 16; o > 0; o >>= 1) v = apply_op(op, v, __shfl_down_sync(0xffffffffu, v, o));
	__syncthreads();
	if (lane == 0) sm[wid] = v;
	__syncthreads();
	if (wid == 0) {
		double w = lane < (RB / 32) ? sm[lane] : op_identity(op);
		for (int o = 16; o > 0; o >>= 1) w = apply_op(op, w, __shfl_down_sync(0xffffffffu, w, o));
		if (lane == 0) sm[32] = w;
	}
	__syncthreads();
	return sm[32];
}

// partials[b] = (+)_{i in block b's range} x_i (*) y_i over entries assigned in both
__global__ void __launch_bounds__(RB) k_dot_partial(int add_op, int mul_op, int64_t n,
	const double *__restrict__ x, const uint8_t *__restrict__ xa, const double *__restrict__ y,
	const uint8_t *__restrict__ ya, double *__restrict__ partials) {
	__shared__ double sm[33];
	double acc = op_identity(add_op);
	for (int64_t i = blockIdx.x * int64_t(RB) + threadIdx.x; i < n; i += int64_t(gridDim.x) * RB) {
		if ((xa && !xa[i]) || (ya && !ya[i])) continue;
		acc = apply_op(add_op, acc, apply_op(mul_op, x[i], y[i]));
	}
	acc = block_reduce_op(add_op, acc, sm);
	if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(RB) k_reduce_partials(int add_op, const double *__restrict__ p,
	int np, double *__restrict__ out, int accumulate) {
	__shared__ double sm[33];
	double acc = op_identity(add_op);
	for (int k = threadIdx.x; k < np; k += RB) acc = apply_op(add_op, acc, p[k]);
	acc = block_reduce_op(add_op, acc, sm);
	if (threadIdx.x == 0) *out = accumulate ? apply_op(add_op, *out, acc) : acc;
}

static int dot_grid(int64_t n) {
	int64_t g = (n + RB * 8 - 1) / (RB * 8);
	const int64_t cap = int64_t(sm_count()) * 4;
	if (g > cap) g = cap;
	return int(g < 1 ? 1 : g);
}

int dot_device(double *d_out, int add_op, int mul_op, int64_t n, const double *x,
	const uint8_t *xa, const double *y, const uint8_t *ya, int accumulate, cudaStream_t s) {
	const int g = dot_grid(n);
	double *partials = nullptr;
	ALPB_CUDA(cudaMallocAsync(&partials, size_t(g) * 8, s));
	k_dot_partial<<<g, RB, 0, s>>>(add_op, mul_op, n, x, xa, y, ya, partials);
	ALPB_LAUNCHED();
	k_reduce_partials<<<1, RB, 0, s>>>(add_op, partials, g, d_out, accumulate);
	ALPB_LAUNCHED();
	ALPB_CUDA(cudaFreeAsync(partials, s));
	return ALPB_SUCCESS;
}

__global__ void k_set_scalar(void *x, int type, int64_t n, double value, uint8_t *assigned) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x) {
		switch (type) {
		case ALPB_FP64: reinterpret_cast<double *>(x)[i] = value; break;
		case ALPB_INT32: reinterpret_cast<int32_t *>(x)[i] = int32_t(value); break;
		case ALPB_BOOL: reinterpret_cast<uint8_t *>(x)[i] = value != 0.0 ? 1 : 0; break;
		case ALPB_INT64: reinterpret_cast<int64_t *>(x)[i] = int64_t(value); break;
		case ALPB_UINT32: reinterpret_cast<uint32_t *>(x)[i] = uint32_t(value); break;
		case ALPB_UINT8: reinterpret_cast<uint8_t *>(x)[i] = uint8_t(int64_t(value)); break;
		case ALPB_INT8: reinterpret_cast<int8_t *>(x)[i] = int8_t(int64_t(value)); break;
		}
		if (assigned) assigned[i] = 1;
	}
}

__global__ void k_ewise_apply(double *__restrict__ out, int op, int64_t n,
	const double *__restrict__ a, double sa, const double *__restrict__ b, double sb) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x)
		out[i] = apply_op(op, a ? a[i] : sa, b ? b[i] : sb);
}

__global__ void k_ewise_muladd(double *__restrict__ out, int add_op, int mul_op, int64_t n,
	const double *__restrict__ a, double sa, const double *__restrict__ b, double sb) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x)
		out[i] = apply_op(add_op, out[i], apply_op(mul_op, a ? a[i] : sa, b ? b[i] : sb));
}

__global__ void k_foldl(double *__restrict__ x, int op, int64_t n, const double *__restrict__ y,
	double sy) {
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x)
		x[i] = apply_op(op, x[i], y ? y[i] : sy);
}

} // namespace alpb

using namespace alpb;

extern "C" {

int alpb_dot_f64(double *result, int add_op, int mul_op, int64_t n, const double *x,
	const uint8_t *x_assigned, const double *y, const uint8_t *y_assigned, void *stream) {
	ALPB_CHECK(result != nullptr, ALPB_ILLEGAL, "alpb_dot_f64: null result");
	ALPB_CHECK(is_monoid(add_op) && valid_op(mul_op), ALPB_UNSUPPORTED,
		"alpb_dot_f64: operators (%d, %d) are not a monoid and an operator", add_op, mul_op);
	ALPB_CHECK(n >= 0, ALPB_ILLEGAL, "alpb_dot_f64: negative size");
	if (n == 0) return ALPB_SUCCESS;
	cudaStream_t s = as_stream(stream);
	double *d = nullptr;
	ALPB_CUDA(cudaMallocAsync(&d, 8, s));
	int rc = dot_device(d, add_op, mul_op, n, x, x_assigned, y, y_assigned, 0, s);
	if (rc != ALPB_SUCCESS) return rc;
	double h = 0;
	ALPB_CUDA(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaFreeAsync(d, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	// z = z (+) dot: the reference folds the dot into the given scalar (blas1.hpp:9334-9336)
	double z = *result;
	switch (add_op) {
	case ALPB_OP_ADD: z = z + h; break;
	case ALPB_OP_MUL: z = z * h; break;
	case ALPB_OP_MIN: z = z < h ? z : h; break;
	case ALPB_OP_MAX: z = z > h ? z : h; break;
	case ALPB_OP_LOR: z = (z != 0 || h != 0) ? 1 : 0; break;
	case ALPB_OP_LAND: z = (z != 0 && h != 0) ? 1 : 0; break;
	}
	*result = z;
	return ALPB_SUCCESS;
}

int alpb_dot_f64_device(double *d_result, int add_op, int mul_op, int64_t n, const double *x,
	const double *y, void *stream) {
	ALPB_CHECK(d_result != nullptr, ALPB_ILLEGAL, "alpb_dot_f64_device: null result");
	ALPB_CHECK(is_monoid(add_op) && valid_op(mul_op), ALPB_UNSUPPORTED,
		"alpb_dot_f64_device: operators (%d, %d)", add_op, mul_op);
	ALPB_CHECK(n >= 0, ALPB_ILLEGAL, "alpb_dot_f64_device: negative size");
	return dot_device(d_result, add_op, mul_op, n, x, nullptr, y, nullptr, 0, as_stream(stream));
}

int alpb_set_scalar(void *x, int type, int64_t n, double value, uint8_t *assigned, int64_t *nnz,
	void *stream) {
	ALPB_CHECK(type_size(type) > 0, ALPB_UNSUPPORTED, "alpb_set_scalar: type %d", type);
	ALPB_CHECK(n >= 0, ALPB_ILLEGAL, "alpb_set_scalar: negative size");
	if (n == 0) return ALPB_SUCCESS;
	cudaStream_t s = as_stream(stream);
	k_set_scalar<<<grid_for(n, 256), 256, 0, s>>>(x, type, n, value, assigned);
	ALPB_LAUNCHED();
	if (nnz) ALPB_CUDA(cudaMemcpyAsync(nnz, &n, 8, cudaMemcpyHostToDevice, s));
	if (nnz) ALPB_CUDA(cudaStreamSynchronize(s));  // n lives on this stack frame
	return ALPB_SUCCESS;
}

int alpb_ewise_apply_f64(double *out, int op, int64_t n, const double *a, double sa,
	const double *b, double sb, void *stream) {
	ALPB_CHECK(valid_op(op), ALPB_UNSUPPORTED, "alpb_ewise_apply_f64: op %d", op);
	if (n <= 0) return n == 0 ? ALPB_SUCCESS : ALPB_ILLEGAL;
	k_ewise_apply<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(out, op, n, a, sa, b, sb);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_ewise_muladd_f64(double *out, int add_op, int mul_op, int64_t n, const double *a,
	double sa, const double *b, double sb, void *stream) {
	ALPB_CHECK(valid_op(add_op) && valid_op(mul_op), ALPB_UNSUPPORTED,
		"alpb_ewise_muladd_f64: ops %d %d", add_op, mul_op);
	if (n <= 0) return n == 0 ? ALPB_SUCCESS : ALPB_ILLEGAL;
	k_ewise_muladd<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(out, add_op, mul_op, n, a, sa,
		b, sb);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_foldl_f64(double *x, int op, int64_t n, const double *y, double sy, void *stream) {
	ALPB_CHECK(valid_op(op), ALPB_UNSUPPORTED, "alpb_foldl_f64: op %d", op);
	if (n <= 0) return n == 0 ? ALPB_SUCCESS : ALPB_ILLEGAL;
	k_foldl<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(x, op, n, y, sy);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

int alpb_reduce_f64(double *result, int op, int64_t n, const double *x, const uint8_t *assigned,
	void *stream) {
	ALPB_CHECK(result != nullptr, ALPB_ILLEGAL, "alpb_reduce_f64: null result");
	ALPB_CHECK(is_monoid(op), ALPB_UNSUPPORTED, "alpb_reduce_f64: op %d is not a monoid", op);
	if (n == 0) return ALPB_SUCCESS;
	// fold(x) = dot(x, 1) under (op, left_assign)
	cudaStream_t s = as_stream(stream);
	double *d = nullptr;
	ALPB_CUDA(cudaMallocAsync(&d, 8, s));
	int rc = dot_device(d, op, ALPB_OP_LEFT_ASSIGN, n, x, assigned, x, nullptr, 0, s);
	if (rc != ALPB_SUCCESS) return rc;
	double h = 0;
	ALPB_CUDA(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaFreeAsync(d, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	double z = *result;
	switch (op) {
	case ALPB_OP_ADD: z = z + h; break;
	case ALPB_OP_MUL: z = z * h; break;
	case ALPB_OP_MIN: z = z < h ? z : h; break;
	case ALPB_OP_MAX: z = z > h ? z : h; break;
	case ALPB_OP_LOR: z = (z != 0 || h != 0) ? 1 : 0; break;
	case ALPB_OP_LAND: z = (z != 0 && h != 0) ? 1 : 0; break;
	}
	*result = z;
	return ALPB_SUCCESS;
}

} // extern "C"
