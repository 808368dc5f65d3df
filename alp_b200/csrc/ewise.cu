// Generic element-wise vector primitive with ALP's sparse semantics: the
// device side of grb::set, grb::foldl / grb::foldr (vector forms),
// grb::eWiseApply and grb::eWiseMul / eWiseMulAdd of the C++ backend
// (reference/blas1.hpp, reference/io.hpp).
//
// Every operand is (values, assigned flags) with flags == nullptr meaning
// dense, or a scalar.  Values are read into the operator's domain -- double,
// int64_t or uint64_t, chosen by the caller from the ALP operator's type --
// computed there and cast to the output type, as the reference's operators
// cast their operands (graphblas/ops.hpp): integer operators compute exactly,
// with two's-complement wrap-around.
#include "common.cuh"

#include <cstring>
#include <type_traits>

namespace alpb {

// ------------------------------------------------------------ domains --
// An ALP operator computes in its own domain: double, or an integer type of
// 32 or 64 bits (int, size_t, ... operators).  Integer domains compute with
// two's-complement wrap-around at their own width, so an int operator's
// overflowing sum wraps before a later min or comparison sees it, exactly as
// the reference's int arithmetic does.
template <class T>
__device__ __forceinline__ T ld_as(const void *p, int type, int64_t i) {
	switch (type) {
	case ALPB_FP64: return T(reinterpret_cast<const double *>(p)[i]);
	case ALPB_INT32: return T(int64_t(reinterpret_cast<const int32_t *>(p)[i]));
	case ALPB_BOOL: return reinterpret_cast<const uint8_t *>(p)[i] ? T(1) : T(0);
	case ALPB_INT64: return T(reinterpret_cast<const int64_t *>(p)[i]);
	case ALPB_UINT32: return T(reinterpret_cast<const uint32_t *>(p)[i]);
	case ALPB_UINT8: return T(reinterpret_cast<const uint8_t *>(p)[i]);
	case ALPB_INT8: return T(int64_t(reinterpret_cast<const int8_t *>(p)[i]));
	case ALPB_UINT64: return T(reinterpret_cast<const uint64_t *>(p)[i]);
	}
	return T(0);
}
template <>
__device__ __forceinline__ uint64_t ld_as<uint64_t>(const void *p, int type, int64_t i) {
	switch (type) {
	case ALPB_FP64: return uint64_t(reinterpret_cast<const double *>(p)[i]);
	case ALPB_INT64:
	case ALPB_UINT64: return reinterpret_cast<const uint64_t *>(p)[i];   // size_t storage
	default: return uint64_t(ld_as<int64_t>(p, type, i));
	}
}

template <class T>
__device__ __forceinline__ void st_as(void *p, int type, int64_t i, T v) {
	switch (type) {
	case ALPB_FP64: reinterpret_cast<double *>(p)[i] = double(v); break;
	case ALPB_INT32: reinterpret_cast<int32_t *>(p)[i] = int32_t(uint32_t(uint64_t(int64_t(v)))); break;
	case ALPB_BOOL: reinterpret_cast<uint8_t *>(p)[i] = v != T(0) ? 1 : 0; break;
	case ALPB_INT64: reinterpret_cast<int64_t *>(p)[i] = int64_t(v); break;
	case ALPB_UINT32: reinterpret_cast<uint32_t *>(p)[i] = uint32_t(uint64_t(int64_t(v))); break;
	case ALPB_UINT8: reinterpret_cast<uint8_t *>(p)[i] = uint8_t(uint64_t(int64_t(v))); break;
	case ALPB_INT8: reinterpret_cast<int8_t *>(p)[i] = int8_t(uint8_t(uint64_t(int64_t(v)))); break;
	case ALPB_UINT64: reinterpret_cast<uint64_t *>(p)[i] = uint64_t(int64_t(v)); break;
	}
}
template <>
__device__ __forceinline__ void st_as<uint64_t>(void *p, int type, int64_t i, uint64_t v) {
	switch (type) {
	case ALPB_FP64: reinterpret_cast<double *>(p)[i] = double(v); break;
	case ALPB_INT64:
	case ALPB_UINT64: reinterpret_cast<uint64_t *>(p)[i] = v; break;
	default: st_as<int64_t>(p, type, i, int64_t(v)); break;
	}
}

// 32-bit integer domains: loaded through the 64-bit ones, narrowed with
// wrap-around (a double converts directly, as C++ converts it)
template <>
__device__ __forceinline__ int32_t ld_as<int32_t>(const void *p, int type, int64_t i) {
	if (type == ALPB_FP64) return int32_t(reinterpret_cast<const double *>(p)[i]);
	return int32_t(uint32_t(uint64_t(ld_as<int64_t>(p, type, i))));
}
template <>
__device__ __forceinline__ uint32_t ld_as<uint32_t>(const void *p, int type, int64_t i) {
	if (type == ALPB_FP64) return uint32_t(reinterpret_cast<const double *>(p)[i]);
	return uint32_t(ld_as<uint64_t>(p, type, i));
}
template <>
__device__ __forceinline__ void st_as<int32_t>(void *p, int type, int64_t i, int32_t v) {
	if (type == ALPB_FP64) reinterpret_cast<double *>(p)[i] = double(v);
	else st_as<int64_t>(p, type, i, int64_t(v));   // sign-extends into 64-bit outputs
}
template <>
__device__ __forceinline__ void st_as<uint32_t>(void *p, int type, int64_t i, uint32_t v) {
	if (type == ALPB_FP64) reinterpret_cast<double *>(p)[i] = double(v);
	else st_as<int64_t>(p, type, i, int64_t(v));   // zero-extends into 64-bit outputs
}

// wrapping + - * for the integer domains (no signed-overflow UB)
template <class T> __device__ __forceinline__ T wrap_add(T a, T b) { return a + b; }
template <class T> __device__ __forceinline__ T wrap_sub(T a, T b) { return a - b; }
template <class T> __device__ __forceinline__ T wrap_mul(T a, T b) { return a * b; }
template <> __device__ __forceinline__ int64_t wrap_add(int64_t a, int64_t b) {
	return int64_t(uint64_t(a) + uint64_t(b));
}
template <> __device__ __forceinline__ int64_t wrap_sub(int64_t a, int64_t b) {
	return int64_t(uint64_t(a) - uint64_t(b));
}
template <> __device__ __forceinline__ int64_t wrap_mul(int64_t a, int64_t b) {
	return int64_t(uint64_t(a) * uint64_t(b));
}
template <> __device__ __forceinline__ int32_t wrap_add(int32_t a, int32_t b) {
	return int32_t(uint32_t(a) + uint32_t(b));
}
template <> __device__ __forceinline__ int32_t wrap_sub(int32_t a, int32_t b) {
	return int32_t(uint32_t(a) - uint32_t(b));
}
template <> __device__ __forceinline__ int32_t wrap_mul(int32_t a, int32_t b) {
	return int32_t(uint32_t(a) * uint32_t(b));
}

template <class T>
__device__ __forceinline__ T opv(int op, T a, T b) {
	switch (op) {
	case ALPB_OP_ADD: return wrap_add(a, b);
	case ALPB_OP_SUB: return wrap_sub(a, b);
	case ALPB_OP_MUL: return wrap_mul(a, b);
	case ALPB_OP_DIV:
		if constexpr (std::is_floating_point<T>::value) return a / b;
		else return b == T(0) ? T(0) : a / b;   // the host's division by zero is undefined
	case ALPB_OP_MIN: return a < b ? a : b;
	case ALPB_OP_MAX: return a > b ? a : b;
	case ALPB_OP_ABS_DIFF: return a > b ? wrap_sub(a, b) : wrap_sub(b, a);
	case ALPB_OP_LEFT_ASSIGN: return a;
	case ALPB_OP_RIGHT_ASSIGN: return b;
	case ALPB_OP_LOR: return (a != T(0) || b != T(0)) ? T(1) : T(0);
	case ALPB_OP_LAND: return (a != T(0) && b != T(0)) ? T(1) : T(0);
	case ALPB_OP_LEFT_ASSIGN_IF: return a;  // callers test opv_skips first
	case ALPB_OP_EQUAL: return a == b ? T(1) : T(0);
	case ALPB_OP_NOT_EQUAL: return a != b ? T(1) : T(0);
	case ALPB_OP_LESS: return a < b ? T(1) : T(0);
	case ALPB_OP_LEQ: return a <= b ? T(1) : T(0);
	case ALPB_OP_GREATER: return a > b ? T(1) : T(0);
	case ALPB_OP_GEQ: return a >= b ? T(1) : T(0);
	}
	return T(0);
}
// True where op leaves its output unchanged (left_assign_if with b false).
template <class T>
__device__ __forceinline__ bool opv_skips(int op, T b) {
	return op == ALPB_OP_LEFT_ASSIGN_IF && b == T(0);
}

template <class T>
struct VecArgs {
	int kind, op, monoid;
	T identity;
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
	T alpha;
	const void *y;
	int yt;
	const uint8_t *ya;
	T beta;
	int mul_op;
};

template <class T>
__global__ void k_vec(VecArgs<T> a) {
	int64_t newly = 0;
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < a.n;
		 i += int64_t(gridDim.x) * blockDim.x) {
		if (a.masked && !eval_mask(a.m, a.ma, a.mt, a.descr, i)) continue;
		const bool zh = a.za == nullptr || a.za[i] != 0;
		const bool xh = a.x == nullptr || a.xa == nullptr || a.xa[i] != 0;
		const bool yh = a.y == nullptr || a.ya == nullptr || a.ya[i] != 0;
		const T xv = a.x ? (xh ? ld_as<T>(a.x, a.xt, i) : T(0)) : a.alpha;
		const T yv = a.y ? (yh ? ld_as<T>(a.y, a.yt, i) : T(0)) : a.beta;
		bool write = false, assign = false;
		T out = T(0);
		switch (a.kind) {
		case ALPB_VEC_SET:  // z_i = x_i (or i under use_index) where x is present
			if (xh) {
				out = (a.descr & ALPB_DESC_USE_INDEX) ? T(i) : xv;
				write = true;
				assign = true;
			}
			break;
		case ALPB_VEC_FOLDL:  // z_i = z_i op x_i
		case ALPB_VEC_FOLDR:  // z_i = x_i op z_i
			if (!xh) break;
			if (zh) {
				const T zv = ld_as<T>(a.z, a.zt, i);
				if (opv_skips(a.op, a.kind == ALPB_VEC_FOLDL ? xv : zv)) break;
				out = a.kind == ALPB_VEC_FOLDL ? opv(a.op, zv, xv) : opv(a.op, xv, zv);
				write = true;
			} else if (a.monoid) {
				// monoid fold into an absent entry: identity op x_i (a scalar x
				// reaches every absent entry, reference/blas1.hpp:957-981)
				out = a.kind == ALPB_VEC_FOLDL ? opv(a.op, a.identity, xv) : opv(a.op, xv, a.identity);
				write = true;
				assign = true;
			}
			break;
		case ALPB_VEC_APPLY:  // z_i = x_i op y_i: operator = intersection, monoid = union
			if (xh && yh) {
				if (opv_skips(a.op, yv)) break;
				out = opv(a.op, xv, yv);
				write = true;
				assign = true;
			}
			else if (a.monoid && (xh || yh)) {
				out = xh ? opv(a.op, xv, a.identity) : opv(a.op, a.identity, yv);
				write = true;
				assign = true;
			}
			break;
		case ALPB_VEC_MULADD: {  // z_i = z_i (+) (x_i (*) y_i) over the ring
			if (!(xh && yh) || opv_skips(a.mul_op, yv)) break;
			const T prod = opv(a.mul_op, xv, yv);
			if (zh) out = opv(a.op, ld_as<T>(a.z, a.zt, i), prod);
			else { out = prod; assign = true; }
			write = true;
			break;
		}
		}
		if (write) st_as<T>(a.z, a.zt, i, out);
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

template <class T>
__device__ __forceinline__ T shfl_down_t(T v, int o) { return __shfl_down_sync(0xffffffffu, v, o); }

// Typed reduction: partial[b] = (+)_i x_i (*) y_i over i where x, y (and the
// mask) are present; y == nullptr means "no second operand" (plain fold).
template <class T>
__global__ void k_vec_dot(int add_op, T ident, int mul_op, int64_t n, const void *x, int xt,
	const uint8_t *xa, const void *y, int yt, const uint8_t *ya, const void *m,
	const uint8_t *ma, int mt, int masked, uint32_t descr, T *partials) {
	__shared__ T sm[32];
	T acc = ident;
	bool any = false;
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
		 i += int64_t(gridDim.x) * blockDim.x) {
		if (xa && !xa[i]) continue;
		if (y && ya && !ya[i]) continue;
		if (masked && !eval_mask(m, ma, mt, descr, i)) continue;
		const T xv = ld_as<T>(x, xt, i);
		const T yv = y ? ld_as<T>(y, yt, i) : T(0);
		if (y && opv_skips(mul_op, yv)) continue;
		const T t = y ? opv(mul_op, xv, yv) : xv;
		acc = any ? opv(add_op, acc, t) : opv(add_op, ident, t);
		any = true;
	}
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	for (int o = 16; o > 0; o >>= 1) acc = opv(add_op, acc, shfl_down_t(acc, o));
	if (lane == 0) sm[wid] = acc;
	__syncthreads();
	if (wid == 0) {
		T w = lane < int(blockDim.x >> 5) ? sm[lane] : ident;
		for (int o = 16; o > 0; o >>= 1) w = opv(add_op, w, shfl_down_t(w, o));
		if (lane == 0) partials[blockIdx.x] = w;
	}
}

// *result = *result (+) partial[0] (+) ... (+) partial[g-1], in block order,
// by one thread (the reference folds into the given scalar).
template <class T>
__global__ void k_vec_dot_finish(int add_op, const T *partials, int g, T *result) {
	if (blockIdx.x != 0 || threadIdx.x != 0) return;
	T acc = *result;
	for (int b = 0; b < g; ++b) acc = opv(add_op, acc, partials[b]);
	*result = acc;
}

template <class T>
static T from_bits(uint64_t bits) {
	T v;
	memcpy(&v, &bits, sizeof(T));
	return v;
}

template <class T>
static int vec_reduce_run(void *result, int add_op, uint64_t identity, int mul_op,
	uint32_t descr, int64_t n, const void *x, int x_type, const uint8_t *x_assigned,
	const void *y, int y_type, const uint8_t *y_assigned, const void *mask,
	const uint8_t *mask_assigned, int mask_type, int masked, cudaStream_t s) {
	int64_t g64 = (n + 256 * 8 - 1) / (256 * 8);
	if (g64 > int64_t(sm_count()) * 4) g64 = int64_t(sm_count()) * 4;
	const int g = int(g64 < 1 ? 1 : g64);
	T *part = nullptr;
	ALPB_CUDA(cudaMallocAsync(&part, size_t(g + 1) * sizeof(T), s));
	k_vec_dot<T><<<g, 256, 0, s>>>(add_op, from_bits<T>(identity), mul_op, n, x, x_type,
		x_assigned, y, y_type, y_assigned, mask, mask_assigned,
		mask == nullptr ? ALPB_VOID : mask_type, masked, descr, part);
	ALPB_LAUNCHED();
	ALPB_CUDA(cudaMemcpyAsync(part + g, result, sizeof(T), cudaMemcpyHostToDevice, s));
	k_vec_dot_finish<T><<<1, 32, 0, s>>>(add_op, part, g, part + g);
	ALPB_LAUNCHED();
	ALPB_CUDA(cudaMemcpyAsync(result, part + g, sizeof(T), cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaFreeAsync(part, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	return ALPB_SUCCESS;
}

template <class T>
static int vec_op_run(int kind, int op, int monoid, uint64_t identity, int mul_op,
	uint32_t descr, int64_t n, void *z, int z_type, uint8_t *z_assigned, int64_t *z_nnz,
	const void *mask, const uint8_t *mask_assigned, int mask_type, int masked,
	const void *x, int x_type, const uint8_t *x_assigned, uint64_t alpha,
	const void *y, int y_type, const uint8_t *y_assigned, uint64_t beta, cudaStream_t s) {
	if (kind == ALPB_VEC_APPLY && z_assigned) {
		k_vec_clear_flags<<<grid_for(n, 256), 256, 0, s>>>(z_assigned, n);
		ALPB_LAUNCHED();
		ALPB_CUDA(cudaMemsetAsync(z_nnz, 0, 8, s));
	}
	VecArgs<T> a;
	a.kind = kind;
	a.op = op;
	a.monoid = monoid;
	a.identity = from_bits<T>(identity);
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
	a.alpha = from_bits<T>(alpha);
	a.y = y;
	a.yt = y_type;
	a.ya = y_assigned;
	a.beta = from_bits<T>(beta);
	a.mul_op = mul_op;
	k_vec<T><<<grid_for(n, 256), 256, 0, s>>>(a);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

// ------------------------------------------------------ fused chains --
// Steps of alpb_vec_chain, with the domain's values decoded; slot values live
// in a per-thread array for the element being processed.
template <class T>
struct ChainStep {
	int32_t kind, op, mul_op, use_index, z, x, y;
	T alpha, beta;
};
template <class T>
struct ChainArgs {
	int64_t n;
	int nslots, nsteps;
	uint32_t load, store;          // slots read before written / written
	void *val[ALPB_CHAIN_SLOTS];
	int type[ALPB_CHAIN_SLOTS];
	ChainStep<T> step[ALPB_CHAIN_STEPS];
	int reduce;                    // the last step is a reduction
	int radd, rmul, rx, ry;
	T rident;
};

template <class T>
__global__ void __launch_bounds__(256) k_vec_chain(ChainArgs<T> c, T *partials) {
	__shared__ T sm[32];
	T acc = c.rident;
	bool any = false;
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < c.n;
		 i += int64_t(gridDim.x) * blockDim.x) {
		T v[ALPB_CHAIN_SLOTS];
#pragma unroll
		for (int q = 0; q < ALPB_CHAIN_SLOTS; ++q)
			if (q < c.nslots && ((c.load >> q) & 1)) v[q] = ld_as<T>(c.val[q], c.type[q], i);
		for (int k = 0; k < c.nsteps; ++k) {
			const ChainStep<T> &o = c.step[k];
			const T xv = o.x >= 0 ? v[o.x] : o.alpha;
			const T yv = o.y >= 0 ? v[o.y] : o.beta;
			switch (o.kind) {
			case ALPB_VEC_SET: v[o.z] = o.use_index ? T(i) : xv; break;
			case ALPB_VEC_FOLDL: v[o.z] = opv(o.op, v[o.z], xv); break;
			case ALPB_VEC_FOLDR: v[o.z] = opv(o.op, xv, v[o.z]); break;
			default: v[o.z] = opv(o.op, v[o.z], opv(o.mul_op, xv, yv)); break;  // MULADD
			}
		}
		if (c.reduce) {   // as k_vec_dot on dense operands
			const T t = c.ry >= 0 ? opv(c.rmul, v[c.rx], v[c.ry]) : v[c.rx];
			acc = any ? opv(c.radd, acc, t) : opv(c.radd, c.rident, t);
			any = true;
		}
#pragma unroll
		for (int q = 0; q < ALPB_CHAIN_SLOTS; ++q)
			if (q < c.nslots && ((c.store >> q) & 1)) st_as<T>(c.val[q], c.type[q], i, v[q]);
	}
	if (!c.reduce) return;
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	for (int o = 16; o > 0; o >>= 1) acc = opv(c.radd, acc, shfl_down_t(acc, o));
	if (lane == 0) sm[wid] = acc;
	__syncthreads();
	if (wid == 0) {
		T w = lane < int(blockDim.x >> 5) ? sm[lane] : c.rident;
		for (int o = 16; o > 0; o >>= 1) w = opv(c.radd, w, shfl_down_t(w, o));
		if (lane == 0) partials[blockIdx.x] = w;
	}
}

static bool domain_type(int domain, int type) {
	return type == domain || (domain == ALPB_UINT64 && type == ALPB_INT64) ||
		(domain == ALPB_INT64 && type == ALPB_UINT64);
}

template <class T>
static int vec_chain_run(int domain, int64_t n, int nslots, void *const *values,
	const int *types, int nsteps, const alpb_vec_step *steps, void *result, cudaStream_t s) {
	ChainArgs<T> c{};
	c.n = n;
	c.nslots = nslots;
	uint32_t written = 0;
	for (int q = 0; q < nslots; ++q) {
		ALPB_CHECK(values[q] != nullptr, ALPB_ILLEGAL, "alpb_vec_chain: null vector in slot %d", q);
		ALPB_CHECK(domain_type(domain, types[q]), ALPB_UNSUPPORTED,
			"alpb_vec_chain: slot %d has type %d, not the domain's", q, types[q]);
		c.val[q] = values[q];
		c.type[q] = types[q];
	}
	const auto slot_ok = [&](int q, bool scalar_ok) { return (scalar_ok && q == -1) || (q >= 0 && q < nslots); };
	const auto read = [&](int q) { if (q >= 0 && !((written >> q) & 1)) c.load |= 1u << q; };
	for (int k = 0; k < nsteps; ++k) {
		const alpb_vec_step &o = steps[k];
		const bool last = k + 1 == nsteps;
		if (o.kind == ALPB_VEC_REDUCE) {
			ALPB_CHECK(last && result != nullptr, ALPB_ILLEGAL,
				"alpb_vec_chain: a reduction must be the last step, with a result");
			ALPB_CHECK(slot_ok(o.x, false) && (o.y == -1 || slot_ok(o.y, false)), ALPB_ILLEGAL,
				"alpb_vec_chain: reduction operands");
			ALPB_CHECK(o.op >= ALPB_OP_ADD && o.op <= ALPB_OP_LAND && o.mul_op >= ALPB_OP_ADD &&
				o.mul_op <= ALPB_OP_GEQ && o.mul_op != ALPB_OP_LEFT_ASSIGN_IF, ALPB_UNSUPPORTED,
				"alpb_vec_chain: reduction ops %d %d", o.op, o.mul_op);
			read(o.x);
			read(o.y);
			c.reduce = 1;
			c.radd = o.op;
			c.rmul = o.mul_op;
			c.rx = o.x;
			c.ry = o.y;
			c.rident = from_bits<T>(o.identity);
			continue;
		}
		ALPB_CHECK(o.kind >= ALPB_VEC_SET && o.kind <= ALPB_VEC_MULADD && o.kind != ALPB_VEC_APPLY,
			ALPB_ILLEGAL, "alpb_vec_chain: step kind %d", o.kind);
		ALPB_CHECK(o.op >= ALPB_OP_ADD && o.op <= ALPB_OP_GEQ && o.op != ALPB_OP_LEFT_ASSIGN_IF &&
			(o.kind != ALPB_VEC_MULADD || (o.mul_op >= ALPB_OP_ADD && o.mul_op <= ALPB_OP_GEQ &&
			o.mul_op != ALPB_OP_LEFT_ASSIGN_IF)), ALPB_UNSUPPORTED, "alpb_vec_chain: step ops");
		ALPB_CHECK(slot_ok(o.z, false) && slot_ok(o.x, true) &&
			(o.kind != ALPB_VEC_MULADD || slot_ok(o.y, true)), ALPB_ILLEGAL,
			"alpb_vec_chain: step %d slots", k);
		read(o.x);
		if (o.kind == ALPB_VEC_MULADD) read(o.y);
		if (o.kind != ALPB_VEC_SET) read(o.z);
		written |= 1u << o.z;
		ChainStep<T> &d = c.step[c.nsteps++];
		d.kind = o.kind;
		d.op = o.op;
		d.mul_op = o.mul_op;
		d.use_index = o.kind == ALPB_VEC_SET && (o.descr & ALPB_DESC_USE_INDEX) ? 1 : 0;
		d.z = o.z;
		d.x = o.x;
		d.y = o.kind == ALPB_VEC_MULADD ? o.y : -1;
		d.alpha = from_bits<T>(o.alpha);
		d.beta = from_bits<T>(o.beta);
	}
	c.store = written;
	if (!c.reduce) {
		k_vec_chain<T><<<grid_for(n, 256), 256, 0, s>>>(c, nullptr);
		ALPB_LAUNCHED();
		return ALPB_SUCCESS;
	}
	// the reduction's grid and order are those of alpb_vec_reduce_dom
	int64_t g64 = (n + 256 * 8 - 1) / (256 * 8);
	if (g64 > int64_t(sm_count()) * 4) g64 = int64_t(sm_count()) * 4;
	const int g = int(g64 < 1 ? 1 : g64);
	T *part = nullptr;
	ALPB_CUDA(cudaMallocAsync(&part, size_t(g + 1) * sizeof(T), s));
	k_vec_chain<T><<<g, 256, 0, s>>>(c, part);
	ALPB_LAUNCHED();
	ALPB_CUDA(cudaMemcpyAsync(part + g, result, sizeof(T), cudaMemcpyHostToDevice, s));
	k_vec_dot_finish<T><<<1, 32, 0, s>>>(c.radd, part, g, part + g);
	ALPB_LAUNCHED();
	ALPB_CUDA(cudaMemcpyAsync(result, part + g, sizeof(T), cudaMemcpyDeviceToHost, s));
	ALPB_CUDA(cudaFreeAsync(part, s));
	ALPB_CUDA(cudaStreamSynchronize(s));
	return ALPB_SUCCESS;
}

static uint64_t bits_of(double v) {
	uint64_t b;
	memcpy(&b, &v, 8);
	return b;
}

} // namespace alpb

using namespace alpb;

extern "C" {

int alpb_vec_reduce_dom(void *result, int add_op, uint64_t identity, int mul_op,
	uint32_t descr, int domain, int64_t n, const void *x, int x_type, const uint8_t *x_assigned,
	const void *y, int y_type, const uint8_t *y_assigned, const void *mask,
	const uint8_t *mask_assigned, int mask_type, int masked, void *stream) {
	ALPB_CHECK(result != nullptr, ALPB_ILLEGAL, "alpb_vec_reduce: null result");
	ALPB_CHECK(add_op >= ALPB_OP_ADD && add_op <= ALPB_OP_LAND && mul_op >= ALPB_OP_ADD &&
		mul_op <= ALPB_OP_GEQ, ALPB_UNSUPPORTED, "alpb_vec_reduce: ops %d %d", add_op,
		mul_op);
	ALPB_CHECK(domain == ALPB_FP64 || domain == ALPB_INT64 || domain == ALPB_UINT64 ||
		domain == ALPB_INT32 || domain == ALPB_UINT32, ALPB_UNSUPPORTED,
		"alpb_vec_reduce: domain %d", domain);
	if (n <= 0) return n == 0 ? ALPB_SUCCESS : ALPB_ILLEGAL;
	cudaStream_t s = as_stream(stream);
	switch (domain) {
	case ALPB_FP64:
		return vec_reduce_run<double>(result, add_op, identity, mul_op, descr, n, x, x_type,
			x_assigned, y, y_type, y_assigned, mask, mask_assigned, mask_type, masked, s);
	case ALPB_INT64:
		return vec_reduce_run<int64_t>(result, add_op, identity, mul_op, descr, n, x, x_type,
			x_assigned, y, y_type, y_assigned, mask, mask_assigned, mask_type, masked, s);
	case ALPB_INT32:
		return vec_reduce_run<int32_t>(result, add_op, identity, mul_op, descr, n, x, x_type,
			x_assigned, y, y_type, y_assigned, mask, mask_assigned, mask_type, masked, s);
	case ALPB_UINT32:
		return vec_reduce_run<uint32_t>(result, add_op, identity, mul_op, descr, n, x, x_type,
			x_assigned, y, y_type, y_assigned, mask, mask_assigned, mask_type, masked, s);
	default:
		return vec_reduce_run<uint64_t>(result, add_op, identity, mul_op, descr, n, x, x_type,
			x_assigned, y, y_type, y_assigned, mask, mask_assigned, mask_type, masked, s);
	}
}

int alpb_vec_reduce(double *result, int add_op, double identity, int mul_op, uint32_t descr,
	int64_t n, const void *x, int x_type, const uint8_t *x_assigned, const void *y, int y_type,
	const uint8_t *y_assigned, const void *mask, const uint8_t *mask_assigned, int mask_type,
	int masked, void *stream) {
	return alpb_vec_reduce_dom(result, add_op, bits_of(identity), mul_op, descr, ALPB_FP64, n, x,
		x_type, x_assigned, y, y_type, y_assigned, mask, mask_assigned, mask_type, masked, stream);
}

int alpb_vec_op_dom(int kind, int op, int monoid, uint64_t identity, int mul_op, uint32_t descr,
	int domain, int64_t n, void *z, int z_type, uint8_t *z_assigned, int64_t *z_nnz,
	const void *mask, const uint8_t *mask_assigned, int mask_type, int masked,
	const void *x, int x_type, const uint8_t *x_assigned, uint64_t alpha,
	const void *y, int y_type, const uint8_t *y_assigned, uint64_t beta, void *stream) {
	ALPB_CHECK(kind >= ALPB_VEC_SET && kind <= ALPB_VEC_MULADD, ALPB_ILLEGAL,
		"alpb_vec_op: kind %d", kind);
	ALPB_CHECK(op >= ALPB_OP_ADD && op <= ALPB_OP_GEQ, ALPB_UNSUPPORTED,
		"alpb_vec_op: op %d", op);
	ALPB_CHECK(type_size(z_type) > 0, ALPB_UNSUPPORTED, "alpb_vec_op: output type %d", z_type);
	ALPB_CHECK(z_assigned == nullptr || z_nnz != nullptr, ALPB_ILLEGAL,
		"alpb_vec_op: sparse output needs its nnz counter");
	ALPB_CHECK(domain == ALPB_FP64 || domain == ALPB_INT64 || domain == ALPB_UINT64 ||
		domain == ALPB_INT32 || domain == ALPB_UINT32, ALPB_UNSUPPORTED,
		"alpb_vec_op: domain %d", domain);
	if (n <= 0) return n == 0 ? ALPB_SUCCESS : ALPB_ILLEGAL;
	cudaStream_t s = as_stream(stream);
	switch (domain) {
	case ALPB_INT32:
		return vec_op_run<int32_t>(kind, op, monoid, identity, mul_op, descr, n, z, z_type,
			z_assigned, z_nnz, mask, mask_assigned, mask_type, masked, x, x_type, x_assigned, alpha,
			y, y_type, y_assigned, beta, s);
	case ALPB_UINT32:
		return vec_op_run<uint32_t>(kind, op, monoid, identity, mul_op, descr, n, z, z_type,
			z_assigned, z_nnz, mask, mask_assigned, mask_type, masked, x, x_type, x_assigned, alpha,
			y, y_type, y_assigned, beta, s);
	case ALPB_FP64:
		return vec_op_run<double>(kind, op, monoid, identity, mul_op, descr, n, z, z_type,
			z_assigned, z_nnz, mask, mask_assigned, mask_type, masked, x, x_type, x_assigned, alpha,
			y, y_type, y_assigned, beta, s);
	case ALPB_INT64:
		return vec_op_run<int64_t>(kind, op, monoid, identity, mul_op, descr, n, z, z_type,
			z_assigned, z_nnz, mask, mask_assigned, mask_type, masked, x, x_type, x_assigned, alpha,
			y, y_type, y_assigned, beta, s);
	default:
		return vec_op_run<uint64_t>(kind, op, monoid, identity, mul_op, descr, n, z, z_type,
			z_assigned, z_nnz, mask, mask_assigned, mask_type, masked, x, x_type, x_assigned, alpha,
			y, y_type, y_assigned, beta, s);
	}
}

int alpb_vec_op(int kind, int op, int monoid, double identity, int mul_op, uint32_t descr,
	int64_t n, void *z, int z_type, uint8_t *z_assigned, int64_t *z_nnz,
	const void *mask, const uint8_t *mask_assigned, int mask_type, int masked,
	const void *x, int x_type, const uint8_t *x_assigned, double alpha,
	const void *y, int y_type, const uint8_t *y_assigned, double beta, void *stream) {
	return alpb_vec_op_dom(kind, op, monoid, bits_of(identity), mul_op, descr, ALPB_FP64, n, z,
		z_type, z_assigned, z_nnz, mask, mask_assigned, mask_type, masked, x, x_type, x_assigned,
		bits_of(alpha), y, y_type, y_assigned, bits_of(beta), stream);
}

int alpb_vec_chain(int domain, int64_t n, int nslots, void *const *values, const int *types,
	int nsteps, const alpb_vec_step *steps, void *result, void *stream) {
	ALPB_CHECK(nslots >= 0 && nslots <= ALPB_CHAIN_SLOTS && nsteps >= 0 &&
		nsteps <= ALPB_CHAIN_STEPS, ALPB_ILLEGAL, "alpb_vec_chain: %d slots, %d steps (at most %d, %d)",
		nslots, nsteps, ALPB_CHAIN_SLOTS, ALPB_CHAIN_STEPS);
	ALPB_CHECK(nsteps == 0 || (values != nullptr && types != nullptr && steps != nullptr),
		ALPB_ILLEGAL, "alpb_vec_chain: null arrays");
	ALPB_CHECK(domain == ALPB_FP64 || domain == ALPB_INT64 || domain == ALPB_UINT64 ||
		domain == ALPB_INT32 || domain == ALPB_UINT32, ALPB_UNSUPPORTED,
		"alpb_vec_chain: domain %d", domain);
	if (n < 0) return ALPB_ILLEGAL;
	if (n == 0 || nsteps == 0) return ALPB_SUCCESS;
	cudaStream_t s = as_stream(stream);
	switch (domain) {
	case ALPB_FP64: return vec_chain_run<double>(domain, n, nslots, values, types, nsteps, steps, result, s);
	case ALPB_INT64: return vec_chain_run<int64_t>(domain, n, nslots, values, types, nsteps, steps, result, s);
	case ALPB_INT32: return vec_chain_run<int32_t>(domain, n, nslots, values, types, nsteps, steps, result, s);
	case ALPB_UINT32: return vec_chain_run<uint32_t>(domain, n, nslots, values, types, nsteps, steps, result, s);
	default: return vec_chain_run<uint64_t>(domain, n, nslots, values, types, nsteps, steps, result, s);
	}
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
