// Shared device/host helpers of the B200 backend: status plumbing, the
// counter-based hash used by all generators, and the semiring functors that
// the SpMV kernels are instantiated on.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <climits>
#include <cstdio>
#include <string>
#include <atomic>

#include "../../include/alp_b200.h"

namespace alpb {

// ---------------------------------------------------------------- status --
void set_error(const char *fmt, ...);
extern std::atomic<int64_t> g_launches;

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Check a CUDA runtime call; on failure record the message and return PANIC
// (a CUDA error leaves device state undefined, which is grb::PANIC).
#define ALPB_CUDA(call)                                                        \
	do {                                                                       \
		cudaError_t _e = (call);                                               \
		if (_e != cudaSuccess) {                                               \
			::alpb::set_error("%s:%d: %s -> %s", __FILE__, __LINE__, #call,    \
				cudaGetErrorString(_e));                                       \
			return ALPB_PANIC;                                                 \
		}                                                                      \
	} while (0)

// After a kernel launch: count it and check the launch configuration.
#define ALPB_LAUNCHED()                                                        \
	do {                                                                       \
		::alpb::g_launches.fetch_add(1, std::memory_order_relaxed);            \
		cudaError_t _e = cudaGetLastError();                                   \
		if (_e != cudaSuccess) {                                               \
			::alpb::set_error("%s:%d: kernel launch -> %s", __FILE__, __LINE__, \
				cudaGetErrorString(_e));                                       \
			return ALPB_PANIC;                                                 \
		}                                                                      \
	} while (0)

#define ALPB_CHECK(cond, code, ...)                                            \
	do {                                                                       \
		if (!(cond)) {                                                         \
			::alpb::set_error(__VA_ARGS__);                                    \
			return (code);                                                     \
		}                                                                      \
	} while (0)

// number of SMs of the current device (cached per device)
int sm_count();

inline unsigned grid_for(int64_t work, int block, int max_blocks_per_sm = 8) {
	int64_t g = (work + block - 1) / block;
	int64_t cap = int64_t(sm_count()) * max_blocks_per_sm;
	if (g > cap) g = cap;
	if (g < 1) g = 1;
	return unsigned(g);
}

// ------------------------------------------------------------------ hash --
// splitmix64 finaliser (Steele, Lea, Flood: "Fast splittable pseudorandom
// number generators", OOPSLA 2014); composed into a 3-input counter hash.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
	z += 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t hash3(uint64_t seed, uint64_t a, uint64_t b) {
	return mix64(mix64(seed ^ mix64(a)) + b * 0xD1B54A32D192ED03ull);
}
// U[0,1) with 53 random bits
__host__ __device__ __forceinline__ double u01(uint64_t h) {
	return double(h >> 11) * (1.0 / 9007199254740992.0);
}

// -------------------------------------------------------------- semirings --
// Each ring: T (domain of vectors and of the matrix values), add (the
// additive monoid's operator), mulr(a, x) = op(A_value, x_value) for the
// right-handed mxv, mull(x, a) = op(x_value, A_value) for the left-handed vxm
// (reference/blas2.hpp:124-160), zero() (additive identity), one() (value of
// a pattern nonzero: the ring's One identity), and immutable
// (grb::has_immutable_nonzeroes, monoid.hpp:139: once an output holds a
// non-identity value, further additions cannot change it).
struct RingPlusTimesF64 {
	using T = double;
	static constexpr bool immutable = false;
	static __device__ __forceinline__ T zero() { return 0.0; }
	static __device__ __forceinline__ T one() { return 1.0; }
	static __device__ __forceinline__ T add(T a, T b) { return a + b; }
	static __device__ __forceinline__ T mulr(T a, T x) { return a * x; }
	static __device__ __forceinline__ T mull(T x, T a) { return x * a; }
};
struct RingLorLandBool {
	using T = uint8_t;
	static constexpr bool immutable = true;
	static __device__ __forceinline__ T zero() { return 0; }
	static __device__ __forceinline__ T one() { return 1; }
	static __device__ __forceinline__ T add(T a, T b) { return (a | b) ? 1 : 0; }
	static __device__ __forceinline__ T mulr(T a, T x) { return (a && x) ? 1 : 0; }
	static __device__ __forceinline__ T mull(T x, T a) { return (x && a) ? 1 : 0; }
};
struct RingMinPlusI32 {
	using T = int32_t;
	static constexpr bool immutable = false;
	static __device__ __forceinline__ T zero() { return INT_MAX; }
	static __device__ __forceinline__ T one() { return 0; }
	static __device__ __forceinline__ T add(T a, T b) { return a < b ? a : b; }
	// two's-complement wrap: what operators::add<int> compiles to
	static __device__ __forceinline__ T mulr(T a, T x) { return int32_t(uint32_t(a) + uint32_t(x)); }
	static __device__ __forceinline__ T mull(T x, T a) { return int32_t(uint32_t(x) + uint32_t(a)); }
};
// out-degree ring of simple_pagerank: left_assign_if(p, q) = bool(q) ? p : 0
// (base/internalops.hpp:485-520), with the additive identity as the "else"
struct RingPlusPatternF64 {
	using T = double;
	static constexpr bool immutable = false;
	static __device__ __forceinline__ T zero() { return 0.0; }
	static __device__ __forceinline__ T one() { return 1.0; }
	static __device__ __forceinline__ T add(T a, T b) { return a + b; }
	static __device__ __forceinline__ T mulr(T a, T x) { return x != 0.0 ? a : 0.0; }
	static __device__ __forceinline__ T mull(T x, T a) { return a != 0.0 ? x : 0.0; }
};
struct RingPlusTimesI32 {
	using T = int32_t;
	static constexpr bool immutable = false;
	static __device__ __forceinline__ T zero() { return 0; }
	static __device__ __forceinline__ T one() { return 1; }
	static __device__ __forceinline__ T add(T a, T b) { return int32_t(uint32_t(a) + uint32_t(b)); }
	static __device__ __forceinline__ T mulr(T a, T x) { return int32_t(uint32_t(a) * uint32_t(x)); }
	static __device__ __forceinline__ T mull(T x, T a) { return int32_t(uint32_t(x) * uint32_t(a)); }
};
// degree ring of interfaces/pregel.hpp:381-386: right_assign_if(p, q) = bool(p) ? q
// : (nothing) over size_t (base/internalops.hpp:580-660), additive identity as the
// "else"; unsigned 64-bit arithmetic on ALPB_INT64 storage
struct RingPlusRightIfU64 {
	using T = uint64_t;
	static constexpr bool immutable = false;
	static __device__ __forceinline__ T zero() { return 0; }
	static __device__ __forceinline__ T one() { return 1; }
	static __device__ __forceinline__ T add(T a, T b) { return a + b; }
	static __device__ __forceinline__ T mulr(T a, T x) { return a != 0 ? x : 0; }
	static __device__ __forceinline__ T mull(T x, T a) { return x != 0 ? a : 0; }
};
// Pregel message ring under max (connected components): max over size_t with
// identity numeric_limits<size_t>::min() = 0, multiplied by left_assign_if
struct RingMaxLeftIfU64 {
	using T = uint64_t;
	static constexpr bool immutable = false;
	static __device__ __forceinline__ T zero() { return 0; }
	static __device__ __forceinline__ T one() { return 1; }
	static __device__ __forceinline__ T add(T a, T b) { return a > b ? a : b; }
	static __device__ __forceinline__ T mulr(T a, T x) { return x != 0 ? a : 0; }
	static __device__ __forceinline__ T mull(T x, T a) { return a != 0 ? x : 0; }
};
// multiplication as the additive monoid (identity 1), addition as the product
// (identity 0)
struct RingTimesPlusF64 {
	using T = double;
	static constexpr bool immutable = false;
	static __device__ __forceinline__ T zero() { return 1.0; }
	static __device__ __forceinline__ T one() { return 0.0; }
	static __device__ __forceinline__ T add(T a, T b) { return a * b; }
	static __device__ __forceinline__ T mulr(T a, T x) { return a + x; }
	static __device__ __forceinline__ T mull(T x, T a) { return x + a; }
};

// mask evaluation of utils::interpretMask (utils.hpp:318-341)
__device__ __forceinline__ bool mask_value_true(const void *vals, int type, int64_t i) {
	switch (type) {
	case ALPB_VOID: return true;
	case ALPB_BOOL: return reinterpret_cast<const uint8_t *>(vals)[i] != 0;
	case ALPB_INT32: return reinterpret_cast<const int32_t *>(vals)[i] != 0;
	case ALPB_FP64: return reinterpret_cast<const double *>(vals)[i] != 0.0;
	case ALPB_UINT32: return reinterpret_cast<const uint32_t *>(vals)[i] != 0;
	case ALPB_UINT8: return reinterpret_cast<const uint8_t *>(vals)[i] != 0;
	case ALPB_INT8: return reinterpret_cast<const int8_t *>(vals)[i] != 0;
	case ALPB_INT64: return reinterpret_cast<const int64_t *>(vals)[i] != 0;
	}
	return false;
}
__device__ __forceinline__ bool eval_mask(const void *vals, const uint8_t *assigned,
	int type, uint32_t descr, int64_t i) {
	const bool a = assigned ? assigned[i] != 0 : true;
	bool r;
	if ((descr & ALPB_DESC_STRUCTURAL) || vals == nullptr || type == ALPB_VOID)
		r = a;
	else
		r = a && mask_value_true(vals, type, i);
	return (descr & ALPB_DESC_INVERT_MASK) ? !r : r;
}

size_t type_size(int type);

} // namespace alpb
