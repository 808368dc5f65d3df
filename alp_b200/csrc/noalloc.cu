// Allocation-free SpMV entry point.
//
// Some callers cannot allocate device memory while they call us: code running
// inside a memory pool that owns every byte of the device, an allocator or
// stream callback, a process that must not grow its footprint after start-up,
// or a host thread that may not call cudaMalloc (which synchronises the
// device) in the middle of a stream of work.  alpb_mxv_dense_noalloc serves
// them: it is the dense merge-path product of alpb_mxv, but the merge-path
// tables it needs as scratch live in one fixed array in this file, which
// every device that loads the library holds until the process exits.  The
// caller passes only the inputs and the output.
#include "common.cuh"
#include "merge.cuh"
#include "spmv.cuh"

#include <cuda.h>

#include <mutex>

namespace alpb {

// Scratch of the allocation-free entry point.  Every call shares these bytes.
constexpr size_t kNoallocBytes = size_t(7) << 20;               // 7 MiB
constexpr int64_t kNoallocTiles = 131072;                       // tiles of MP_TILE items
constexpr int64_t kNoallocMaxItems = kNoallocTiles * MP_TILE;   // rows + nonzeroes

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// Byte offsets of the merge tables inside the scratch array (50 B per tile + 8).
struct NoallocLayout {
	static constexpr size_t tile_row = 0;                                     // int64[T+1]
	static constexpr size_t head_first = tile_row + 8 * (kNoallocTiles + 1);  // int64[T]
	static constexpr size_t tail_first = head_first + 8 * kNoallocTiles;      // int64[T]
	static constexpr size_t head_val = tail_first + 8 * kNoallocTiles;        // u64[T]
	static constexpr size_t tail_val = head_val + 8 * kNoallocTiles;          // u64[T]
	static constexpr size_t span_len = tail_val + 8 * kNoallocTiles;          // int32[T]
	static constexpr size_t counter = span_len + 4 * kNoallocTiles;           // int32[T]
	static constexpr size_t head_has = counter + 4 * kNoallocTiles;           // u8[T]
	static constexpr size_t tail_has = head_has + kNoallocTiles;              // u8[T]
	static constexpr size_t end = tail_has + kNoallocTiles;
};
static_assert(NoallocLayout::end <= kNoallocBytes, "scratch layout exceeds the array");

// Device address of g_noalloc_scratch, resolved once per device and context
// with that device current.  In host code the array's name only stands in for
// the symbol -- it is not a device address -- so kernels always get this
// pointer.  The cache is keyed on the current context's process-unique id
// (cuCtxGetId), not only on the device index: after cudaDeviceReset the
// runtime makes a new context, the library's module loads again, possibly at
// another address, and the first call in the new context resolves it anew.
constexpr int kNoallocMaxDevices = 64;
struct NoallocSlot {
	unsigned long long ctx_id;
	unsigned char *ptr;
};
static std::mutex g_noalloc_mutex;
static NoallocSlot g_noalloc_slot[kNoallocMaxDevices] = {};

// Id of the calling thread's current context; 0 when there is none yet (or
// the driver lacks cuCtxGetId).  The two driver calls are looked up through
// the runtime, so the library does not link the driver library itself.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);
static unsigned long long noalloc_context_id() {
	static CtxGetCurrentFn get_current = nullptr;
	static CtxGetIdFn get_id = nullptr;
	static bool looked_up = false;
	if (!looked_up) {   // under g_noalloc_mutex
		void *f = nullptr, *g = nullptr;
		cudaDriverEntryPointQueryResult q1, q2;
		if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q1) == cudaSuccess &&
			q1 == cudaDriverEntryPointSuccess &&
			cudaGetDriverEntryPoint("cuCtxGetId", &g, cudaEnableDefault, &q2) == cudaSuccess &&
			q2 == cudaDriverEntryPointSuccess) {
			get_current = reinterpret_cast<CtxGetCurrentFn>(f);
			get_id = reinterpret_cast<CtxGetIdFn>(g);
		}
		(void) cudaGetLastError();
		looked_up = true;
	}
	if (!get_current || !get_id) return 0;
	CUcontext ctx = nullptr;
	unsigned long long id = 0;
	if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
	if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
	return id;
}

static int noalloc_scratch(unsigned char **out) {
	int dev = 0;
	ALPB_CUDA(cudaGetDevice(&dev));
	ALPB_CHECK(dev >= 0 && dev < kNoallocMaxDevices, ALPB_PANIC,
		"alpb_mxv_dense_noalloc: device %d is beyond the %d devices it serves", dev,
		kNoallocMaxDevices);
	std::lock_guard<std::mutex> lock(g_noalloc_mutex);
	NoallocSlot &slot = g_noalloc_slot[dev];
	unsigned long long id = noalloc_context_id();
	if (id == 0 || slot.ptr == nullptr || slot.ctx_id != id) {
		void *p = nullptr;
		// also makes the device's primary context current if nothing had yet
		const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess || p == nullptr) {
			set_error("alpb_mxv_dense_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
				cudaGetErrorString(e));
			return ALPB_PANIC;
		}
		slot.ptr = static_cast<unsigned char *>(p);
		slot.ctx_id = noalloc_context_id();   // 0 keeps the next call resolving again
	}
	*out = slot.ptr;
	return ALPB_SUCCESS;
}

// The array keeps the previous call's contents: the arrival counters of the
// spanning rows must start at zero.
__global__ void k_noalloc_clear(int32_t *counter, int64_t ntiles) {
	for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < ntiles;
		 t += int64_t(gridDim.x) * blockDim.x)
		counter[t] = 0;
}

template <class R>
struct NoallocAccumulate {
	typename R::T *__restrict__ y;
	__device__ __forceinline__ void row(int64_t r, typename R::T v, bool has) {
		if (has) y[r] = R::add(y[r], v);
	}
	__device__ __forceinline__ void row_span(int64_t, int64_t r, typename R::T v, bool has) {
		row(r, v, has);
	}
};

template <class R>
__global__ void __launch_bounds__(MP_BLOCK)
k_spmv_merge_noalloc(MergeTables mt, const int64_t *__restrict__ offsets,
	const uint32_t *__restrict__ indices, const typename R::T *__restrict__ values,
	const typename R::T *__restrict__ x, typename R::T *__restrict__ y, int left) {
	__shared__ MergeSmem<R> sm;
	PlainX<typename R::T> xl{x};
	NoallocAccumulate<R> epi{y};
	for (int64_t t = blockIdx.x; t < mt.ntiles; t += gridDim.x)
		merge_tile<R>(t, mt, offsets, indices, values, xl, epi, left, sm);
}

template <class R>
int noalloc_run(const MergeTables &mt, const int64_t *offsets, const uint32_t *indices,
	const void *values, const void *v, void *u, int left, cudaStream_t s) {
	using T = typename R::T;
	k_spmv_merge_noalloc<R><<<unsigned(mt.ntiles), MP_BLOCK, 0, s>>>(mt, offsets, indices,
		reinterpret_cast<const T *>(values), reinterpret_cast<const T *>(v),
		reinterpret_cast<T *>(u), left);
	ALPB_LAUNCHED();
	return ALPB_SUCCESS;
}

} // namespace alpb

using namespace alpb;

extern "C" int alpb_mxv_dense_noalloc(int ring, int form, int64_t m_out, int64_t n_in,
	int64_t nnz, const int64_t *offsets, const uint32_t *indices, const void *values,
	int value_type, void *u, const void *v, void *stream) {
	ALPB_CHECK(ring_value_type(ring) >= 0, ALPB_UNSUPPORTED,
		"alpb_mxv_dense_noalloc: semiring %d is not instantiated on the device", ring);
	ALPB_CHECK(value_type == ALPB_VOID || value_type == ring_value_type(ring), ALPB_UNSUPPORTED,
		"alpb_mxv_dense_noalloc: matrix value type %d does not match semiring %d", value_type, ring);
	ALPB_CHECK(m_out >= 0 && n_in >= 0 && nnz >= 0, ALPB_ILLEGAL,
		"alpb_mxv_dense_noalloc: negative size");
	ALPB_CHECK(m_out + nnz <= kNoallocMaxItems, ALPB_ILLEGAL,
		"alpb_mxv_dense_noalloc: rows + nonzeroes = %lld exceeds the fixed scratch limit of %lld "
		"(use alpb_mxv with a plan)", (long long) (m_out + nnz), (long long) kNoallocMaxItems);
	{
		// u holds m_out elements and v holds n_in: any shared byte is an overlap
		const size_t es = type_size(ring_value_type(ring));
		const uintptr_t ub = reinterpret_cast<uintptr_t>(u), vb = reinterpret_cast<uintptr_t>(v);
		const uintptr_t ue = ub + size_t(m_out) * es, ve = vb + size_t(n_in) * es;
		ALPB_CHECK(!(u && v && m_out > 0 && n_in > 0 && ub < ve && vb < ue), ALPB_OVERLAP,
			"alpb_mxv_dense_noalloc: output and input vectors overlap");
	}
	if (m_out == 0 || nnz == 0 || n_in == 0) return ALPB_SUCCESS;  // no row gets a value
	ALPB_CHECK(offsets && indices && u && v, ALPB_ILLEGAL, "alpb_mxv_dense_noalloc: null pointer");
	unsigned char *base = nullptr;
	const int rc = noalloc_scratch(&base);
	if (rc != ALPB_SUCCESS) return rc;
	cudaStream_t s = as_stream(stream);
	const int64_t ntiles = (m_out + nnz + MP_TILE - 1) / MP_TILE;
	MergeTables mt;
	mt.m = m_out;
	mt.nnz = nnz;
	mt.ntiles = ntiles;
	int64_t *tile_row = reinterpret_cast<int64_t *>(base + NoallocLayout::tile_row);
	int64_t *head_first = reinterpret_cast<int64_t *>(base + NoallocLayout::head_first);
	int64_t *tail_first = reinterpret_cast<int64_t *>(base + NoallocLayout::tail_first);
	int32_t *span_len = reinterpret_cast<int32_t *>(base + NoallocLayout::span_len);
	int32_t *counter = reinterpret_cast<int32_t *>(base + NoallocLayout::counter);
	mt.tile_row = tile_row;
	mt.head_first = head_first;
	mt.tail_first = tail_first;
	mt.span_len = span_len;
	mt.counter = counter;
	mt.head_val = reinterpret_cast<uint64_t *>(base + NoallocLayout::head_val);
	mt.tail_val = reinterpret_cast<uint64_t *>(base + NoallocLayout::tail_val);
	mt.head_has = base + NoallocLayout::head_has;
	mt.tail_has = base + NoallocLayout::tail_has;
	// counters start at zero; every other table is rewritten below before it is read
	k_noalloc_clear<<<grid_for(ntiles, 256), 256, 0, s>>>(counter, ntiles);
	ALPB_LAUNCHED();
	k_merge_tiles<<<grid_for(ntiles + 1, 256), 256, 0, s>>>(offsets, m_out, nnz, ntiles, tile_row);
	ALPB_LAUNCHED();
	k_merge_tables<<<grid_for(ntiles, 256), 256, 0, s>>>(offsets, m_out, nnz, ntiles, tile_row,
		head_first, tail_first, span_len);
	ALPB_LAUNCHED();
	const int left = (form & ALPB_FORM_LEFT) ? 1 : 0;
	if (value_type == ALPB_VOID) values = nullptr;  // pattern matrix: nonzeroes take One
	switch (ring) {
	case ALPB_RING_PLUS_TIMES_F64:
		return noalloc_run<RingPlusTimesF64>(mt, offsets, indices, values, v, u, left, s);
	case ALPB_RING_LOR_LAND_BOOL:
		return noalloc_run<RingLorLandBool>(mt, offsets, indices, values, v, u, left, s);
	case ALPB_RING_MIN_PLUS_I32:
		return noalloc_run<RingMinPlusI32>(mt, offsets, indices, values, v, u, left, s);
	case ALPB_RING_PLUS_PATTERN_F64:
		return noalloc_run<RingPlusPatternF64>(mt, offsets, indices, values, v, u, left, s);
	case ALPB_RING_PLUS_TIMES_I32:
		return noalloc_run<RingPlusTimesI32>(mt, offsets, indices, values, v, u, left, s);
	case ALPB_RING_PLUS_RIGHT_IF_U64:
		return noalloc_run<RingPlusRightIfU64>(mt, offsets, indices, values, v, u, left, s);
	case ALPB_RING_MAX_LEFT_IF_U64:
		return noalloc_run<RingMaxLeftIfU64>(mt, offsets, indices, values, v, u, left, s);
	case ALPB_RING_TIMES_PLUS_F64:
		return noalloc_run<RingTimesPlusF64>(mt, offsets, indices, values, v, u, left, s);
	}
	return ALPB_UNSUPPORTED;
}
