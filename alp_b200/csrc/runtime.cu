// Runtime entry points: init/finalize, error reporting, device memory and
// copies used by the container classes of the grb::b200 backend.
#include "common.cuh"

#include <cstdarg>
#include <mutex>

namespace alpb {

std::atomic<int64_t> g_launches{0};

static thread_local char t_err[1024] = "";

void set_error(const char *fmt, ...) {
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(t_err, sizeof(t_err), fmt, ap);
	va_end(ap);
}

int sm_count() {
	static int cached[64] = {0};
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
	if (cached[dev] == 0) {
		int v = 0;
		if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
			v = 148;
		cached[dev] = v;
	}
	return cached[dev];
}

size_t type_size(int type) {
	switch (type) {
	case ALPB_VOID: return 0;
	case ALPB_BOOL: return 1;
	case ALPB_INT32: return 4;
	case ALPB_FP64: return 8;
	case ALPB_UINT32: return 4;
	case ALPB_INT64: return 8;
	case ALPB_UINT8: return 1;
	case ALPB_INT8: return 1;
	case ALPB_UINT64: return 8;
	}
	return 0;
}

} // namespace alpb

using namespace alpb;

extern "C" {

int alpb_version(void) { return 1; }

const char *alpb_last_error(void) { return t_err; }

int64_t alpb_launch_count(void) { return g_launches.load(); }

int alpb_init(int device) {
	int n = 0;
	ALPB_CUDA(cudaGetDeviceCount(&n));
	ALPB_CHECK(device >= 0 && device < n, ALPB_ILLEGAL, "alpb_init: device %d of %d", device, n);
	ALPB_CUDA(cudaSetDevice(device));
	ALPB_CUDA(cudaFree(nullptr));  // create the primary context now
	// the entry points take their small per-call scratch (block partials,
	// solver state) stream-ordered from the device's default pool: keep what
	// they free in the pool instead of returning it to the driver at every
	// synchronisation, so that repeated calls reuse it
	cudaMemPool_t pool;
	ALPB_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
	uint64_t keep = UINT64_MAX;
	ALPB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
	return ALPB_SUCCESS;
}

int alpb_finalize(void) {
	ALPB_CUDA(cudaDeviceSynchronize());
	return ALPB_SUCCESS;
}

int alpb_malloc(void **ptr, size_t bytes) {
	ALPB_CHECK(ptr != nullptr, ALPB_ILLEGAL, "alpb_malloc: null out pointer");
	*ptr = nullptr;
	if (bytes == 0) return ALPB_SUCCESS;
	bytes = (bytes + 255) & ~size_t(255);
	cudaError_t e = cudaMalloc(ptr, bytes);
	if (e == cudaErrorMemoryAllocation) {
		cudaGetLastError();
		set_error("alpb_malloc: out of device memory for %zu bytes", bytes);
		return ALPB_OUTOFMEM;
	}
	ALPB_CUDA(e);
	return ALPB_SUCCESS;
}

int alpb_malloc_managed(void **ptr, size_t bytes) {
	ALPB_CHECK(ptr != nullptr, ALPB_ILLEGAL, "alpb_malloc_managed: null out pointer");
	*ptr = nullptr;
	if (bytes == 0) return ALPB_SUCCESS;
	bytes = (bytes + 255) & ~size_t(255);
	cudaError_t e = cudaMallocManaged(ptr, bytes, cudaMemAttachGlobal);
	if (e == cudaErrorMemoryAllocation) {
		cudaGetLastError();
		set_error("alpb_malloc_managed: out of memory for %zu bytes", bytes);
		return ALPB_OUTOFMEM;
	}
	ALPB_CUDA(e);
	return ALPB_SUCCESS;
}

int alpb_prefetch(const void *ptr, size_t bytes, int to_device, void *stream) {
	if (!ptr || bytes == 0) return ALPB_SUCCESS;
	int dev = 0;
	ALPB_CUDA(cudaGetDevice(&dev));
	cudaMemLocation loc;
	loc.type = to_device ? cudaMemLocationTypeDevice : cudaMemLocationTypeHost;
	loc.id = to_device ? dev : 0;
	cudaError_t e = cudaMemPrefetchAsync(ptr, bytes, loc, 0, as_stream(stream));
	if (e != cudaSuccess) {
		// prefetching is a hint: ignore devices without managed-memory support
		cudaGetLastError();
	}
	return ALPB_SUCCESS;
}

int alpb_free(void *ptr) {
	if (ptr) ALPB_CUDA(cudaFree(ptr));
	return ALPB_SUCCESS;
}

int alpb_memcpy_h2d(void *dst, const void *src, size_t bytes, void *stream) {
	if (bytes == 0) return ALPB_SUCCESS;
	ALPB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, as_stream(stream)));
	return ALPB_SUCCESS;
}

int alpb_memcpy_d2h(void *dst, const void *src, size_t bytes, void *stream) {
	if (bytes == 0) return ALPB_SUCCESS;
	ALPB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, as_stream(stream)));
	return ALPB_SUCCESS;
}

int alpb_memcpy_d2d(void *dst, const void *src, size_t bytes, void *stream) {
	if (bytes == 0) return ALPB_SUCCESS;
	ALPB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, as_stream(stream)));
	return ALPB_SUCCESS;
}

int alpb_memset(void *dst, int byte, size_t bytes, void *stream) {
	if (bytes == 0) return ALPB_SUCCESS;
	ALPB_CUDA(cudaMemsetAsync(dst, byte, bytes, as_stream(stream)));
	return ALPB_SUCCESS;
}

int alpb_stream_sync(void *stream) {
	ALPB_CUDA(cudaStreamSynchronize(as_stream(stream)));
	return ALPB_SUCCESS;
}

} // extern "C"
