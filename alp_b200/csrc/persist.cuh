// Persistent (cooperative) kernel support: a grid barrier whose every wait is
// bounded, and a deterministic block reduction.
#pragma once
#include "common.cuh"

namespace alpb {

// Barrier state in device memory; zero-initialise before the launch.  The
// arrival counter only grows: barrier k of the launch completes when it
// reaches k * gridDim.x, so no block resets it and no second word is flipped.
// The counter and the error flag sit on separate 128-byte lines.
struct alignas(128) GridSync {
	unsigned long long count;
	unsigned int pad0[30];
	unsigned int gen;   // not used by grid_sync (kept for the layout)
	int err;    // 1: a barrier or tile wait gave up (the kernel exits; host reports PANIC)
	unsigned int pad1[30];
};

// ~1 s at the sleep granularity below: far beyond any legitimate wait of a
// co-resident grid, short enough to keep the context usable on a fault.
constexpr long long kSpinLimit = 1ll << 24;

// All blocks of a cooperative launch call this the same number of times.
// Thread 0 arrives with one acquire-release add (its block's writes before
// the barrier are released; the last arrival acquires everyone's) and the
// others poll the counter with acquire loads until their barrier's target,
// so the last block to arrive goes on after one atomic round trip and the
// others one poll later.  Returns false once any block has timed out; callers
// then leave their loop.
__device__ __forceinline__ bool grid_sync(GridSync *gs) {
	__syncthreads();
	if (threadIdx.x == 0) {
		const unsigned long long G = gridDim.x;
		unsigned long long old;
		asm volatile("atom.add.acq_rel.gpu.global.u64 %0, [%1], 1;"
					 : "=l"(old) : "l"(&gs->count) : "memory");
		const unsigned long long target = (old / G + 1) * G;
		if (old + 1 != target) {
			volatile int *verr = &gs->err;
			long long spins = 0;
			for (;;) {
				unsigned long long c;
				asm volatile("ld.acquire.gpu.global.u64 %0, [%1];"
							 : "=l"(c) : "l"(&gs->count) : "memory");
				if (c >= target) break;
				if ((++spins & 63) == 0 && *verr) break;
				if (spins > kSpinLimit) {
					atomicExch(&gs->err, 1);
					break;
				}
				__nanosleep(32);
			}
		}
	}
	__syncthreads();
	return *((volatile int *) &gs->err) == 0;
}

// Sum over the block in a fixed order (warp trees, then warp 0 over the warp
// sums); the result is returned to every thread.
__device__ __forceinline__ double block_sum(double v, double *smem /* >= 33 */) {
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
	__syncthreads();
	if (lane == 0) smem[wid] = v;
	__syncthreads();
	if (wid == 0) {
		const int nw = (blockDim.x + 31) >> 5;
		double w = lane < nw ? smem[lane] : 0.0;
		for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
		if (lane == 0) smem[32] = w;
	}
	__syncthreads();
	return smem[32];
}

// Every block sums the same array in the same order (same value everywhere).
__device__ __forceinline__ double block_sum_array(const double *a, int64_t n, double *smem) {
	double v = 0.0;
	for (int64_t k = threadIdx.x; k < n; k += blockDim.x) v += ((const volatile double *) a)[k];
	return block_sum(v, smem);
}

// Largest grid of `kernel` whose blocks are all co-resident.
template <class K>
int cooperative_grid(K kernel, int block, size_t smem, int64_t want) {
	int per_sm = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess)
		return 0;
	int64_t g = int64_t(per_sm) * sm_count();
	if (want > 0 && want < g) g = want;
	return int(g);
}

// Grid of a persistent solver kernel over `ntiles` warp tiles: about four
// tiles per warp, at least two blocks per SM (latency hiding), at most the
// co-resident maximum.  Every grid barrier and every scalar reduction costs
// time in proportion to the block count, so small systems get small grids.
template <class K>
int solver_grid(K kernel, int block, int64_t ntiles, int warps_per_block, size_t smem = 0) {
	const int max_grid = cooperative_grid(kernel, block, smem, 0);
	int64_t g = ntiles / (4 * int64_t(warps_per_block));
	if (g < 2 * int64_t(sm_count())) g = 2 * int64_t(sm_count());
	if (g > max_grid) g = max_grid;
	return int(g);
}

} // namespace alpb
