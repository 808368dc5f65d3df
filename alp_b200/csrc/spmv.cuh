// Internal interface of the SpMV engine, shared by the solvers.
#pragma once
#include "common.cuh"

// Schedule chosen for one compressed storage, with the merge-path tile table
// and carry table (the scratch memory of the merge-path kernel).
struct alpb_spmv_plan_s {
	int64_t m = 0, nnz = 0;
	const int64_t *offsets = nullptr;  // storage the plan was made for
	int sched = ALPB_SCHED_VECTOR;
	int vw = 8;
	int device = 0;
	int64_t ntiles = 0;
	int64_t tile = 0;               // merge items per tile of the tables below
	// merge-path tables (the scratch memory of the merge-path schedule)
	int64_t *tile_row = nullptr;    // ntiles + 1 merge-path row splits
	int64_t *head_first = nullptr;  // ntiles
	int64_t *tail_first = nullptr;  // ntiles
	int32_t *span_len = nullptr;    // ntiles
	int32_t *counter = nullptr;     // ntiles (zero between products)
	uint64_t *head_val = nullptr;   // ntiles
	uint64_t *tail_val = nullptr;   // ntiles
	uint8_t *head_has = nullptr;    // ntiles
	uint8_t *tail_has = nullptr;    // ntiles
	int32_t *ready = nullptr;       // ntiles (publication epochs, fused solvers)
	// [ntiles+1] first merge diagonal of each tile when the tiles are cut at
	// row boundaries (short rows: no row crosses a tile); null: t * tile
	int64_t *tile_d = nullptr;
	double mean = 0, maxlen = 0, cv = 0;
	float tuned_ms = 0;
	// Hot-column cache of the merge path, for skewed (power-law) matrices;
	// made by the autotuner when it wins.  The hot_k most frequent columns of
	// the index array `hot_src` get shared-memory slots: hot_idx is that
	// array with every hot column replaced by (slot | 1 << 31), and each
	// product gathers x at hot_cols into hot_x, which every block copies into
	// shared memory, so the gathers of those nonzeroes never leave the SM.
	int64_t hot_k = 0;
	int hot_on = 0;
	double hot_cover = 0;               // share of the nonzeroes in hot columns
	const uint32_t *hot_src = nullptr;  // the column indices hot_idx was made from
	uint32_t *hot_idx = nullptr;        // nnz
	uint32_t *hot_cols = nullptr;       // hot_k
	uint64_t *hot_x = nullptr;          // hot_k values (8 bytes hold any ring's type)
	// Boolean lor/land path: the nonzeroes of every row beyond its first
	// LOR_HEAD, cut in chunks of LOR_CHUNK; chunk c covers
	// [lor_k0[c], min(lor_k0[c] + LOR_CHUNK, offsets[lor_row[c] + 1])).
	// lor_n < 0: not built (the plan was made for a fused solver).
	int64_t lor_n = -1;
	int64_t *lor_row = nullptr;
	int64_t *lor_k0 = nullptr;
};

namespace alpb {

struct SpmvArgs {
	int64_t m_out, n_in, nnz;
	const int64_t *offsets;
	const uint32_t *indices;
	const void *values;  // nullptr: pattern matrix
	void *u;
	uint8_t *u_assigned;
	int64_t *u_nnz;
	const void *u_mask;
	const uint8_t *u_mask_assigned;
	int u_mask_type;
	const void *v;
	const uint8_t *v_assigned;
	const void *v_mask;
	const uint8_t *v_mask_assigned;
	int v_mask_type;
	uint32_t descr;
	int left;
	bool masked, input_masked, dense_all, trivial;
	// Path semantics of the reference (see alpb_mxv): the output mask is read
	// by structure only when the reference walks the mask's assigned set, and
	// the scatter path applies add_identity outside the output mask and
	// ignores explicit_zero.
	bool mask_by_structure, scatter_sem;
};

// Run one SpMV with the plan's schedule (force_sched != 0 overrides it).
int dispatch_spmv(int ring, const SpmvArgs &a, const alpb_spmv_plan_s *p, int force_sched,
	cudaStream_t s);
int ring_value_type(int ring);

// merge-path geometry of the block-tile engine (merge.cuh), shared with the
// fused solvers
constexpr int MP_BLOCK = 256;
constexpr int MP_IPT = 8;
constexpr int MP_TILE = MP_BLOCK * MP_IPT;

// Rows per row-aligned warp tile for rows of at most `maxlen` (mean `mean`)
// nonzeroes, or 0 when whole-row tiles would be poorly filled.
int64_t aligned_rows_per_tile(double maxlen, double mean, int64_t tile);
// Longest row (and sum of squared row lengths) of a compressed storage.
int row_profile(const int64_t *offsets, int64_t m, double *maxlen, double *sumsq, cudaStream_t s);

// Plan with merge tables of `tile` items per tile (MP_TILE for the block
// engine, WM_TILE for the warp engine).
int plan_create_tiles(alpb_spmv_plan_s **plan, int64_t m, int64_t nnz, const int64_t *offsets,
	int sched, int vector_width, int64_t tile, cudaStream_t s);

} // namespace alpb
