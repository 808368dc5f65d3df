/*
 * The b200 overload of grb::algorithms::simple_pagerank (fused device PageRank).
 * See graphblas/b200/fused_algorithms.hpp for when the fused path is taken.
 */
#ifndef _H_GRB_B200_FUSED_PAGERANK
#define _H_GRB_B200_FUSED_PAGERANK

#include <graphblas/b200/fused_algorithms.hpp>

namespace grb {

	namespace algorithms {

		/**
		 * simple_pagerank on b200 containers (simple_pagerank.hpp:140-533): for
		 * an FP64 or pattern (void) link matrix and FP64 vectors with no
		 * descriptor, ONE
		 * persistent cooperative launch (alpb_pagerank_planned over L's column
		 * storage, on its cached plan) runs the out-degree scaling and every
		 * iteration with the template's numerics: initial guess 1/n unless pr
		 * is dense, teleport and dangling term (alpha * dangling + 1 - alpha) / n,
		 * L1 residual, stop when it is <= conv (conv != 0) or after max
		 * iterations, FAILED when not converged, *quality = the last residual.
		 * pr_next, pr_nextnext, row_sum and is_dangling are work space, as in
		 * the template, and are left untouched.  Anything else runs ALP's
		 * template unchanged.
		 */
		template< Descriptor descr = descriptors::no_operation, typename NonzeroT >
		RC simple_pagerank(
			Vector< double, b200 > &pr,
			const Matrix< NonzeroT, b200 > &L,
			Vector< double, b200 > &pr_next,
			Vector< double, b200 > &pr_nextnext,
			Vector< double, b200 > &row_sum,
			Vector< bool, b200 > &is_dangling,
			const double alpha = 0.85,
			const double conv = 0.0000001,
			const size_t max = 1000,
			size_t * const iterations = nullptr,
			double * const quality = nullptr
		) {
			using namespace grb::internal::b200rt;
			constexpr bool pattern = std::is_void< NonzeroT >::value;
			constexpr bool fusable = pattern || std::is_same< NonzeroT, double >::value;
			const size_t n = L.b200_rows();
			const bool ok = fusable &&
				( descr & ~descriptors::no_casting ) == descriptors::no_operation &&
				n > 0 && L.b200_cols() == n && pr.b200_size() == n && pr_next.b200_size() == n &&
				pr_nextnext.b200_size() == n && row_sum.b200_size() == n &&
				alpha > 0 && alpha < 1 && max > 0;
			if( !ok ) {
				return grb::algorithms::simple_pagerank< descr, double, NonzeroT >( pr, L, pr_next,
					pr_nextnext, row_sum, is_dangling, alpha, conv, max, iterations, quality );
			}
			const bool init_given = internal_b200_fused::is_dense( pr );
			pr.b200_device_ready();
			const auto &crs = L.b200_crs();
			const auto &ccs = L.b200_ccs();
			const alpb_spmv_plan plan = L.b200_nnz() > 0 ? L.b200_plan( false ) : nullptr;
			int64_t it = 0;
			double res = 0.0;
			// a pattern matrix passes no values: every stored entry is a one
			const double * const crs_val = pattern ? nullptr :
				reinterpret_cast< const double * >( crs.values );
			const double * const ccs_val = pattern ? nullptr :
				reinterpret_cast< const double * >( ccs.values );
			RC rc = check( alpb_pagerank_planned( static_cast< int64_t >( n ), crs.offsets,
				crs.indices, crs_val, ccs.offsets, ccs.indices, ccs_val, pr.b200_values(),
				init_given ? 1 : 0, alpha, conv, static_cast< int64_t >( max ), &it, &res, nullptr,
				plan, stream() ), "simple_pagerank" );
			if( rc == SUCCESS || rc == FAILED ) {
				const RC d = internal_b200_fused::mark_dense( pr );
				if( rc == SUCCESS ) { rc = d; }
				if( iterations != nullptr ) { *iterations = static_cast< size_t >( it ); }
				if( quality != nullptr ) { *quality = res; }
			}
			internal_b200_fused::trace( "simple_pagerank", n, it );
			return rc;
		}

	} // namespace algorithms

} // namespace grb

#endif
