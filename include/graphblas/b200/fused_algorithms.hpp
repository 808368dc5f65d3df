/*
 * Shared helpers of the fused device solvers of the b200 backend behind ALP's
 * own algorithm API (fused_cg.hpp, fused_pagerank.hpp, fused_hpcg.hpp).
 * ALP's algorithms are templates over the backend; these overloads fix it to
 * b200, so partial ordering picks them for b200 containers, and an unchanged
 * ALP program that calls
 *
 *   grb::algorithms::conjugate_gradient   (conjugate_gradient.hpp:490-583)
 *   grb::algorithms::simple_pagerank      (simple_pagerank.hpp:140-533)
 *   grb::algorithms::hpcg                 (hpcg/hpcg.hpp:60-223)
 *
 * gets one persistent device launch per solve (alpb_cg_solve,
 * alpb_pagerank_planned, alpb_hpcg_solve) instead of a blocking primitive per
 * step.  Each overload takes the fused path only where the fused kernel
 * computes exactly what the template computes: FP64 containers, the
 * default (+, *) ring and operators, no descriptor, dense inputs, and for
 * HPCG a system that build_hpcg_system made (recognised on the device).
 * Everything else -- other domains, rings, descriptors, sparse inputs, size
 * errors -- goes to ALP's template unchanged, which then returns the
 * reference's codes.  Results equal the templates' within FP64 rounding
 * (the same iteration counts and stopping rules; sums in another order).
 *
 * Each overload sits in its own header, included by the overlay of the ALP
 * header it overloads (graphblas/algorithms/conjugate_gradient.hpp,
 * simple_pagerank.hpp, hpcg/hpcg.hpp) right after that header, so that its
 * fall-back call names ALP's template.
 */
#ifndef _H_GRB_B200_FUSED_ALGORITHMS
#define _H_GRB_B200_FUSED_ALGORITHMS

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <type_traits>

#include <graphblas.hpp>
#include <graphblas/b200/runtime.hpp>

namespace grb {

	namespace algorithms {

		namespace internal_b200_fused {

			typedef Semiring< operators::add< double >, operators::mul< double >,
				identities::zero, identities::one > RealRing;

			template< typename D, typename C >
			bool is_dense( const Vector< D, b200, C > &x ) {
				const_cast< Vector< D, b200, C > & >( x ).b200_refresh();
				return x.b200_dense() || x.b200_size() == 0;
			}

			/** With ALPB_TRACE set in the environment, one line on stderr per
			 *  solve that took the fused path: which solver, its size and the
			 *  iterations it ran. */
			inline void trace( const char * const solver, const size_t n, const int64_t iterations ) {
				static const bool on = std::getenv( "ALPB_TRACE" ) != nullptr;
				if( on ) {
					std::fprintf( stderr, "grb::b200: fused %s, n = %zu, %lld iterations\n", solver, n,
						static_cast< long long >( iterations ) );
				}
			}

			/** A kernel wrote all n entries of x: mark every one assigned. */
			template< typename D, typename C >
			RC mark_dense( Vector< D, b200, C > &x ) {
				using namespace grb::internal::b200rt;
				const size_t n = x.b200_size();
				if( n == 0 ) { return SUCCESS; }
				RC rc = check( alpb_memset( x.b200_flags(), 1, n, stream() ), "mark_dense" );
				const int64_t cnt = static_cast< int64_t >( n );
				rc = rc ? rc : check( alpb_memcpy_h2d( x.b200_counter(), &cnt, 8, stream() ),
					"mark_dense" );
				rc = rc ? rc : check( alpb_stream_sync( stream() ), "mark_dense" );
				if( rc == SUCCESS ) { x.b200_mark_dense(); }
				return rc;
			}

		}

	} // namespace algorithms

} // namespace grb

#endif
