/*
 * The b200 overload of grb::algorithms::conjugate_gradient (fused device CG).
 * See graphblas/b200/fused_algorithms.hpp for when the fused path is taken.
 */
#ifndef _H_GRB_B200_FUSED_CG
#define _H_GRB_B200_FUSED_CG

#include <graphblas/b200/fused_algorithms.hpp>

namespace grb {

	namespace algorithms {

		/**
		 * conjugate_gradient on b200 containers (conjugate_gradient.hpp:490-583):
		 * for FP64 x, A, b with the default ring, minus and divide and no
		 * descriptor other than no_casting, dense and force_row_major (which the
		 * fused path meets anyway: dense inputs, row storage), ONE persistent
		 * cooperative launch (alpb_cg_solve, on the
		 * matrix's cached plan) runs the whole solve with the template's numerics
		 * -- relative tolerance tol * ||b||, stop when sqrt(r.r) < tol, residual
		 * = r.r, FAILED when not converged after max_iterations.  r receives the
		 * final residual vector; u and temp are work space, as in the template.
		 * Anything else runs ALP's template unchanged.
		 */
		template<
			Descriptor descr = descriptors::no_operation,
			typename IOType,
			typename ResidualType,
			typename NonzeroType,
			typename InputType,
			class Ring = Semiring<
				grb::operators::add< IOType >, grb::operators::mul< IOType >,
				grb::identities::zero, grb::identities::one
			>,
			class Minus = operators::subtract< IOType >,
			class Divide = operators::divide< IOType >,
			typename RSI, typename NZI
		>
		grb::RC conjugate_gradient(
			grb::Vector< IOType, b200 > &x,
			const grb::Matrix< NonzeroType, b200, RSI, RSI, NZI > &A,
			const grb::Vector< InputType, b200 > &b,
			const size_t max_iterations,
			ResidualType tol,
			size_t &iterations,
			ResidualType &residual,
			grb::Vector< IOType, b200 > &r,
			grb::Vector< IOType, b200 > &u,
			grb::Vector< IOType, b200 > &temp,
			const Ring &ring = Ring(),
			const Minus &minus = Minus(),
			const Divide &divide = Divide()
		) {
			using namespace grb::internal::b200rt;
			constexpr bool fusable =
				std::is_same< IOType, double >::value && std::is_same< ResidualType, double >::value &&
				std::is_same< NonzeroType, double >::value && std::is_same< InputType, double >::value &&
				std::is_same< Ring, internal_b200_fused::RealRing >::value &&
				std::is_same< Minus, operators::subtract< double > >::value &&
				std::is_same< Divide, operators::divide< double > >::value &&
				( descr & ~( descriptors::no_casting | descriptors::dense |
					descriptors::force_row_major ) ) == descriptors::no_operation;
			const size_t n = A.b200_rows();
			const bool ok = fusable && A.b200_cols() == n && x.b200_size() == n &&
				b.b200_size() == n && r.b200_size() == n && u.b200_size() == n &&
				temp.b200_size() == n && n > 0 && max_iterations > 0 && tol > 0 &&
				internal_b200_fused::is_dense( x ) && internal_b200_fused::is_dense( b );
			if( !ok ) {
				return grb::algorithms::conjugate_gradient< descr, IOType, ResidualType, NonzeroType,
					InputType, Ring, Minus, Divide, RSI, NZI, b200 >( x, A, b, max_iterations, tol,
					iterations, residual, r, u, temp, ring, minus, divide );
			}
			x.b200_device_ready();
			b.b200_device_ready();
			const auto &crs = A.b200_crs();
			const alpb_spmv_plan plan = A.b200_plan( true );
			double *work = nullptr;
			RC rc = check( alpb_malloc( reinterpret_cast< void ** >( &work ), 4 * n * sizeof( double ) ),
				"conjugate_gradient" );
			if( rc != SUCCESS ) { return rc; }
			int64_t it = 0;
			double res = 0.0;
			rc = check( alpb_cg_solve( static_cast< int64_t >( n ), crs.offsets, crs.indices,
				reinterpret_cast< const double * >( crs.values ),
				reinterpret_cast< const double * >( b.b200_values() ),
				reinterpret_cast< double * >( x.b200_values() ), static_cast< int64_t >( max_iterations ),
				static_cast< double >( tol ), &it, &res, work, plan, stream() ),
				"conjugate_gradient" );
			if( rc == SUCCESS || rc == FAILED ) {
				// r is the final residual vector, as the template leaves it
				r.b200_device_ready();
				const RC c = check( alpb_memcpy_d2d( r.b200_values(), work, n * sizeof( double ),
					stream() ), "conjugate_gradient" );
				const RC d1 = internal_b200_fused::mark_dense( r );
				const RC d2 = internal_b200_fused::mark_dense( x );
				if( rc == SUCCESS ) { rc = c ? c : ( d1 ? d1 : d2 ); }
			}
			(void) alpb_stream_sync( stream() );
			(void) alpb_free( work );
			iterations = static_cast< size_t >( it );
			residual = static_cast< ResidualType >( res );
			internal_b200_fused::trace( "conjugate_gradient", n, it );
			return rc;
		}

	} // namespace algorithms

} // namespace grb

#endif
