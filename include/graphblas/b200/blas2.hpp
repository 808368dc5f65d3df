/*
 * grb::mxv / grb::vxm of the b200 backend (reference: graphblas/reference/
 * blas2.hpp:1532-2230).  Every overload resolves, as the reference does at
 * blas2.hpp:1848, which orientation is gathered -- mxv gathers A's CRS, vxm
 * A's CCS, and transpose_matrix swaps them -- and calls alpb_mxv, which
 * carries the semiring, masks and descriptor semantics on the device.
 */
#ifndef _H_GRB_B200_BLAS2
#define _H_GRB_B200_BLAS2

#include <type_traits>

#include <graphblas/base/blas2.hpp>
#include <graphblas/b200/io.hpp>
#include <graphblas/b200/matrix.hpp>
#include <graphblas/b200/runtime.hpp>
#include <graphblas/b200/vector.hpp>

namespace grb {

	namespace internal {
		namespace b200rt {

			/** u (+)= A (x) v (left = false) or v (x) A (left = true). */
			template< Descriptor descr, bool left, class Ring, typename IOType,
				typename InputType1, typename InputType2, typename InputType3,
				typename InputType4, typename RIT, typename CIT, typename NIT, typename Coords >
			RC spmv( Vector< IOType, grb::b200, Coords > &u,
				const Vector< InputType3, grb::b200, Coords > &u_mask,
				const Matrix< InputType2, grb::b200, RIT, CIT, NIT > &A,
				const Vector< InputType1, grb::b200, Coords > &v,
				const Vector< InputType4, grb::b200, Coords > &v_mask, const Ring &ring,
				const Phase &phase
			) {
				constexpr int ring_id = ring_code< typename Ring::AdditiveOperator,
					typename Ring::MultiplicativeOperator >::value;
				constexpr bool transposed = ( descr & descriptors::transpose_matrix ) != 0;
				// the gather runs over A's CRS for mxv, over its CCS for vxm; the
				// transpose_matrix descriptor swaps the orientation
				constexpr bool rows = left ? transposed : !transposed;
				const size_t m = nrows( A ), n = ncols( A );
				const size_t out_len = rows ? m : n, in_len = rows ? n : m;
				if( size( u ) != out_len || size( v ) != in_len ) { return MISMATCH; }
				const bool masked = size( u_mask ) > 0, input_masked = size( v_mask ) > 0;
				if( masked && size( u_mask ) != out_len ) { return MISMATCH; }
				if( input_masked && size( v_mask ) != in_len ) { return MISMATCH; }
				if( phase == RESIZE ) { return SUCCESS; }
				if( ring_id < 0 ) { return UNSUPPORTED; }
				const int vt = type_code< InputType2 >::value;
				const int ut = type_code< IOType >::value, xt = type_code< InputType1 >::value;
				// vectors of another domain than the ring's are cast element-wise, as
				// ALP's operators cast their operands: stage them through vectors of
				// the ring's output domain, keeping their sparsity
				typedef typename Ring::D4 RD;
				constexpr int rt = type_code< RD >::value;
				if( rt >= 0 && ut >= 0 && xt >= 0 && ( ut != rt || xt != rt ) ) {
					Vector< RD, grb::b200, Coords > us( out_len ), vs( in_len );
					RC rc = set( us, u );
					rc = rc ? rc : set( vs, v );
					rc = rc ? rc : spmv< descr, left >( us, u_mask, A, vs, v_mask, ring, phase );
					rc = rc ? rc : set( u, us );
					return rc;
				}
				const int mt = type_code< InputType3 >::value, vmt = type_code< InputType4 >::value;
				if( vt < 0 || mt < 0 || vmt < 0 || ut != xt || ut < 0 ) { return UNSUPPORTED; }
				if( vt != ALPB_VOID && vt != ut ) { return UNSUPPORTED; }
				// the ring's identities must be the standard ones of its operators
				{
					const double z0 = static_cast< double >( ring.template getZero< IOType >() );
					const double o1 = static_cast< double >( ring.template getOne< IOType >() );
					if( ring_id == ALPB_RING_PLUS_TIMES_F64 && ( z0 != 0.0 || o1 != 1.0 ) ) {
						return UNSUPPORTED;
					}
					if( ring_id == ALPB_RING_TIMES_PLUS_F64 && ( z0 != 1.0 || o1 != 0.0 ) ) {
						return UNSUPPORTED;
					}
					if( ( ring_id == ALPB_RING_PLUS_RIGHT_IF_U64 ||
						ring_id == ALPB_RING_MAX_LEFT_IF_U64 ) && z0 != 0.0 ) {
						return UNSUPPORTED;
					}
				}
				const auto &S = rows ? A.b200_crs() : A.b200_ccs();
				u.b200_device_ready();
				v.b200_device_ready();
				if( masked ) { u_mask.b200_device_ready(); }
				if( input_masked ) { v_mask.b200_device_ready(); }
				const int form = ( left ? ALPB_FORM_LEFT : 0 ) | ( rows ? ALPB_FORM_ROWS : 0 );
				const int64_t u_mask_count = masked ? static_cast< int64_t >( nnz( u_mask ) ) : -1;
				const int64_t v_mask_count = input_masked ? static_cast< int64_t >( nnz( v_mask ) ) : -1;
				const RC rc = check( alpb_mxv( ring_id, static_cast< uint32_t >(
						descr & ~descriptors::transpose_matrix ), form,
					static_cast< int64_t >( out_len ), static_cast< int64_t >( in_len ),
					static_cast< int64_t >( nnz( A ) ), S.offsets, S.indices,
					vt == ALPB_VOID ? nullptr : S.values, vt,
					u.b200_values(), u.b200_flags_or_dense(), u.b200_counter(),
					masked ? u_mask.b200_values() : nullptr,
					masked ? u_mask.b200_flags_or_dense() : nullptr, mt, u_mask_count,
					v.b200_values(), v.b200_flags_or_dense(), static_cast< int64_t >( nnz( v ) ),
					input_masked ? v_mask.b200_values() : nullptr,
					input_masked ? v_mask.b200_flags_or_dense() : nullptr, vmt, v_mask_count,
					A.b200_plan( rows ), stream() ), left ? "vxm" : "mxv" );
				(void) alpb_stream_sync( stream() );
				u.b200_refresh();
				return rc;
			}

		}
	}

	// ------------------------------------------------------------------ mxv --
	template< Descriptor descr = descriptors::no_operation, class Ring, typename IOType,
		typename InputType1, typename InputType2, typename InputType3, typename InputType4,
		typename RIT, typename CIT, typename NIT, typename Coords >
	RC mxv( Vector< IOType, b200, Coords > &u, const Vector< InputType3, b200, Coords > &mask,
		const Matrix< InputType2, b200, RIT, CIT, NIT > &A,
		const Vector< InputType1, b200, Coords > &v,
		const Vector< InputType4, b200, Coords > &v_mask, const Ring &ring = Ring(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_semiring< Ring >::value, void >::type * const = nullptr
	) {
		return internal::b200rt::spmv< descr, false >( u, mask, A, v, v_mask, ring, phase );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename IOType,
		typename InputType1, typename InputType2, typename InputType3, typename RIT,
		typename CIT, typename NIT, typename Coords >
	RC mxv( Vector< IOType, b200, Coords > &u, const Vector< InputType3, b200, Coords > &mask,
		const Matrix< InputType2, b200, RIT, CIT, NIT > &A,
		const Vector< InputType1, b200, Coords > &v, const Ring &ring = Ring(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_semiring< Ring >::value, void >::type * const = nullptr
	) {
		const Vector< bool, b200, Coords > empty( 0 );
		return internal::b200rt::spmv< descr, false >( u, mask, A, v, empty, ring, phase );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename IOType,
		typename InputType1, typename InputType2, typename RIT, typename CIT, typename NIT,
		typename Coords >
	RC mxv( Vector< IOType, b200, Coords > &u, const Matrix< InputType2, b200, RIT, CIT, NIT > &A,
		const Vector< InputType1, b200, Coords > &v, const Ring &ring = Ring(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_semiring< Ring >::value, void >::type * const = nullptr
	) {
		const Vector< bool, b200, Coords > empty( 0 );
		return internal::b200rt::spmv< descr, false >( u, empty, A, v, empty, ring, phase );
	}

	// ------------------------------------------------------------------ vxm --
	template< Descriptor descr = descriptors::no_operation, class Ring, typename IOType,
		typename InputType1, typename InputType2, typename InputType3, typename InputType4,
		typename RIT, typename CIT, typename NIT, typename Coords >
	RC vxm( Vector< IOType, b200, Coords > &u, const Vector< InputType3, b200, Coords > &mask,
		const Vector< InputType1, b200, Coords > &v,
		const Vector< InputType4, b200, Coords > &v_mask,
		const Matrix< InputType2, b200, RIT, CIT, NIT > &A, const Ring &ring = Ring(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_semiring< Ring >::value, void >::type * const = nullptr
	) {
		return internal::b200rt::spmv< descr, true >( u, mask, A, v, v_mask, ring, phase );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename IOType,
		typename InputType1, typename InputType2, typename InputType3, typename RIT,
		typename CIT, typename NIT, typename Coords >
	RC vxm( Vector< IOType, b200, Coords > &u, const Vector< InputType3, b200, Coords > &mask,
		const Vector< InputType1, b200, Coords > &v,
		const Matrix< InputType2, b200, RIT, CIT, NIT > &A, const Ring &ring = Ring(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_semiring< Ring >::value, void >::type * const = nullptr
	) {
		const Vector< bool, b200, Coords > empty( 0 );
		return internal::b200rt::spmv< descr, true >( u, mask, A, v, empty, ring, phase );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename IOType,
		typename InputType1, typename InputType2, typename RIT, typename CIT, typename NIT,
		typename Coords >
	RC vxm( Vector< IOType, b200, Coords > &u, const Vector< InputType1, b200, Coords > &v,
		const Matrix< InputType2, b200, RIT, CIT, NIT > &A, const Ring &ring = Ring(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_semiring< Ring >::value, void >::type * const = nullptr
	) {
		const Vector< bool, b200, Coords > empty( 0 );
		return internal::b200rt::spmv< descr, true >( u, empty, A, v, empty, ring, phase );
	}


	/** eWiseLambda over a matrix: f( i, j, a_ij ) on the host for every stored
	 *  entry; changed values reach both stored orientations.  Vectors among
	 *  `args` are made readable on the host first. */
	template< Descriptor descr = descriptors::no_operation, class Func, typename DataType,
		typename RIT, typename CIT, typename NIT, typename... Args >
	RC eWiseLambda( const Func f, const Matrix< DataType, b200, RIT, CIT, NIT > &A,
		const Args &... args
	) {
		internal::b200rt::touch( args... );
		Func g = f;
		return const_cast< Matrix< DataType, b200, RIT, CIT, NIT > & >( A ).b200_host_lambda( g );
	}

}

#endif
