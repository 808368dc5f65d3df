/*
 * I/O and container primitives of the b200 backend (reference:
 * graphblas/reference/io.hpp): size / nnz / capacity / clear / resize,
 * set and setElement, buildVector, buildMatrixUnique, wait.
 */
#ifndef _H_GRB_B200_IO
#define _H_GRB_B200_IO

#include <cstdint>
#include <string>
#include <type_traits>
#include <vector>

#include <graphblas/base/io.hpp>
#include <graphblas/blas0.hpp>

#include <graphblas/b200/matrix.hpp>
#include <graphblas/b200/runtime.hpp>
#include <graphblas/b200/vector.hpp>
#include <graphblas/iomode.hpp>

namespace grb {

	// ------------------------------------------------------------ queries --
	template< typename DataType, typename Coords >
	size_t size( const Vector< DataType, b200, Coords > &x ) noexcept { return x.b200_size(); }

	template< typename DataType, typename Coords >
	size_t nnz( const Vector< DataType, b200, Coords > &x ) noexcept { return x.b200_nnz(); }

	template< typename DataType, typename Coords >
	size_t capacity( const Vector< DataType, b200, Coords > &x ) noexcept { return x.b200_size(); }

	template< typename InputType, typename RIT, typename CIT, typename NIT >
	size_t nrows( const Matrix< InputType, b200, RIT, CIT, NIT > &A ) noexcept { return A.b200_rows(); }

	template< typename InputType, typename RIT, typename CIT, typename NIT >
	size_t ncols( const Matrix< InputType, b200, RIT, CIT, NIT > &A ) noexcept { return A.b200_cols(); }

	template< typename InputType, typename RIT, typename CIT, typename NIT >
	size_t nnz( const Matrix< InputType, b200, RIT, CIT, NIT > &A ) noexcept { return A.b200_nnz(); }

	template< typename DataType, typename RIT, typename CIT, typename NIT >
	size_t capacity( const Matrix< DataType, b200, RIT, CIT, NIT > &A ) noexcept {
		return A.b200_capacity();
	}

	template< typename InputType, typename Coords >
	uintptr_t getID( const Vector< InputType, b200, Coords > &x ) {
		return reinterpret_cast< uintptr_t >( x.b200_values() );
	}

	template< typename InputType, typename RIT, typename CIT, typename NIT >
	uintptr_t getID( const Matrix< InputType, b200, RIT, CIT, NIT > &A ) {
		return reinterpret_cast< uintptr_t >( A.b200_crs().offsets );
	}

	// ------------------------------------------------------ clear / resize --
	template< typename DataType, typename Coords >
	RC clear( Vector< DataType, b200, Coords > &x ) noexcept {
		const size_t n = x.b200_size();
		if( n == 0 ) { return SUCCESS; }
		x.b200_device_ready();
		RC rc = internal::b200rt::check( alpb_memset( x.b200_flags(), 0, n, internal::b200rt::stream() ),
			"clear" );
		if( rc == SUCCESS ) {
			rc = internal::b200rt::check( alpb_memset( x.b200_counter(), 0, 8, internal::b200rt::stream() ),
				"clear" );
		}
		(void) alpb_stream_sync( internal::b200rt::stream() );
		x.b200_mark_sparse();
		return rc;
	}

	template< typename InputType, typename RIT, typename CIT, typename NIT >
	RC clear( Matrix< InputType, b200, RIT, CIT, NIT > &A ) noexcept {
		try { A.b200_clear(); } catch( ... ) { return OUTOFMEM; }
		return SUCCESS;
	}

	/** Vector capacities are fixed at their size (IMPLEMENTATION<b200>). */
	template< typename InputType, typename Coords >
	RC resize( Vector< InputType, b200, Coords > &x, const size_t new_nz ) noexcept {
		return new_nz <= x.b200_size() ? SUCCESS : ILLEGAL;
	}

	template< typename InputType, typename RIT, typename CIT, typename NIT >
	RC resize( Matrix< InputType, b200, RIT, CIT, NIT > &A, const size_t new_nz ) noexcept {
		A.b200_reserve( new_nz );
		return SUCCESS;
	}

	/** C = A, structure and values cast to C's domain (reference/io.hpp
	 *  set( Matrix, Matrix )); same signature as the base declaration, so that
	 *  this b200 overload is the more specialised one. */
	template< Descriptor descr = descriptors::no_operation, typename OutputType,
		typename InputType, typename RIT, typename CIT, typename NIT >
	RC set( Matrix< OutputType, b200, RIT, CIT, NIT > &C,
		const Matrix< InputType, b200, RIT, CIT, NIT > &A, const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType >::value, void >::type * const = nullptr
	) {
		if( nrows( C ) != nrows( A ) || ncols( C ) != ncols( A ) ) { return MISMATCH; }
		if( static_cast< const void * >( &C ) == static_cast< const void * >( &A ) ) {
			return ILLEGAL;
		}
		if( phase == RESIZE ) {
			C.b200_reserve( nnz( A ) );
			return SUCCESS;
		}
		try {
			return C.b200_assign_from( A );
		} catch( ... ) {
			return OUTOFMEM;
		}
	}

	// ----------------------------------------------------------------- set --
	namespace internal {
		namespace b200rt {

			/** z = value over `mask` (or everywhere) through alpb_vec_op_dom (or
			 *  alpb_set_scalar for values a double holds exactly). */
			template< Descriptor descr, typename DataType, typename MaskType, typename T,
				typename Coords >
			RC set_scalar( Vector< DataType, grb::b200, Coords > &x,
				const Vector< MaskType, grb::b200, Coords > * const mask, const T val
			) {
				const size_t n = x.b200_size();
				if( n == 0 ) { return SUCCESS; }
				const int zt = type_code< DataType >::value;
				const int mt = mask ? type_code< MaskType >::value : ALPB_VOID;
				if( zt < 0 || mt < 0 ) { return UNSUPPORTED; }
				x.b200_device_ready();
				if( mask ) {
					mask->b200_device_ready();
					// the output is replaced, not updated, unless the dense descriptor
					// comes with a structurally dense mask (reference/io.hpp:509-520)
					const bool mask_dense = ( descr & descriptors::structural ) &&
						!( descr & descriptors::invert_mask ) &&
						( ( descr & descriptors::dense ) || nnz( *mask ) == n );
					if( ( descr & descriptors::dense ) && mask_dense ) {
						return set_scalar< descr, DataType, MaskType, T, Coords >( x, nullptr, val );
					}
					const RC crc = clear( x );
					if( crc != SUCCESS ) { return crc; }
				}
				// a 64-bit integer value does not fit a double: it takes the typed path
				constexpr int dom = domain_of< DataType, T >::value;
				// a dense vector set to a value joins the pending level-1 chain
				if( !mask && x.b200_dense() && fusion_enabled() && chain_type_ok( dom, zt ) &&
					record_step( ALPB_VEC_SET, ALPB_OP_RIGHT_ASSIGN, ALPB_OP_ADD, descr, dom, n,
						x.b200_values(), zt, nullptr, zt, static_cast< scalar_t >( val ), nullptr, zt, 0 )
				) {
					return SUCCESS;
				}
				if( !mask && !( descr & descriptors::use_index ) &&
					!( std::is_integral< DataType >::value && sizeof( DataType ) == 8 )
				) {
					const RC rc = check( alpb_set_scalar( x.b200_values(), zt, n, static_cast< double >( val ),
						x.b200_flags(), x.b200_counter(), stream() ), "set" );
					if( rc == SUCCESS ) { x.b200_mark_dense(); }
					return rc;
				}
				const RC rc = check( alpb_vec_op_dom( ALPB_VEC_SET, ALPB_OP_RIGHT_ASSIGN, 0, 0, 0,
					descr, dom, n, x.b200_values(), zt, x.b200_flags(), x.b200_counter(),
					mask ? mask->b200_values() : nullptr,
					mask ? mask->b200_flags_or_dense() : nullptr, mt, mask ? 1 : 0,
					nullptr, zt, nullptr, domain_bits( static_cast< scalar_t >( val ), dom ),
					nullptr, zt, nullptr, 0, stream() ), "set" );
				x.b200_refresh();
				return rc;
			}

		}
	}

	template< Descriptor descr = descriptors::no_operation, typename DataType, typename T,
		typename Coords >
	RC set( Vector< DataType, b200, Coords > &x, const T val, const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< DataType >::value &&
			!grb::is_object< T >::value, void >::type * const = nullptr
	) {
		// the dense descriptor promises a dense output (reference/io.hpp:404-406)
		if( ( descr & descriptors::dense ) && nnz( x ) < size( x ) ) { return ILLEGAL; }
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::set_scalar< descr, DataType, bool, T, Coords >( x, nullptr, val );
	}

	template< Descriptor descr = descriptors::no_operation, typename DataType,
		typename MaskType, typename T, typename Coords >
	RC set( Vector< DataType, b200, Coords > &x, const Vector< MaskType, b200, Coords > &m,
		const T val, const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< DataType >::value &&
			!grb::is_object< T >::value, void >::type * const = nullptr
	) {
		if( size( m ) == 0 ) { return set< descr >( x, val, phase ); }
		if( size( m ) != size( x ) ) { return MISMATCH; }
		if( ( descr & descriptors::dense ) && ( nnz( x ) < size( x ) || nnz( m ) < size( x ) ) ) {
			return ILLEGAL;  // reference/io.hpp:498-501
		}
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::set_scalar< descr >( x, &m, val );
	}

	template< Descriptor descr = descriptors::no_operation, typename DataType, typename T,
		typename Coords >
	RC setElement( Vector< DataType, b200, Coords > &x, const T val, const size_t i,
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< DataType >::value &&
			!grb::is_object< T >::value, void >::type * const = nullptr
	) {
		if( i >= size( x ) ) { return MISMATCH; }
		if( ( descr & descriptors::dense ) && nnz( x ) < size( x ) ) { return ILLEGAL; }
		if( phase == RESIZE ) { return SUCCESS; }
		x.b200_host_set( i, static_cast< DataType >( val ) );
		return SUCCESS;
	}

	/** x = y, values and sparsity (reference/io.hpp set(x, y)). */
	template< Descriptor descr = descriptors::no_operation, typename OutputType,
		typename InputType, typename Coords >
	RC set( Vector< OutputType, b200, Coords > &x, const Vector< InputType, b200, Coords > &y,
		const Phase &phase = EXECUTE
	) {
		using namespace internal::b200rt;
		if( size( x ) != size( y ) ) { return MISMATCH; }
		if( ( descr & descriptors::dense ) && ( nnz( y ) < size( y ) || nnz( x ) < size( x ) ) ) {
			return ILLEGAL;  // reference/io.hpp:698-702
		}
		if( phase == RESIZE ) { return SUCCESS; }
		const size_t n = size( x );
		if( n == 0 ) { return SUCCESS; }
		if( reinterpret_cast< const void * >( &x ) == reinterpret_cast< const void * >( &y ) ) {
			return ILLEGAL;
		}
		const int zt = type_code< OutputType >::value, yt = type_code< InputType >::value;
		if( zt < 0 || yt < 0 ) { return UNSUPPORTED; }
		x.b200_device_ready();
		y.b200_device_ready();
		// dense to dense: a step of the pending level-1 chain
		constexpr int dom = domain_of< OutputType, InputType >::value;
		if( x.b200_dense() && y.b200_dense() && fusion_enabled() && chain_type_ok( dom, zt ) &&
			chain_type_ok( dom, yt ) && record_step( ALPB_VEC_SET, ALPB_OP_RIGHT_ASSIGN,
				ALPB_OP_ADD, descr, dom, n, x.b200_values(), zt, y.b200_values(), yt, 0, nullptr, zt, 0 )
		) {
			return SUCCESS;
		}
		RC rc = clear( x );
		if( rc != SUCCESS ) { return rc; }
		rc = check( alpb_vec_op_dom( ALPB_VEC_SET, ALPB_OP_RIGHT_ASSIGN, 0, 0, 0, descr,
			domain_of< OutputType, InputType >::value, n,
			x.b200_values(), zt, x.b200_flags(), x.b200_counter(), nullptr, nullptr, ALPB_VOID, 0,
			y.b200_values(), yt, y.b200_flags_or_dense(), 0, nullptr, zt, nullptr, 0, stream() ),
			"set (vector)" );
		x.b200_refresh();
		return rc;
	}

	/** x = y where the mask allows it; x's other entries are removed
	 *  (reference/io.hpp:826-1000, masked set). */
	template< Descriptor descr = descriptors::no_operation, typename OutputType,
		typename MaskType, typename InputType, typename Coords >
	RC set( Vector< OutputType, b200, Coords > &x, const Vector< MaskType, b200, Coords > &mask,
		const Vector< InputType, b200, Coords > &y, const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< MaskType >::value && !grb::is_object< InputType >::value,
			void >::type * const = nullptr
	) {
		using namespace internal::b200rt;
		if( size( mask ) == 0 ) { return set< descr >( x, y, phase ); }
		if( size( x ) != size( y ) || size( x ) != size( mask ) ) { return MISMATCH; }
		if( ( descr & descriptors::dense ) && ( nnz( x ) < size( x ) || nnz( y ) < size( y ) ||
				nnz( mask ) < size( mask ) ) ) {
			return ILLEGAL;  // reference/io.hpp:865-871
		}
		if( phase == RESIZE ) { return SUCCESS; }
		const size_t n = size( x );
		const int zt = type_code< OutputType >::value, yt = type_code< InputType >::value,
			mt = type_code< MaskType >::value;
		if( zt < 0 || yt < 0 || mt < 0 ) { return UNSUPPORTED; }
		x.b200_device_ready();
		y.b200_device_ready();
		mask.b200_device_ready();
		// the output is replaced, not updated, unless the dense descriptor comes
		// with a structurally dense mask (reference/io.hpp:899-907)
		const bool mask_dense = ( descr & descriptors::structural ) &&
			!( descr & descriptors::invert_mask ) && nnz( mask ) == n;
		if( !( ( descr & descriptors::dense ) && mask_dense ) ) {
			const RC crc = clear( x );
			if( crc != SUCCESS ) { return crc; }
		}
		const RC rc = check( alpb_vec_op_dom( ALPB_VEC_SET, ALPB_OP_RIGHT_ASSIGN, 0, 0, 0, descr,
			domain_of< OutputType, InputType >::value, n,
			x.b200_values(), zt, x.b200_flags(), x.b200_counter(), mask.b200_values(),
			mask.b200_flags_or_dense(), mt, 1, y.b200_values(), yt, y.b200_flags_or_dense(), 0,
			nullptr, zt, nullptr, 0, stream() ), "set (masked vector)" );
		x.b200_refresh();
		return rc;
	}

	// --------------------------------------------------------- buildVector --
	template< Descriptor descr = descriptors::no_operation, typename InputType,
		typename fwd_iterator, typename Coords,
		class Dup = operators::right_assign< InputType > >
	RC buildVector( Vector< InputType, b200, Coords > &x, fwd_iterator start,
		const fwd_iterator end, const IOMode mode, const Dup &dup = Dup()
	) {
		(void) mode;
		const size_t n = size( x );
		x.b200_host_ready();
		InputType * const raw = x.raw();
		uint8_t * const fl = x.b200_flags();
		size_t i = 0;
		RC ret = SUCCESS;
		// an entry that exists already is folded with dup, or is an error under
		// no_duplicates (reference/vector.hpp:482-495)
		for( ; start != end && i < n; ++start, ++i ) {
			const InputType v = static_cast< InputType >( *start );
			if( fl[ i ] ) {
				if( descr & descriptors::no_duplicates ) { ret = ILLEGAL; break; }
				InputType out;
				(void) grb::apply( out, raw[ i ], v, dup );
				raw[ i ] = out;
			} else {
				raw[ i ] = v;
				fl[ i ] = 1;
			}
		}
		if( ret == SUCCESS && start != end ) { ret = MISMATCH; }
		// entries beyond the input keep their assigned state
		size_t cnt = 0;
		for( size_t k = 0; k < n; ++k ) { cnt += fl[ k ] ? 1 : 0; }
		*x.b200_counter() = static_cast< int64_t >( cnt );
		if( cnt == n ) { x.b200_mark_dense(); } else { x.b200_mark_sparse(); }
		return ret;
	}

	template< Descriptor descr = descriptors::no_operation, typename InputType,
		typename fwd_iterator1, typename fwd_iterator2, typename Coords,
		class Dup = operators::right_assign< InputType > >
	RC buildVector( Vector< InputType, b200, Coords > &x, fwd_iterator1 ind_start,
		const fwd_iterator1 ind_end, fwd_iterator2 val_start, const fwd_iterator2 val_end,
		const IOMode mode, const Dup &dup = Dup()
	) {
		(void) mode;
		const size_t n = size( x );
		x.b200_host_ready();
		InputType * const raw = x.raw();
		uint8_t * const fl = x.b200_flags();
		RC ret = SUCCESS;
		for( ; ind_start != ind_end && val_start != val_end; ++ind_start, ++val_start ) {
			const size_t i = static_cast< size_t >( *ind_start );
			if( i >= n ) { ret = MISMATCH; break; }
			const InputType v = static_cast< InputType >( *val_start );
			if( fl[ i ] ) {
				if( descr & descriptors::no_duplicates ) { ret = ILLEGAL; break; }
				InputType out;
				(void) grb::apply( out, raw[ i ], v, dup );
				raw[ i ] = out;
			} else {
				raw[ i ] = v;
				fl[ i ] = 1;
			}
		}
		size_t cnt = 0;
		for( size_t k = 0; k < n; ++k ) { cnt += fl[ k ] ? 1 : 0; }
		*x.b200_counter() = static_cast< int64_t >( cnt );
		if( cnt == n ) { x.b200_mark_dense(); } else { x.b200_mark_sparse(); }
		return ret;
	}

	// --------------------------------------------------- buildMatrixUnique --
	namespace internal {
		namespace b200rt {
			template< typename D >
			struct nz_value {
				template< typename It >
				static typename storage< D >::type get( const It &it ) {
					return static_cast< typename storage< D >::type >( it.v() );
				}
			};
			template<>
			struct nz_value< void > {
				template< typename It >
				static char get( const It & ) { return 0; }
			};
		}
	}

	/** Builds both orientations on the device from the host iterator; the
	 *  entries of a row keep the reference's order (reverse of the input,
	 *  reference/matrix.hpp:1921-1930).  Input must hold no duplicates. */
	template< Descriptor descr = descriptors::no_operation, typename InputType,
		typename RIT, typename CIT, typename NIT, typename fwd_iterator >
	RC buildMatrixUnique( Matrix< InputType, b200, RIT, CIT, NIT > &A, fwd_iterator start,
		const fwd_iterator end, const IOMode mode
	) {
		(void) mode;
		typedef typename Matrix< InputType, b200, RIT, CIT, NIT >::storage_type S;
		std::vector< uint32_t > I, J;
		std::vector< S > V;
		const size_t m = nrows( A ), n = ncols( A );
		for( ; start != end; ++start ) {
			const size_t i = static_cast< size_t >( start.i() ), j = static_cast< size_t >( start.j() );
			if( i >= m || j >= n ) { return MISMATCH; }
			I.push_back( static_cast< uint32_t >( i ) );
			J.push_back( static_cast< uint32_t >( j ) );
			V.push_back( internal::b200rt::nz_value< InputType >::get( start ) );
		}
		try {
			return A.b200_build( I, J, V );
		} catch( ... ) {
			return OUTOFMEM;
		}
	}

	// ---------------------------------------------------------------- wait --
	template<>
	inline RC wait< b200 >() { return internal::b200rt::check( alpb_stream_sync( nullptr ), "wait" ); }

	template< typename InputType, typename Coords, typename... Args >
	RC wait( const Vector< InputType, b200, Coords > &, const Args &... ) {
		return wait< b200 >();
	}

	template< typename InputType, typename RIT, typename CIT, typename NIT, typename... Args >
	RC wait( const Matrix< InputType, b200, RIT, CIT, NIT > &, const Args &... ) {
		return wait< b200 >();
	}

	/**
	 * A MatrixMarket coordinate file straight into a b200 matrix: an extension
	 * of the b200 backend with no counterpart in the reference, where a program
	 * reads the file through grb::utils::MatrixFileReader and passes its
	 * nonzero iterator to buildMatrixUnique (the text parsed and the storage
	 * built on one host core).  Here the file is parsed by every host core
	 * (alpb_mm_read), the triples go to the device in one copy, and the device
	 * builds both orientations -- the same matrix, nonzero for nonzero and in
	 * the same in-row order, as ALP's reader followed by buildMatrixUnique.
	 * Symmetric files are expanded as ALP's reader expands them; a pattern
	 * file's entries take the value one.  Value types: double, int, bool and
	 * void (pattern).  MISMATCH when the file's dimensions are not A's.
	 */
	template< typename D, typename RIT, typename CIT, typename NIT >
	RC buildMatrixUniqueFromFile( Matrix< D, b200, RIT, CIT, NIT > &A, const std::string &path ) {
		using namespace internal::b200rt;
		const int vt = type_code< D >::value;
		if( vt != ALPB_FP64 && vt != ALPB_INT32 && vt != ALPB_BOOL && vt != ALPB_VOID ) {
			return UNSUPPORTED;
		}
		int64_t m = 0, n = 0, nz = 0;
		uint32_t *I = nullptr, *J = nullptr;
		void *V = nullptr;
		RC rc = check( alpb_mm_read( path.c_str(), vt, &m, &n, &nz, &I, &J, &V, stream() ),
			"buildMatrixUniqueFromFile" );
		if( rc != SUCCESS ) { return rc; }
		if( size_t( m ) != A.b200_rows() || size_t( n ) != A.b200_cols() ) {
			rc = MISMATCH;
		} else {
			try {
				rc = A.b200_build_device( I, J,
					static_cast< const typename Matrix< D, b200, RIT, CIT, NIT >::storage_type * >( V ),
					static_cast< size_t >( nz ) );
			} catch( ... ) {
				rc = OUTOFMEM;
			}
		}
		release( I );
		release( J );
		release( V );
		return rc;
	}

}

#endif
