/*
 * grb::Matrix for the b200 backend (reference: graphblas/reference/matrix.hpp,
 * Matrix<D, reference, RIT, CIT, NIT> at :1018-2300).
 *
 * Like the reference, the matrix keeps BOTH orientations: a CRS for the
 * row gather (mxv) and a CCS for the column gather (vxm, transposed products,
 * adjoint solves), each in the reference's compressed-storage layout
 * (int64 offsets, uint32 indices, values of D, none for a pattern matrix) and
 * in device memory.  SpMV plans (schedule + merge-path tables) are made the
 * first time an orientation is multiplied and kept with the matrix.
 */
#ifndef _H_GRB_B200_MATRIX
#define _H_GRB_B200_MATRIX

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <type_traits>
#include <utility>
#include <vector>
#include <algorithm>

#include <graphblas/distribution.hpp>  // one process: ALP's base distribution
#include <graphblas/base/matrix.hpp>
#include <graphblas/b200/runtime.hpp>

namespace grb {

	namespace internal {

		namespace b200rt {

			/** One compressed orientation on the device. */
			template< typename S >
			struct Storage {
				int64_t * offsets = nullptr;
				uint32_t * indices = nullptr;
				S * values = nullptr;
				mutable alpb_spmv_plan plan = nullptr;

				void release_all() noexcept {
					if( plan ) { (void) alpb_spmv_plan_destroy( plan ); }
					release( offsets );
					release( indices );
					release( values );
					plan = nullptr;
					offsets = nullptr;
					indices = nullptr;
					values = nullptr;
				}
			};

			template< typename D >
			struct value_storage { typedef typename storage< D >::type type; };
			template<>
			struct value_storage< void > { typedef char type; };

		}

	}

	template< typename D, typename RIT, typename CIT, typename NIT >
	class Matrix< D, b200, RIT, CIT, NIT > {

		static_assert( sizeof( RIT ) <= 8 && sizeof( CIT ) <= 8,
			"row and column index types of at most 64 bits" );

		public:

			typedef D value_type;
			typedef typename internal::b200rt::value_storage< D >::type storage_type;
			typedef internal::b200rt::Storage< storage_type > storage_t;

		private:

			size_t _m = 0, _n = 0, _cap = 0, _nz = 0;
			storage_t _crs, _ccs;

			void init( const size_t m, const size_t n, const size_t cap ) {
				// a capacity above m * n cannot be used (reference/matrix.hpp:1462-1472 throws
				// ILLEGAL by name); the division form cannot overflow
				if( m > 0 && n > 0 && ( cap / m > n || ( cap / m == n && cap % m > 0 ) ) ) {
					throw std::runtime_error( toString( ILLEGAL ) );
				}
				// the device stores 32-bit row and column indices, whatever RIT/CIT
				if( m > 0xFFFFFFFFull || n > 0xFFFFFFFFull ) {
					throw std::runtime_error( "grb::Matrix< b200 >: dimensions beyond 32-bit indices" );
				}
				_m = m;
				_n = n;
				_cap = cap;
				_nz = 0;
				_crs.offsets = internal::b200rt::alloc< int64_t >( m + 1 );
				_ccs.offsets = internal::b200rt::alloc< int64_t >( n + 1 );
				(void) alpb_memset( _crs.offsets, 0, ( m + 1 ) * 8, internal::b200rt::stream() );
				(void) alpb_memset( _ccs.offsets, 0, ( n + 1 ) * 8, internal::b200rt::stream() );
				(void) alpb_stream_sync( internal::b200rt::stream() );
			}

			void move_from( Matrix &o ) noexcept {
				_m = o._m; _n = o._n; _cap = o._cap; _nz = o._nz;
				_crs = o._crs;
				_ccs = o._ccs;
				o._crs = storage_t();
				o._ccs = storage_t();
				o._m = o._n = o._cap = o._nz = 0;
			}

			static void copy_storage( storage_t &dst, const storage_t &src, const size_t outer,
				const size_t nz
			) {
				dst.offsets = internal::b200rt::alloc< int64_t >( outer + 1 );
				(void) alpb_memcpy_d2d( dst.offsets, src.offsets, ( outer + 1 ) * 8,
					internal::b200rt::stream() );
				if( nz > 0 ) {
					dst.indices = internal::b200rt::alloc< uint32_t >( nz );
					(void) alpb_memcpy_d2d( dst.indices, src.indices, nz * 4, internal::b200rt::stream() );
					if( internal::b200rt::type_code< D >::value != ALPB_VOID ) {
						dst.values = internal::b200rt::alloc< storage_type >( nz );
						(void) alpb_memcpy_d2d( dst.values, src.values, nz * sizeof( storage_type ),
							internal::b200rt::stream() );
					}
				}
			}

		public:

			Matrix( const size_t rows, const size_t columns, const size_t nz ) {
				init( rows, columns, nz );
			}

			/** Default capacity max( rows, columns ), as the reference's
			 *  (reference/matrix.hpp:2110-2116). */
			Matrix( const size_t rows, const size_t columns ) :
				Matrix( rows, columns, rows > columns ? rows : columns ) {}

			Matrix( const Matrix &o ) {
				_m = o._m; _n = o._n; _cap = o._cap; _nz = o._nz;
				copy_storage( _crs, o._crs, _m, _nz );
				copy_storage( _ccs, o._ccs, _n, _nz );
				(void) alpb_stream_sync( internal::b200rt::stream() );
			}

			Matrix( Matrix &&o ) noexcept { move_from( o ); }

			Matrix & operator=( Matrix &&o ) noexcept {
				if( this != &o ) {
					_crs.release_all();
					_ccs.release_all();
					move_from( o );
				}
				return *this;
			}

			~Matrix() {
				_crs.release_all();
				_ccs.release_all();
			}

			/** Const iterator over ((row, column), value) -- host copy of the CRS. */
			class const_iterator {
				private:
					std::vector< int64_t > _off;
					std::vector< uint32_t > _idx;
					std::vector< storage_type > _val;
					size_t _row = 0, _k = 0;
				public:
					// ((row, column), value); a pattern matrix yields (row, column), as
					// the reference's pattern iterator does
					typedef typename std::conditional< std::is_void< D >::value,
						std::pair< size_t, size_t >,
						std::pair< std::pair< size_t, size_t >,
							typename std::conditional< std::is_void< D >::value, char, D >::type > >::type
						value_type;
					// the start-end iterator interface of ALP's matrix iterators
					// (reference/compressed_storage.hpp: i(), j(), v() and their types)
					typedef RIT RowIndexType;
					typedef CIT ColumnIndexType;
					typedef D ValueType;
					const_iterator() = default;
					RowIndexType i() const { return static_cast< RowIndexType >( _row ); }
					ColumnIndexType j() const { return static_cast< ColumnIndexType >( _idx[ _k ] ); }
					template< typename DD = D >
					typename std::enable_if< !std::is_void< DD >::value, DD >::type v() const {
						return _val.empty() ? DD() : static_cast< DD >( _val[ _k ] );
					}
					const_iterator( const Matrix &A, const bool at_end ) {
						if( at_end ) { _k = A._nz; _row = A._m; return; }
						_off.resize( A._m + 1 );
						_idx.resize( A._nz );
						(void) alpb_memcpy_d2h( _off.data(), A._crs.offsets, ( A._m + 1 ) * 8,
							internal::b200rt::stream() );
						if( A._nz ) {
							(void) alpb_memcpy_d2h( _idx.data(), A._crs.indices, A._nz * 4,
								internal::b200rt::stream() );
							if( A._crs.values ) {
								_val.resize( A._nz );
								(void) alpb_memcpy_d2h( _val.data(), A._crs.values,
									A._nz * sizeof( storage_type ), internal::b200rt::stream() );
							}
						}
						(void) alpb_stream_sync( internal::b200rt::stream() );
						while( _row < A._m && _off[ _row + 1 ] <= static_cast< int64_t >( _k ) ) { ++_row; }
					}
					bool operator!=( const const_iterator &o ) const { return _k != o._k; }
					bool operator==( const const_iterator &o ) const { return _k == o._k; }
					const_iterator & operator++() {
						++_k;
						while( _row + 1 < _off.size() && _off[ _row + 1 ] <= static_cast< int64_t >( _k ) ) {
							++_row;
						}
						return *this;
					}
					value_type operator*() const {
						return entry( std::integral_constant< bool, std::is_void< D >::value >() );
					}
					value_type entry( std::true_type ) const {
						return value_type( _row, static_cast< size_t >( _idx[ _k ] ) );
					}
					value_type entry( std::false_type ) const {
						return value_type( std::make_pair( _row, static_cast< size_t >( _idx[ _k ] ) ),
							_val.empty() ? value_type().second : static_cast< D >( _val[ _k ] ) );
					}
					// it->first / it->second on the entry by value (a proxy holds it)
					struct arrow {
						value_type v;
						const value_type * operator->() const { return &v; }
					};
					arrow operator->() const { return arrow{ **this }; }
			};

			const_iterator cbegin() const { return const_iterator( *this, false ); }
			const_iterator cend() const { return const_iterator( *this, true ); }
			const_iterator begin() const { return cbegin(); }
			const_iterator end() const { return cend(); }

			// ---- backend-internal access ----
			/** This matrix becomes A: both orientations copied on the device, A's
			 *  values cast to D (reference/io.hpp set( Matrix, Matrix ), execute
			 *  phase of internal::set_copy, :1520-1548); a pattern (void) target
			 *  keeps the structure only.  Values cannot come from a pattern A
			 *  (UNSUPPORTED).  As in the reference: nothing happens for an empty
			 *  dimension, an A without nonzeroes clears this matrix, and an A with
			 *  more nonzeroes than this matrix's capacity clears it and returns
			 *  ILLEGAL (only the RESIZE phase reserves).  A failed device copy also
			 *  leaves this matrix cleared, with the error returned. */
			template< typename D2, typename R2, typename C2, typename N2 >
			RC b200_assign_from( const Matrix< D2, b200, R2, C2, N2 > &A ) {
				using namespace internal::b200rt;
				const int dt = type_code< D >::value, st = type_code< D2 >::value;
				if( dt < 0 || st < 0 || ( dt != ALPB_VOID && st == ALPB_VOID ) ) { return UNSUPPORTED; }
				const size_t m = A.b200_rows(), n = A.b200_cols(), nz = A.b200_nnz();
				if( m == 0 || n == 0 ) { return SUCCESS; }
				if( nz == 0 ) {
					b200_clear();
					return SUCCESS;
				}
				if( nz > _cap ) {
					b200_clear();
					return ILLEGAL;
				}
				_crs.release_all();
				_ccs.release_all();
				init( m, n, _cap );
				RC rc = SUCCESS;
				const auto keep = [&]( const RC r ) { if( rc == SUCCESS ) { rc = r; } };
				const auto one = [&]( storage_t &dst, const typename Matrix< D2, b200, R2, C2, N2 >::storage_t
					&src, const size_t outer ) {
					keep( check( alpb_memcpy_d2d( dst.offsets, src.offsets, ( outer + 1 ) * 8, stream() ),
						"set (matrix offsets)" ) );
					dst.indices = alloc< uint32_t >( nz );
					keep( check( alpb_memcpy_d2d( dst.indices, src.indices, nz * 4, stream() ),
						"set (matrix indices)" ) );
					if( dt == ALPB_VOID ) { return; }
					dst.values = alloc< storage_type >( nz );
					keep( check( alpb_vec_op_dom( ALPB_VEC_SET, ALPB_OP_RIGHT_ASSIGN, 0, 0, 0, 0,
						domain_of< D, D2 >::value, static_cast< int64_t >( nz ), dst.values, dt, nullptr,
						nullptr, nullptr, nullptr, ALPB_VOID, 0, src.values, st, nullptr, 0, nullptr, st,
						nullptr, 0, stream() ), "set (matrix values)" ) );
				};
				one( _crs, A.b200_crs(), m );
				one( _ccs, A.b200_ccs(), n );
				keep( check( alpb_stream_sync( stream() ), "set (matrix)" ) );
				if( rc != SUCCESS ) {
					b200_clear();
					return rc;
				}
				_nz = nz;
				return SUCCESS;
			}

			size_t b200_rows() const noexcept { return _m; }
			size_t b200_cols() const noexcept { return _n; }
			size_t b200_nnz() const noexcept { return _nz; }
			size_t b200_capacity() const noexcept { return _cap; }
			const storage_t & b200_crs() const noexcept { return _crs; }
			const storage_t & b200_ccs() const noexcept { return _ccs; }

			/** Plan of one orientation, made on first use. */
			alpb_spmv_plan b200_plan( const bool rows ) const {
				const storage_t &s = rows ? _crs : _ccs;
				if( !s.plan && _nz > 0 ) {
					(void) alpb_spmv_plan_create( &s.plan, static_cast< int64_t >( rows ? _m : _n ),
						static_cast< int64_t >( _nz ), s.offsets, ALPB_SCHED_AUTO, 0,
						internal::b200rt::stream() );
				}
				return s.plan;
			}

			void b200_clear() {
				_crs.release_all();
				_ccs.release_all();
				const size_t m = _m, n = _n, cap = _cap;
				init( m, n, cap );
			}

			void b200_reserve( const size_t cap ) { if( cap > _cap ) { _cap = cap; } }

			/** Runs f( i, j, v ) on the host for every stored entry, in CRS order,
			 *  and writes the (possibly changed) values back to both orientations.
			 *  Host lambdas cannot run on the device; this is the matrix form of
			 *  eWiseLambda (reference/blas2.hpp, eWiseLambda over a matrix). */
			template< class F >
			RC b200_host_lambda( F &f ) {
				using namespace internal::b200rt;
				if( _nz == 0 ) { return SUCCESS; }
				if( !_crs.values || !_ccs.values ) { return UNSUPPORTED; }
				std::vector< int64_t > ro( _m + 1 ), co( _n + 1 );
				std::vector< uint32_t > ri( _nz ), ci( _nz );
				std::vector< storage_type > rv( _nz ), cv( _nz );
				(void) alpb_memcpy_d2h( ro.data(), _crs.offsets, ( _m + 1 ) * 8, stream() );
				(void) alpb_memcpy_d2h( ri.data(), _crs.indices, _nz * 4, stream() );
				(void) alpb_memcpy_d2h( rv.data(), _crs.values, _nz * sizeof( storage_type ), stream() );
				(void) alpb_memcpy_d2h( co.data(), _ccs.offsets, ( _n + 1 ) * 8, stream() );
				(void) alpb_memcpy_d2h( ci.data(), _ccs.indices, _nz * 4, stream() );
				RC rc = check( alpb_stream_sync( stream() ), "eWiseLambda (matrix)" );
				if( rc != SUCCESS ) { return rc; }
				for( size_t i = 0; i < _m; ++i ) {
					for( int64_t k = ro[ i ]; k < ro[ i + 1 ]; ++k ) {
						D v = static_cast< D >( rv[ k ] );
						f( i, static_cast< size_t >( ri[ k ] ), v );
						rv[ k ] = static_cast< storage_type >( v );
					}
				}
				// the CCS holds the same entries: find each (j, i) in row i of the CRS
				std::vector< std::pair< uint32_t, int64_t > > byrow( _nz );
				for( size_t i = 0; i < _m; ++i ) {
					for( int64_t k = ro[ i ]; k < ro[ i + 1 ]; ++k ) { byrow[ k ] = { ri[ k ], k }; }
					std::sort( byrow.begin() + ro[ i ], byrow.begin() + ro[ i + 1 ] );
				}
				for( size_t j = 0; j < _n; ++j ) {
					for( int64_t kk = co[ j ]; kk < co[ j + 1 ]; ++kk ) {
						const uint32_t i = ci[ kk ];
						const auto first = byrow.begin() + ro[ i ], last = byrow.begin() + ro[ i + 1 ];
						const auto it = std::lower_bound( first, last,
							std::make_pair( static_cast< uint32_t >( j ), int64_t( -1 ) ) );
						if( it == last || it->first != j ) { return PANIC; }
						cv[ kk ] = rv[ it->second ];
					}
				}
				(void) alpb_memcpy_h2d( _crs.values, rv.data(), _nz * sizeof( storage_type ), stream() );
				(void) alpb_memcpy_h2d( _ccs.values, cv.data(), _nz * sizeof( storage_type ), stream() );
				return check( alpb_stream_sync( stream() ), "eWiseLambda (matrix)" );
			}

			/** Replace the contents by the (I, J, V) triples, in input order: both
			 *  orientations are built on the device with the reference's in-row
			 *  order (alpb_coo_to_crs). */
			/** Both orientations from a host CRS kept in its given in-row order
			 *  (the CCS by a stable device transpose). */
			RC b200_set_crs( const std::vector< int64_t > &off, const std::vector< uint32_t > &col,
				const std::vector< storage_type > &val
			) {
				using namespace internal::b200rt;
				const size_t nz = col.size();
				const int vt = type_code< D >::value;
				if( vt < 0 ) { return UNSUPPORTED; }
				if( off.size() != _m + 1 ) { return MISMATCH; }
				_crs.release_all();
				_ccs.release_all();
				init( _m, _n, nz > _cap ? nz : _cap );
				(void) alpb_memcpy_h2d( _crs.offsets, off.data(), ( _m + 1 ) * 8, stream() );
				if( nz > 0 ) {
					_crs.indices = alloc< uint32_t >( nz );
					_ccs.indices = alloc< uint32_t >( nz );
					(void) alpb_memcpy_h2d( _crs.indices, col.data(), nz * 4, stream() );
					if( vt != ALPB_VOID ) {
						_crs.values = alloc< storage_type >( nz );
						_ccs.values = alloc< storage_type >( nz );
						(void) alpb_memcpy_h2d( _crs.values, val.data(), nz * sizeof( storage_type ),
							stream() );
					}
				}
				const RC rc = nz == 0 ? SUCCESS : check( alpb_crs_transpose( _m, _n, nz, _crs.offsets,
					_crs.indices, _crs.values, vt, _ccs.offsets, _ccs.indices, _ccs.values, stream() ),
					"wrapCRSMatrix (CCS)" );
				(void) alpb_stream_sync( stream() );
				if( rc == SUCCESS ) { _nz = nz; }
				return rc;
			}

			RC b200_build( const std::vector< uint32_t > &I, const std::vector< uint32_t > &J,
				const std::vector< storage_type > &V
			) {
				using namespace internal::b200rt;
				const size_t nz = I.size();
				const int vt = type_code< D >::value;
				if( vt < 0 ) { return UNSUPPORTED; }
				if( nz == 0 ) { return b200_build_device( nullptr, nullptr, nullptr, 0 ); }
				uint32_t * dI = alloc< uint32_t >( nz );
				uint32_t * dJ = alloc< uint32_t >( nz );
				storage_type * dV = vt == ALPB_VOID ? nullptr : alloc< storage_type >( nz );
				(void) alpb_memcpy_h2d( dI, I.data(), nz * 4, stream() );
				(void) alpb_memcpy_h2d( dJ, J.data(), nz * 4, stream() );
				if( dV ) { (void) alpb_memcpy_h2d( dV, V.data(), nz * sizeof( storage_type ), stream() ); }
				const RC rc = b200_build_device( dI, dJ, dV, nz );
				release( dI );
				release( dJ );
				release( dV );
				return rc;
			}

			/** Both orientations from device triples (I, J, V: nz entries, V of
			 *  this matrix's storage type or null for a pattern), in the
			 *  reference's in-row order; the triples stay the caller's. */
			RC b200_build_device( const uint32_t * const dI, const uint32_t * const dJ,
				const storage_type * const dV, const size_t nz
			) {
				using namespace internal::b200rt;
				const int vt = type_code< D >::value;
				if( vt < 0 ) { return UNSUPPORTED; }
				_crs.release_all();
				_ccs.release_all();
				init( _m, _n, nz > _cap ? nz : _cap );
				if( nz == 0 ) { return SUCCESS; }
				_crs.indices = alloc< uint32_t >( nz );
				_ccs.indices = alloc< uint32_t >( nz );
				if( dV ) {
					_crs.values = alloc< storage_type >( nz );
					_ccs.values = alloc< storage_type >( nz );
				}
				RC rc = check( alpb_coo_to_crs( _m, _n, nz, dI, dJ, dV, vt, _crs.offsets, _crs.indices,
					_crs.values, stream() ), "buildMatrixUnique (CRS)" );
				if( rc == SUCCESS ) {
					rc = check( alpb_coo_to_crs( _n, _m, nz, dJ, dI, dV, vt, _ccs.offsets, _ccs.indices,
						_ccs.values, stream() ), "buildMatrixUnique (CCS)" );
				}
				(void) alpb_stream_sync( stream() );
				if( rc == SUCCESS ) { _nz = nz; }
				return rc;
			}
	};


	namespace internal {

		/**
		 * A b200 matrix holding a copy of the host CRS (value_array,
		 * index_array, offst_array) of an m x n matrix, in the given in-row
		 * order; the CCS is built on the device.  Serves
		 * internal::wrapCRSMatrix (reference/matrix.hpp:65-88), whose reference
		 * form views the caller's arrays: the device cannot, so the b200 form
		 * copies them (the transition API, src/transition/solver.cpp:169,
		 * keeps the arrays unchanged while its handle lives).  Throws when the
		 * value type has no device storage.
		 */
		template<
			typename ValType, typename ColType, typename IndType,
			Backend backend = config::default_backend
		>
		const grb::Matrix< ValType, backend, ColType, ColType, IndType > wrapCRSMatrix(
			const ValType *__restrict__ const value_array,
			const ColType *__restrict__ const index_array,
			const IndType *__restrict__ const offst_array,
			const size_t m, const size_t n
		) {
			static_assert( backend == b200, "the b200 form of wrapCRSMatrix" );
			using namespace internal::b200rt;
			typedef grb::Matrix< ValType, backend, ColType, ColType, IndType > M;
			typedef typename M::storage_type S;
			const int vt = type_code< ValType >::value;
			if( vt < 0 ) {
				throw std::runtime_error( "grb::internal::wrapCRSMatrix< b200 >: value type "
					"without device storage" );
			}
			const size_t nz = static_cast< size_t >( offst_array[ m ] );
			M A( m, n, nz );
			std::vector< int64_t > off( m + 1 );
			for( size_t i = 0; i <= m; ++i ) { off[ i ] = static_cast< int64_t >( offst_array[ i ] ); }
			std::vector< uint32_t > col( nz );
			for( size_t k = 0; k < nz; ++k ) {
				if( static_cast< size_t >( index_array[ k ] ) >= n ) {
					throw std::runtime_error( "grb::internal::wrapCRSMatrix< b200 >: column index "
						"out of range" );
				}
				col[ k ] = static_cast< uint32_t >( index_array[ k ] );
			}
			std::vector< S > val( vt == ALPB_VOID ? 0 : nz );
			for( size_t k = 0; k < val.size(); ++k ) { val[ k ] = static_cast< S >( value_array[ k ] ); }
			const RC rc = A.b200_set_crs( off, col, val );
			if( rc != SUCCESS ) {
				throw std::runtime_error( "grb::internal::wrapCRSMatrix< b200 >: device build failed" );
			}
			return A;
		}

		/** Storage accessors under the names ALP's utilities use for the
		 *  reference backend; a b200 matrix keeps both orientations on the
		 *  device, so these give the device-side descriptors. */
		template< typename D, typename RIT, typename CIT, typename NIT >
		auto getCRS( const Matrix< D, b200, RIT, CIT, NIT > &A ) noexcept
			-> decltype( A.b200_crs() )
		{
			return A.b200_crs();
		}

		template< typename D, typename RIT, typename CIT, typename NIT >
		auto getCCS( const Matrix< D, b200, RIT, CIT, NIT > &A ) noexcept
			-> decltype( A.b200_ccs() )
		{
			return A.b200_ccs();
		}

	}

}

#endif
