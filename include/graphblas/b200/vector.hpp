/*
 * grb::Vector for the b200 backend (reference: graphblas/reference/vector.hpp,
 * Vector<D, reference, C> at :280-1400).
 *
 * Values and assigned flags live in CUDA managed memory: the kernels of
 * libalp_b200.so read and write them on the device, while ALP's host-side
 * accessors (raw(), operator[], iterators, eWiseLambda, PinnedVector) read
 * the same pointers after the primitive has synchronised -- execution is
 * blocking, as the reference's (Properties<b200>::isBlockingExecution).  A
 * host-side write marks the vector so that the next device primitive first
 * prefetches it back to the GPU.
 *
 * A device counter holds the number of assigned entries; `dense` caches on
 * the host that all entries are assigned, which lets the kernels skip the
 * flags (they are kept valid either way).
 */
#ifndef _H_GRB_B200_VECTOR
#define _H_GRB_B200_VECTOR

#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <iterator>
#include <stdexcept>
#include <utility>

#include <graphblas/base/vector.hpp>
#include <graphblas/b200/coordinates.hpp>
#include <graphblas/b200/runtime.hpp>

namespace grb {

	template< typename D, typename MyCoordinates >
	class Vector< D, b200, MyCoordinates > {

		public:

			typedef D value_type;
			typedef D & lambda_reference;
			typedef typename internal::b200rt::storage< D >::type storage_type;

		private:

			size_t _n = 0;
			storage_type * _val = nullptr;   // managed [n]
			uint8_t * _flags = nullptr;      // managed [n]
			int64_t * _count = nullptr;      // managed [1]
			bool _dense = false;
			mutable bool _host_touched = false;
			D * _wrap_back = nullptr;        // caller's array a wrapped vector writes back to

			void allocate( const size_t n ) {
				_n = n;
				if( n == 0 ) { return; }
				void * p = nullptr;
				if( alpb_malloc_managed( &p, n * sizeof( storage_type ) ) != ALPB_SUCCESS ) {
					throw std::runtime_error( std::string( "grb::Vector< b200 >: " ) + alpb_last_error() );
				}
				_val = static_cast< storage_type * >( p );
				if( alpb_malloc_managed( &p, n ) != ALPB_SUCCESS ) {
					throw std::runtime_error( std::string( "grb::Vector< b200 >: " ) + alpb_last_error() );
				}
				_flags = static_cast< uint8_t * >( p );
				if( alpb_malloc_managed( &p, sizeof( int64_t ) ) != ALPB_SUCCESS ) {
					throw std::runtime_error( std::string( "grb::Vector< b200 >: " ) + alpb_last_error() );
				}
				_count = static_cast< int64_t * >( p );
				(void) alpb_memset( _flags, 0, n, internal::b200rt::stream() );
				(void) alpb_memset( _count, 0, sizeof( int64_t ), internal::b200rt::stream() );
				(void) alpb_stream_sync( internal::b200rt::stream() );
			}

			void free_all() noexcept {
				if( _wrap_back && _n > 0 ) {   // a wrapped caller array gets the final values
					b200_host_ready();
					for( size_t i = 0; i < _n; ++i ) { _wrap_back[ i ] = static_cast< D >( _val[ i ] ); }
				}
				_wrap_back = nullptr;
				internal::b200rt::release( _val );
				internal::b200rt::release( _flags );
				internal::b200rt::release( _count );
				_val = nullptr;
				_flags = nullptr;
				_count = nullptr;
				_n = 0;
				_dense = false;
			}

			void copy_from( const Vector &o ) {
				allocate( o._n );
				if( _n > 0 ) {
					o.b200_device_ready();
					(void) alpb_memcpy_d2d( _val, o._val, _n * sizeof( storage_type ), internal::b200rt::stream() );
					(void) alpb_memcpy_d2d( _flags, o._flags, _n, internal::b200rt::stream() );
					(void) alpb_memcpy_d2d( _count, o._count, sizeof( int64_t ), internal::b200rt::stream() );
					(void) alpb_stream_sync( internal::b200rt::stream() );
				}
				_dense = o._dense;
			}

		public:

			/** Const iterator over the assigned entries, as (index, value) pairs. */
			class const_iterator {
				private:
					const Vector * _v = nullptr;
					size_t _i = 0;
					void skip() { while( _v && _i < _v->_n && !_v->_flags[ _i ] ) { ++_i; } }
				public:
					typedef std::pair< const size_t, const D > value_type;
					typedef const value_type * pointer;
					typedef value_type reference;
					typedef std::forward_iterator_tag iterator_category;
					typedef std::ptrdiff_t difference_type;
					const_iterator() = default;
					const_iterator( const Vector * v, const size_t i ) : _v( v ), _i( i ) { skip(); }
					bool operator==( const const_iterator &o ) const { return _i == o._i; }
					bool operator!=( const const_iterator &o ) const { return _i != o._i; }
					value_type operator*() const {
						return value_type( _i, static_cast< D >( _v->_val[ _i ] ) );
					}
					/** it->first, it->second on the (index, value) pair, held by value */
					struct arrow {
						value_type v;
						const value_type * operator->() const { return &v; }
					};
					arrow operator->() const { return arrow{ **this }; }
					const_iterator & operator++() { ++_i; skip(); return *this; }
			};

			/** A capacity above the size is refused as the reference refuses it
			 *  (reference/vector.hpp:365-371: ILLEGAL thrown by name). */
			Vector( const size_t n, const size_t nz ) {
				if( nz > n ) { throw std::runtime_error( toString( ILLEGAL ) ); }
				allocate( n );
			}

			Vector( const size_t n ) { allocate( n ); }

			Vector() : Vector( 0 ) {}

			Vector( const std::initializer_list< D > vals ) {
				allocate( vals.size() );
				size_t i = 0;
				for( const D &v : vals ) {
					_val[ i ] = static_cast< storage_type >( v );
					_flags[ i ] = 1;
					++i;
				}
				*_count = static_cast< int64_t >( _n );
				_dense = true;
				_host_touched = true;
			}

			Vector( const Vector &o ) { copy_from( o ); }

			Vector( Vector &&o ) noexcept { *this = std::move( o ); }

			Vector & operator=( const Vector &o ) {
				if( this != &o ) {
					free_all();
					copy_from( o );
				}
				return *this;
			}

			Vector & operator=( Vector &&o ) noexcept {
				if( this != &o ) {
					free_all();
					_n = o._n;
					_val = o._val;
					_flags = o._flags;
					_count = o._count;
					_dense = o._dense;
					_host_touched = o._host_touched;
					_wrap_back = o._wrap_back;
					o._val = nullptr;
					o._flags = nullptr;
					o._count = nullptr;
					o._wrap_back = nullptr;
					o._n = 0;
					o._dense = false;
				}
				return *this;
			}

			~Vector() { free_all(); }

			const_iterator cbegin() const { b200_host_ready(); return const_iterator( this, 0 ); }
			const_iterator cend() const { return const_iterator( this, _n ); }
			const_iterator begin() const { return cbegin(); }
			const_iterator end() const { return cend(); }

			/** Host pointer to the values (managed memory), valid after the last
			 *  primitive returned; host writes are seen by the next primitive. */
			D * raw() const {
				b200_host_ready();
				_host_touched = true;
				return reinterpret_cast< D * >( _val );
			}

			lambda_reference operator[]( const size_t i ) {
				if( internal::b200rt::chain().nsteps ) { b200_host_ready(); }  // fused steps pending
				_host_touched = true;
				return reinterpret_cast< D * >( _val )[ i ];
			}
			lambda_reference operator[]( const size_t i ) const {
				if( internal::b200rt::chain().nsteps ) { b200_host_ready(); }
				_host_touched = true;
				return reinterpret_cast< D * >( _val )[ i ];
			}

			// ---- backend-internal access (used by the b200 primitives) ----
			size_t b200_size() const noexcept { return _n; }
			storage_type * b200_values() const noexcept { return _val; }
			uint8_t * b200_flags() const noexcept { return _flags; }
			/** flags to hand to a kernel: NULL when every entry is assigned */
			uint8_t * b200_flags_or_dense() const noexcept { return _dense ? nullptr : _flags; }
			int64_t * b200_counter() const noexcept { return _count; }
			bool b200_dense() const noexcept { return _dense; }

			/** Number of assigned entries (reads the device counter). */
			size_t b200_nnz() const {
				if( _dense ) { return _n; }
				if( _n == 0 ) { return 0; }
				(void) alpb_stream_sync( internal::b200rt::stream() );
				return static_cast< size_t >( *_count );
			}

			/** After a primitive that may have assigned entries: refresh `dense`. */
			void b200_refresh() {
				if( !_dense && _n > 0 ) {
					(void) alpb_stream_sync( internal::b200rt::stream() );
					_dense = static_cast< size_t >( *_count ) == _n;
				}
			}

			/** Every entry assigned (the caller has set all flags and the counter). */
			void b200_mark_dense() noexcept { _dense = _n > 0; }
			void b200_mark_sparse() noexcept { _dense = false; }

			/** Before a kernel touches this vector: move host-written pages back. */
			void b200_device_ready() const {
				if( _host_touched && _n > 0 ) {
					(void) alpb_prefetch( _val, _n * sizeof( storage_type ), 1, internal::b200rt::stream() );
					(void) alpb_prefetch( _flags, _n, 1, internal::b200rt::stream() );
					_host_touched = false;
				}
			}

			/** Before the host reads this vector. */
			void b200_host_ready() const { (void) alpb_stream_sync( internal::b200rt::stream() ); }

			/** Every entry from a host array (managed memory: written in place). */
			void b200_load_host( const D * const src ) {
				b200_host_ready();
				for( size_t i = 0; i < _n; ++i ) {
					_val[ i ] = static_cast< storage_type >( src[ i ] );
					_flags[ i ] = 1;
				}
				if( _n > 0 ) { *_count = static_cast< int64_t >( _n ); }
				_dense = _n > 0;
				_host_touched = true;
			}

			/** Copy the final values back to `dst` when this vector is destroyed. */
			void b200_write_back_to( D * const dst ) noexcept { _wrap_back = dst; }

			/** Host-side single-entry update (setElement). */
			void b200_host_set( const size_t i, const D &v ) {
				b200_host_ready();
				_val[ i ] = static_cast< storage_type >( v );
				if( !_flags[ i ] ) {
					_flags[ i ] = 1;
					*_count += 1;
					_dense = static_cast< size_t >( *_count ) == _n;
				}
				_host_touched = true;
			}
	};

	namespace internal {

		/** Host pointer to a vector's values (reference/vector.hpp:117-121):
		 *  managed memory, valid once the device work before it finished; host
		 *  writes are moved back before the next primitive. */
		template< typename D, typename C >
		inline D * getRaw( Vector< D, b200, C > &x ) noexcept { return x.raw(); }

		template< typename D, typename C >
		inline const D * getRaw( const Vector< D, b200, C > &x ) noexcept { return x.raw(); }

		/**
		 * A dense b200 vector over the caller's host array
		 * (reference/vector.hpp:150-180).  The reference form uses the array as
		 * its storage; the device cannot, so the b200 form copies it in and,
		 * for a non-const array, copies the final values back when the vector
		 * is destroyed (so a solver's result lands in the caller's array, as in
		 * sparse_cg_solve, src/transition/solver.cpp:770-780).
		 */
		template< typename D, Backend backend = config::default_backend >
		grb::Vector< D, backend, internal::Coordinates<
			config::IMPLEMENTATION< backend >::coordinatesBackend() > >
		wrapRawVector( const size_t n, D *__restrict__ const raw ) {
			static_assert( backend == b200, "the b200 form of wrapRawVector" );
			grb::Vector< D, backend, internal::Coordinates<
				config::IMPLEMENTATION< backend >::coordinatesBackend() > > v( n );
			v.b200_load_host( raw );
			v.b200_write_back_to( raw );
			return v;
		}

		template< typename D, Backend backend = config::default_backend >
		const grb::Vector< D, backend, internal::Coordinates<
			config::IMPLEMENTATION< backend >::coordinatesBackend() > >
		wrapRawVector( const size_t n, const D *__restrict__ const raw ) {
			static_assert( backend == b200, "the b200 form of wrapRawVector" );
			grb::Vector< D, backend, internal::Coordinates<
				config::IMPLEMENTATION< backend >::coordinatesBackend() > > v( n );
			v.b200_load_host( raw );
			return v;
		}

		/** Device size helper used by the b200 primitives. */
		template< typename D, typename C >
		inline size_t b200_nnz( const Vector< D, b200, C > &x ) { return x.b200_nnz(); }

	}

}

#endif
