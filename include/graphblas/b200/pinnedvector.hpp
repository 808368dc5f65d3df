/*
 * PinnedVector of the b200 backend: a host copy of a vector's assigned
 * entries (reference: graphblas/reference/pinnedvector.hpp).
 */
#ifndef _H_GRB_B200_PINNEDVECTOR
#define _H_GRB_B200_PINNEDVECTOR

#include <cstddef>
#include <limits>
#include <vector>

#include <graphblas/base/pinnedvector.hpp>
#include <graphblas/b200/vector.hpp>

namespace grb {

	template< typename IOType >
	class PinnedVector< IOType, b200 > {

		private:

			size_t _n = 0;
			std::vector< IOType > _val;
			std::vector< size_t > _idx;

		public:

			PinnedVector() = default;

			template< typename Coord >
			PinnedVector( const Vector< IOType, b200, Coord > &x, const IOMode mode ) {
				(void) mode;
				_n = x.b200_size();
				for( const auto &p : x ) {
					_idx.push_back( p.first );
					_val.push_back( p.second );
				}
			}

			inline size_t size() const noexcept { return _n; }
			inline size_t nonzeroes() const noexcept { return _idx.size(); }

			template< typename OutputType >
			inline OutputType getNonzeroValue( const size_t k, const OutputType one = OutputType() ) const noexcept {
				(void) one;
				return static_cast< OutputType >( _val[ k ] );
			}
			inline IOType getNonzeroValue( const size_t k ) const noexcept { return _val[ k ]; }
			inline size_t getNonzeroIndex( const size_t k ) const noexcept {
				return k < _idx.size() ? _idx[ k ] : std::numeric_limits< size_t >::max();
			}
	};

}

#endif
