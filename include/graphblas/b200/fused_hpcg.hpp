/*
 * The b200 overload of grb::algorithms::hpcg (fused device HPCG).
 * See graphblas/b200/fused_algorithms.hpp for when the fused path is taken.
 */
#ifndef _H_GRB_B200_FUSED_HPCG
#define _H_GRB_B200_FUSED_HPCG

#include <algorithm>
#include <cstdint>
#include <vector>

#include <graphblas/b200/fused_algorithms.hpp>

namespace grb {

	namespace algorithms {

		namespace internal_b200_fused {

			/** Device HPCG handles made for recognised systems, kept for the
			 *  process (a solve is usually repeated on one system); the oldest is
			 *  released beyond four. */
			struct HpcgKey {
				int64_t nx, ny, nz, colors, levels;
				double diag, off;
				alpb_hpcg h;
			};

			inline std::vector< HpcgKey > & hpcg_handles() {
				static std::vector< HpcgKey > handles;
				return handles;
			}

			/** One level of the caller's data against level l of h. */
			template< typename SysData >
			bool hpcg_level_matches( alpb_hpcg h, const int64_t l, const SysData &sys,
				const Matrix< double, b200 > * const coarsening, const int64_t fine_n
			) {
				using namespace grb::internal::b200rt;
				int64_t ln = 0, lnnz = 0;
				if( alpb_hpcg_matrix( h, l, nullptr, nullptr, nullptr, &ln, &lnnz ) != ALPB_SUCCESS ) {
					return false;
				}
				const Matrix< double, b200 > &A = sys.A;
				if( A.b200_rows() != size_t( ln ) || A.b200_cols() != size_t( ln ) ||
					A.b200_nnz() != size_t( lnnz ) || sys.A_diagonal.b200_size() != size_t( ln )
				) {
					return false;
				}
				std::vector< const uint8_t * > mv, mf;
				for( const auto &mask : sys.color_masks ) {
					if( mask.b200_size() != size_t( ln ) ) { return false; }
					mask.b200_device_ready();
					mv.push_back( reinterpret_cast< const uint8_t * >( mask.b200_values() ) );
					mf.push_back( mask.b200_flags_or_dense() );
				}
				int64_t cnnz = 0;
				const int64_t *co = nullptr;
				const uint32_t *ci = nullptr;
				const double *cv = nullptr;
				if( l > 0 ) {
					if( coarsening == nullptr || coarsening->b200_rows() != size_t( ln ) ||
						coarsening->b200_cols() != size_t( fine_n )
					) {
						return false;
					}
					cnnz = static_cast< int64_t >( coarsening->b200_nnz() );
					co = coarsening->b200_crs().offsets;
					ci = coarsening->b200_crs().indices;
					cv = reinterpret_cast< const double * >( coarsening->b200_crs().values );
				}
				sys.A_diagonal.b200_device_ready();
				int ok = 0;
				const int rc = alpb_hpcg_match_level( h, l, ln, lnnz, A.b200_crs().offsets,
					A.b200_crs().indices, reinterpret_cast< const double * >( A.b200_crs().values ),
					reinterpret_cast< const double * >( sys.A_diagonal.b200_values() ),
					sys.A_diagonal.b200_flags_or_dense(), static_cast< int64_t >( mv.size() ),
					mv.data(), mf.data(), cnnz, co, ci, cv, &ok, stream() );
				return rc == ALPB_SUCCESS && ok == 1;
			}

			/**
			 * A device HPCG handle that solves \a data's system, or nullptr.  The
			 * system is recognised as build_hpcg_system's (3-D 27-point box
			 * stencil, hpcg/system_building_utils.hpp:84-150): the grid sizes and
			 * the two values are read off row 0 (its eight stored columns are
			 * 0, 1, nx, nx+1, nx ny, nx ny+1, nx ny+nx, nx ny+nx+1), then every
			 * level -- matrix, diagonal, colour masks, coarsening -- is compared
			 * on the device with the handle's (alpb_hpcg_match_level).
			 */
			inline alpb_hpcg recognise_hpcg( const hpcg_data< double, double, double > &data ) {
				using namespace grb::internal::b200rt;
				const Matrix< double, b200 > &A = data.A;
				const size_t n = A.b200_rows();
				if( n < 8 || A.b200_cols() != n || A.b200_nnz() == 0 ) { return nullptr; }
				int64_t off01[ 2 ] = { 0, 0 };
				if( alpb_memcpy_d2h( off01, A.b200_crs().offsets, 16, stream() ) != ALPB_SUCCESS ||
					alpb_stream_sync( stream() ) != ALPB_SUCCESS || off01[ 0 ] != 0 || off01[ 1 ] != 8
				) {
					return nullptr;
				}
				uint32_t cols[ 8 ];
				double vals[ 8 ];
				if( alpb_memcpy_d2h( cols, A.b200_crs().indices, sizeof( cols ), stream() ) !=
						ALPB_SUCCESS ||
					alpb_memcpy_d2h( vals, A.b200_crs().values, sizeof( vals ), stream() ) !=
						ALPB_SUCCESS ||
					alpb_stream_sync( stream() ) != ALPB_SUCCESS
				) {
					return nullptr;
				}
				std::vector< std::pair< uint32_t, double > > row0;
				for( int k = 0; k < 8; ++k ) { row0.emplace_back( cols[ k ], vals[ k ] ); }
				std::sort( row0.begin(), row0.end() );
				const int64_t nx = row0[ 2 ].first, nxny = row0[ 4 ].first;
				const int64_t want[ 8 ] = { 0, 1, nx, nx + 1, nxny, nxny + 1, nxny + nx, nxny + nx + 1 };
				for( int k = 0; k < 8; ++k ) {
					if( int64_t( row0[ k ].first ) != want[ k ] ) { return nullptr; }
				}
				if( nx < 2 || nxny % nx != 0 || int64_t( n ) % nxny != 0 ) { return nullptr; }
				const int64_t ny = nxny / nx, nz = int64_t( n ) / nxny;
				if( ny < 2 || nz < 2 ) { return nullptr; }
				const double diag = row0[ 0 ].second, off = row0[ 1 ].second;
				const int64_t colors = static_cast< int64_t >( data.color_masks.size() );
				int64_t levels = 1;
				for( const auto *c = data.coarser_level; c != nullptr; c = c->coarser_level ) { ++levels; }
				if( colors < 1 || diag == 0.0 ) { return nullptr; }
				auto &cache = hpcg_handles();
				alpb_hpcg h = nullptr;
				for( const HpcgKey &k : cache ) {
					if( k.nx == nx && k.ny == ny && k.nz == nz && k.colors == colors &&
						k.levels == levels && k.diag == diag && k.off == off
					) {
						h = k.h;
					}
				}
				if( h == nullptr ) {
					if( alpb_hpcg_create( &h, nx, ny, nz, diag, off, colors, 1, levels - 1, 1,
							stream() ) != ALPB_SUCCESS
					) {
						return nullptr;
					}
					int64_t got = 0;
					(void) alpb_hpcg_info( h, &got, nullptr, nullptr, nullptr );
					if( got != levels ) {
						(void) alpb_hpcg_destroy( h );
						return nullptr;
					}
					if( cache.size() >= 4 ) {
						(void) alpb_hpcg_destroy( cache.front().h );
						cache.erase( cache.begin() );
					}
					cache.push_back( HpcgKey{ nx, ny, nz, colors, levels, diag, off, h } );
				}
				if( !hpcg_level_matches( h, 0, data, nullptr, 0 ) ) { return nullptr; }
				int64_t l = 1, fine_n = static_cast< int64_t >( n );
				for( const auto *c = data.coarser_level; c != nullptr; c = c->coarser_level, ++l ) {
					if( !hpcg_level_matches( h, l, *c, &c->coarsening_matrix, fine_n ) ) { return nullptr; }
					fine_n = static_cast< int64_t >( c->A.b200_rows() );
				}
				return h;
			}

		}

		/**
		 * hpcg on a b200 system (hpcg/hpcg.hpp:60-223): when the default ring
		 * and minus are used and the system is build_hpcg_system's
		 * (recognised on the device, every call), the whole multigrid-
		 * preconditioned CG -- V-cycle with the multi-colour Gauss-Seidel
		 * smoother, injection restriction and prolongation, the CG updates and
		 * their scalars -- runs as device kernels with no host round trip per
		 * step (alpb_hpcg_solve), from data.x as the initial guess, with the
		 * template's stopping rule (after an iteration with iter >=
		 * max_iterations or ||r|| / ||r_0|| <= tolerance) and norm_residual =
		 * ||r||.  data.r, z, p, u and smoother_temp are work space, as in the
		 * template, and are left untouched.  Anything else runs ALP's template
		 * unchanged.
		 */
		template<
			class Ring = internal_b200_fused::RealRing,
			class Minus = operators::subtract< double >
		>
		grb::RC hpcg( hpcg_data< double, double, double > &data,
			bool with_preconditioning,
			const size_t presmoother_steps,
			const size_t postsmoother_steps,
			const size_t max_iterations,
			const double tolerance,
			size_t &iterations,
			double &norm_residual,
			const Ring &ring = Ring(),
			const Minus &minus = Minus()
		) {
			using namespace grb::internal::b200rt;
			constexpr bool fusable = std::is_same< Ring, internal_b200_fused::RealRing >::value &&
				std::is_same< Minus, operators::subtract< double > >::value;
			alpb_hpcg h = nullptr;
			if( fusable && max_iterations > 0 && internal_b200_fused::is_dense( data.x ) &&
				internal_b200_fused::is_dense( data.b ) && data.x.b200_size() == data.A.b200_rows() &&
				data.b.b200_size() == data.A.b200_rows()
			) {
				h = internal_b200_fused::recognise_hpcg( data );
			}
			if( h == nullptr ) {
				return grb::algorithms::hpcg< double, double, double, double, Ring, Minus >( data,
					with_preconditioning, presmoother_steps, postsmoother_steps, max_iterations,
					tolerance, iterations, norm_residual, ring, minus );
			}
			data.x.b200_device_ready();
			data.b.b200_device_ready();
			int64_t it = 0;
			double res = 0.0;
			RC rc = check( alpb_hpcg_solve( h, reinterpret_cast< const double * >( data.b.b200_values() ),
				reinterpret_cast< double * >( data.x.b200_values() ), with_preconditioning ? 1 : 0,
				static_cast< int64_t >( presmoother_steps ), static_cast< int64_t >( postsmoother_steps ),
				static_cast< int64_t >( max_iterations ), tolerance, &it, &res, stream() ), "hpcg" );
			if( rc == SUCCESS ) {
				rc = internal_b200_fused::mark_dense( data.x );
				iterations = static_cast< size_t >( it );
				norm_residual = res;
			}
			internal_b200_fused::trace( "hpcg", data.x.b200_size(), it );
			return rc;
		}

	} // namespace algorithms

} // namespace grb

#endif
