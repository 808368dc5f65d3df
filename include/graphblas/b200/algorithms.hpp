/*
 * Differentiated solvers of the b200 backend, in ALP's C++ API.  No
 * counterpart exists in the reference, whose algorithms
 * (graphblas/algorithms/conjugate_gradient.hpp, simple_pagerank.hpp) are
 * forward-only; these are their implicit-function adjoints, which store no
 * iterate of the forward solve.
 *
 *   conjugate_gradient_adjoint   dL/db and dL/dA of x = A^{-1} b
 *   PersonalisedPageRank         simple_pagerank with one-hot teleport vectors
 *                                (seeds) over weighted edges, its adjoint and
 *                                the gradient with respect to every weight
 *
 * Include after <graphblas.hpp> in a program compiled for the b200 backend.
 */
#ifndef _H_GRB_B200_ALGORITHMS
#define _H_GRB_B200_ALGORITHMS

#include <cstdint>
#include <vector>

#include <graphblas.hpp>
#include <graphblas/b200/runtime.hpp>

namespace grb {

	namespace algorithms {

		namespace internal_b200 {

			/** A kernel wrote all n entries of x: mark every one assigned. */
			template< typename D, typename C >
			RC assign_all( Vector< D, b200, C > &x ) {
				using namespace grb::internal::b200rt;
				const size_t n = x.b200_size();
				if( n == 0 ) { return SUCCESS; }
				RC rc = check( alpb_memset( x.b200_flags(), 1, n, stream() ), "assign_all" );
				const int64_t cnt = static_cast< int64_t >( n );
				rc = rc ? rc : check( alpb_memcpy_h2d( x.b200_counter(), &cnt, 8, stream() ),
					"assign_all" );
				rc = rc ? rc : check( alpb_stream_sync( stream() ), "assign_all" );
				if( rc == SUCCESS ) { x.b200_mark_dense(); }
				return rc;
			}

			template< typename D, typename C >
			bool dense( const Vector< D, b200, C > &x ) {
				const_cast< Vector< D, b200, C > & >( x ).b200_refresh();
				return x.b200_dense() || x.b200_size() == 0;
			}

		}

		/**
		 * Adjoint of a conjugate-gradient solve x = A^{-1} b (A symmetric positive
		 * definite, as conjugate_gradient requires; conjugate_gradient.hpp:507-590)
		 * for a loss L whose gradient at x is \a dL_dx:
		 *
		 *   lambda = A^{-T} dL_dx      (= dL/db), by CG on A's column storage from
		 *                              lambda = 0 with conjugate_gradient's stopping
		 *                              rule (relative tolerance \a tol);
		 *   grad_values[k] = -lambda_i x_j  for the k-th stored entry (i, j) of A, in
		 *                              the order A's iterator visits them (= dL/dA
		 *                              on A's pattern).
		 *
		 * \a x, \a dL_dx must be dense; \a lambda has size nrows(A) and
		 * \a grad_values size nnz(A).  Returns FAILED when the adjoint CG did not
		 * converge within \a max_iterations (the outputs hold the last iterate).
		 */
		template<
			Descriptor descr = descriptors::no_operation,
			typename RIT, typename CIT, typename NIT, typename C
		>
		RC conjugate_gradient_adjoint(
			Vector< double, b200, C > &lambda,
			Vector< double, b200, C > &grad_values,
			const Matrix< double, b200, RIT, CIT, NIT > &A,
			const Vector< double, b200, C > &x,
			const Vector< double, b200, C > &dL_dx,
			const size_t max_iterations,
			const double tol,
			size_t &iterations,
			double &residual
		) {
			using namespace grb::internal::b200rt;
			const size_t n = A.b200_rows();
			if( A.b200_cols() != n || x.b200_size() != n || dL_dx.b200_size() != n ||
				lambda.b200_size() != n || grad_values.b200_size() != A.b200_nnz()
			) {
				return MISMATCH;
			}
			if( !internal_b200::dense( x ) || !internal_b200::dense( dL_dx ) ) { return ILLEGAL; }
			x.b200_device_ready();
			dL_dx.b200_device_ready();
			lambda.b200_device_ready();
			grad_values.b200_device_ready();
			const auto &crs = A.b200_crs();
			const auto &ccs = A.b200_ccs();
			int64_t it = 0;
			RC rc = check( alpb_cg_adjoint( static_cast< int64_t >( n ), crs.offsets, crs.indices,
				crs.values, ccs.offsets, ccs.indices, ccs.values, x.b200_values(),
				dL_dx.b200_values(), lambda.b200_values(),
				A.b200_nnz() > 0 ? grad_values.b200_values() : nullptr,
				static_cast< int64_t >( max_iterations ), tol, &it, &residual, nullptr, nullptr,
				stream() ), "conjugate_gradient_adjoint" );
			iterations = static_cast< size_t >( it );
			if( rc == SUCCESS || rc == FAILED ) {
				const RC r1 = internal_b200::assign_all( lambda );
				const RC r2 = internal_b200::assign_all( grad_values );
				if( rc == SUCCESS ) { rc = r1 ? r1 : r2; }
			}
			return rc;
		}

		/**
		 * Personalised PageRank over the weighted graph \a W (row i -> column j,
		 * weight w_ij >= 0) for up to 128 seeds at once, and its adjoint.  The
		 * forward solve is simple_pagerank (simple_pagerank.hpp:146-533) with the
		 * uniform teleport vector replaced by the one-hot vector of each seed and
		 * the out-degree count by the weighted out-degree d_i = sum_j w_ij:
		 *
		 *   x_s = alpha M x_s + (alpha dangling(x_s) + 1 - alpha) e_{seed_s},
		 *   M_ji = w_ij / d_i,
		 *
		 * by the same power iteration and L1 stopping rule, each seed on its own.
		 * With unit weights the normalisation is the reference's.
		 *
		 * Containers holding all seeds (X, dL/dX, Lambda) are vectors of
		 * nrows(W) * nseeds entries: entry i * nseeds + s belongs to seed s.
		 * W's pattern and storage must stay unchanged while this object lives;
		 * after changing W's values call refresh_weights().
		 */
		template<
			typename RIT = config::RowIndexType,
			typename CIT = config::ColIndexType,
			typename NIT = config::NonzeroIndexType
		>
		class PersonalisedPageRank {

			public:

				typedef Matrix< double, b200, RIT, CIT, NIT > matrix_type;

				PersonalisedPageRank( const matrix_type &W, const size_t nseeds ) :
					_W( W ), _n( W.b200_rows() ), _S( nseeds )
				{
					using namespace grb::internal::b200rt;
					if( W.b200_cols() != _n ) {
						_status = MISMATCH;
						return;
					}
					const auto &crs = W.b200_crs();
					_status = check( alpb_ppr_create( &_h, static_cast< int64_t >( _n ),
						static_cast< int64_t >( W.b200_nnz() ), crs.offsets, crs.indices, crs.values,
						static_cast< int >( nseeds ), stream() ), "PersonalisedPageRank" );
				}

				~PersonalisedPageRank() {
					if( _h ) { (void) alpb_ppr_destroy( _h ); }
				}

				PersonalisedPageRank( const PersonalisedPageRank & ) = delete;
				PersonalisedPageRank & operator=( const PersonalisedPageRank & ) = delete;

				/** SUCCESS when the constructor built the transpose and chunk tables. */
				RC status() const noexcept { return _status; }

				/** W's values changed in place (same pattern, same storage). */
				RC refresh_weights() {
					using namespace grb::internal::b200rt;
					if( _status != SUCCESS ) { return _status; }
					return check( alpb_ppr_set_weights( _h, _W.b200_crs().values, stream() ),
						"PersonalisedPageRank::refresh_weights" );
				}

				/**
				 * The personalised vectors of \a seeds (nseeds rows of W) into \a X.
				 * \a X starts from 1/n, or from its contents when \a initial_guess.
				 * Returns FAILED when some seed did not reach \a conv within
				 * \a max_iterations (X then holds its last iterate).
				 */
				RC solve(
					Vector< double, b200 > &X,
					const std::vector< size_t > &seeds,
					const double alpha = 0.85,
					const double conv = 1e-8,
					const size_t max_iterations = 1000,
					const bool initial_guess = false,
					std::vector< size_t > * const iterations = nullptr,
					std::vector< double > * const residuals = nullptr
				) {
					using namespace grb::internal::b200rt;
					if( _status != SUCCESS ) { return _status; }
					if( seeds.size() != _S || X.b200_size() != _n * _S ) { return MISMATCH; }
					if( initial_guess && !internal_b200::dense( X ) ) { return ILLEGAL; }
					std::vector< int64_t > sd( seeds.begin(), seeds.end() );
					std::vector< int64_t > it( _S );
					std::vector< double > res( _S );
					X.b200_device_ready();
					RC rc = check( alpb_ppr_solve( _h, sd.data(), alpha, conv,
						static_cast< int64_t >( max_iterations ), X.b200_values(), initial_guess ? 1 : 0,
						it.data(), res.data(), stream() ), "PersonalisedPageRank::solve" );
					if( rc == SUCCESS || rc == FAILED ) {
						const RC r = internal_b200::assign_all( X );
						if( rc == SUCCESS ) { rc = r; }
						copy_out( it, res, iterations, residuals );
					}
					return rc;
				}

				/**
				 * Adjoint of the last solve's fixed point: Lambda with
				 *   lambda_s = alpha M^T lambda_s + alpha [i dangling] lambda_s[seed_s]
				 *              + dL/dx_s,
				 * iterated from lambda = dL/dX with the forward's stopping rule.
				 * dL/d(teleport weight of seed s) = (1 - alpha) lambda_s[seed_s].
				 */
				RC adjoint(
					Vector< double, b200 > &Lambda,
					const Vector< double, b200 > &dL_dX,
					const double conv = 1e-8,
					const size_t max_iterations = 1000,
					std::vector< size_t > * const iterations = nullptr,
					std::vector< double > * const residuals = nullptr
				) {
					using namespace grb::internal::b200rt;
					if( _status != SUCCESS ) { return _status; }
					if( Lambda.b200_size() != _n * _S || dL_dX.b200_size() != _n * _S ) {
						return MISMATCH;
					}
					if( !internal_b200::dense( dL_dX ) ) { return ILLEGAL; }
					std::vector< int64_t > it( _S );
					std::vector< double > res( _S );
					dL_dX.b200_device_ready();
					Lambda.b200_device_ready();
					RC rc = check( alpb_ppr_adjoint( _h, dL_dX.b200_values(), Lambda.b200_values(),
						conv, static_cast< int64_t >( max_iterations ), it.data(), res.data(),
						stream() ), "PersonalisedPageRank::adjoint" );
					if( rc == SUCCESS || rc == FAILED ) {
						const RC r = internal_b200::assign_all( Lambda );
						if( rc == SUCCESS ) { rc = r; }
						copy_out( it, res, iterations, residuals );
					}
					return rc;
				}

				/**
				 * dL/dw for every stored edge of W, in the order W's iterator visits
				 * them:  alpha / d_i sum_s x_is (lambda_js - (M^T lambda_s)_i), zero
				 * on dangling rows.  \a dL_dW has size nnz(W).
				 */
				RC gradient(
					Vector< double, b200 > &dL_dW,
					const Vector< double, b200 > &X,
					const Vector< double, b200 > &Lambda
				) {
					using namespace grb::internal::b200rt;
					if( _status != SUCCESS ) { return _status; }
					if( dL_dW.b200_size() != _W.b200_nnz() || X.b200_size() != _n * _S ||
						Lambda.b200_size() != _n * _S
					) {
						return MISMATCH;
					}
					if( !internal_b200::dense( X ) || !internal_b200::dense( Lambda ) ) {
						return ILLEGAL;
					}
					X.b200_device_ready();
					Lambda.b200_device_ready();
					dL_dW.b200_device_ready();
					RC rc = check( alpb_ppr_grad_weights( _h, X.b200_values(), Lambda.b200_values(),
						_W.b200_nnz() > 0 ? dL_dW.b200_values() : nullptr, stream() ),
						"PersonalisedPageRank::gradient" );
					return rc ? rc : internal_b200::assign_all( dL_dW );
				}

			private:

				const matrix_type &_W;
				size_t _n, _S;
				alpb_ppr _h = nullptr;
				RC _status = PANIC;

				void copy_out( const std::vector< int64_t > &it, const std::vector< double > &res,
					std::vector< size_t > * const iterations, std::vector< double > * const residuals
				) const {
					if( iterations ) { iterations->assign( it.begin(), it.end() ); }
					if( residuals ) { *residuals = res; }
				}

		};

	} // namespace algorithms

} // namespace grb

#endif
