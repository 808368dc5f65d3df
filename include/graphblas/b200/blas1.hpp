/*
 * Level-1 primitives of the b200 backend (reference: graphblas/reference/
 * blas1.hpp).  Every primitive runs on the device through alpb_vec_op_dom /
 * alpb_vec_reduce_dom with ALP's sparse semantics and returns once the result
 * is in place (blocking execution).  Values are computed in the operands'
 * domain (internal::b200rt::domain_of): double, or exact 64-bit integers with
 * wrap-around, so integer primitives give the reference's bits.  Operators and monoids are those of
 * graphblas/ops.hpp that have a device code (internal::b200rt::op_code); any
 * other operator, or a domain without a device type, gives UNSUPPORTED.
 *
 * eWiseLambda is the exception: its lambda is host code, so it runs on the
 * host over the vectors' managed memory (no device copy of user code exists).
 */
#ifndef _H_GRB_B200_BLAS1
#define _H_GRB_B200_BLAS1

#include <type_traits>

#include <graphblas/base/blas1.hpp>
#include <graphblas/b200/io.hpp>
#include <graphblas/b200/runtime.hpp>
#include <graphblas/b200/vector.hpp>

namespace grb {

	namespace internal {
		namespace b200rt {

			/** Keeps a template argument out of deduction (for nullable operands). */
			template< typename T >
			struct nd { typedef T type; };

			template< class Monoid >
			struct monoid_code {
				static constexpr int value = op_code< typename Monoid::Operator >::value;
				/** The identity in the monoid's own domain (exact as a scalar_t). */
				static scalar_t identity() {
					return static_cast< scalar_t >(
						Monoid().template getIdentity< typename Monoid::D3 >() );
				}
			};

			/** z <- kind(z, x, y) through alpb_vec_op_dom; x / y may be scalars. */
			template< Descriptor descr, typename Z, typename X, typename Y, typename M,
				typename Coords >
			RC vec_op( const int kind, const int op, const bool monoid, const scalar_t identity,
				const int mul_op, Vector< Z, grb::b200, Coords > &z,
				const Vector< M, grb::b200, typename nd< Coords >::type > * const mask,
				const Vector< X, grb::b200, typename nd< Coords >::type > * const x, const scalar_t alpha,
				const Vector< Y, grb::b200, typename nd< Coords >::type > * const y, const scalar_t beta
			) {
				const size_t n = z.b200_size();
				if( mask && size( *mask ) > 0 && size( *mask ) != n ) { return MISMATCH; }
				if( ( x && size( *x ) != n ) || ( y && size( *y ) != n ) ) { return MISMATCH; }
				if( op < 0 ) { return UNSUPPORTED; }
				if( descr & descriptors::dense ) {
					if( nnz( z ) < n && kind != ALPB_VEC_SET && kind != ALPB_VEC_APPLY ) { return ILLEGAL; }
					if( ( x && nnz( *x ) < n ) || ( y && nnz( *y ) < n ) ) { return ILLEGAL; }
				}
				const int zt = type_code< Z >::value;
				const int xt = x ? type_code< X >::value : zt;
				const int yt = y ? type_code< Y >::value : zt;
				const bool masked = mask && size( *mask ) > 0;
				const int mt = masked ? type_code< M >::value : ALPB_VOID;
				if( zt < 0 || xt < 0 || yt < 0 || mt < 0 ) { return UNSUPPORTED; }
				if( n == 0 ) { return SUCCESS; }
				// the operands' domain: integer operators compute exactly on the device
				constexpr int dom = domain_of< Z, X, Y >::value;
				// dense, unmasked steps join the pending chain (run at the next flush)
				const bool y_used = kind == ALPB_VEC_MULADD || kind == ALPB_VEC_APPLY;
				if( fusion_enabled() && !masked && kind != ALPB_VEC_APPLY && z.b200_dense() &&
					( !x || x->b200_dense() ) && ( !y_used || !y || y->b200_dense() ) &&
					op != ALPB_OP_LEFT_ASSIGN_IF &&
					( kind != ALPB_VEC_MULADD || ( mul_op >= 0 && mul_op != ALPB_OP_LEFT_ASSIGN_IF ) ) &&
					chain_type_ok( dom, zt ) && ( !x || chain_type_ok( dom, xt ) ) &&
					( !y_used || !y || chain_type_ok( dom, yt ) )
				) {
					z.b200_device_ready();   // host-written pages back (this may flush)
					if( x ) { x->b200_device_ready(); }
					if( y_used && y ) { y->b200_device_ready(); }
					if( record_step( kind, op, kind == ALPB_VEC_MULADD ? mul_op : ALPB_OP_ADD, descr, dom,
						n, z.b200_values(), zt, x ? x->b200_values() : nullptr, xt, alpha,
						( y_used && y ) ? y->b200_values() : nullptr, yt, beta ) ) { return SUCCESS; }
				}
				z.b200_device_ready();
				if( x ) { x->b200_device_ready(); }
				if( y ) { y->b200_device_ready(); }
				if( masked ) { mask->b200_device_ready(); }
				// a dense output stays dense unless eWiseApply may drop entries
				const bool out_sparse = !z.b200_dense() || kind == ALPB_VEC_APPLY;
				const RC rc = check( alpb_vec_op_dom( kind, op, monoid ? 1 : 0,
					domain_bits( identity, dom ), mul_op, descr, dom, n,
					z.b200_values(), zt, out_sparse ? z.b200_flags() : nullptr,
					out_sparse ? z.b200_counter() : nullptr,
					masked ? mask->b200_values() : nullptr,
					masked ? mask->b200_flags_or_dense() : nullptr, mt, masked ? 1 : 0,
					x ? x->b200_values() : nullptr, xt, x ? x->b200_flags_or_dense() : nullptr,
					domain_bits( alpha, dom ),
					y ? y->b200_values() : nullptr, yt, y ? y->b200_flags_or_dense() : nullptr,
					domain_bits( beta, dom ), stream() ), "blas1" );
				(void) alpb_stream_sync( stream() );
				if( kind == ALPB_VEC_APPLY ) { z.b200_mark_sparse(); }
				z.b200_refresh();
				return rc;
			}

			/** *out (+)= reduce( x (*) y ) through alpb_vec_reduce_dom. */
			template< Descriptor descr, typename OutT, typename X, typename Y, typename M,
				typename Coords >
			RC vec_reduce( OutT &out, const int add_op, const scalar_t identity, const int mul_op,
				const Vector< X, grb::b200, Coords > &x,
				const Vector< Y, grb::b200, typename nd< Coords >::type > * const y,
				const Vector< M, grb::b200, typename nd< Coords >::type > * const mask
			) {
				const size_t n = x.b200_size();
				if( y && size( *y ) != n ) { return MISMATCH; }
				const bool masked = mask && size( *mask ) > 0;
				if( masked && size( *mask ) != n ) { return MISMATCH; }
				if( add_op < 0 || mul_op < 0 ) { return UNSUPPORTED; }
				if( descr & descriptors::dense ) {
					if( nnz( x ) < n || ( y && nnz( *y ) < n ) ) { return ILLEGAL; }
				}
				const int xt = type_code< X >::value, yt = y ? type_code< Y >::value : xt;
				const int mt = masked ? type_code< M >::value : ALPB_VOID;
				if( xt < 0 || yt < 0 || mt < 0 ) { return UNSUPPORTED; }
				if( n == 0 ) { return SUCCESS; }
				// folded on the device in the operands' domain, exactly for integers
				constexpr int dom = domain_of< OutT, X, Y >::value;
				uint64_t r = domain_bits( static_cast< scalar_t >( out ), dom );
				// a dense, unmasked reduction closes a pending chain of its domain in
				// the same device pass (same grid and order as alpb_vec_reduce_dom)
				Chain &c = chain();
				if( c.nsteps > 0 && c.domain == dom && c.n == static_cast< int64_t >( n ) &&
					!masked && x.b200_dense() && ( !y || y->b200_dense() ) &&
					mul_op != ALPB_OP_LEFT_ASSIGN_IF && chain_type_ok( dom, xt ) &&
					( !y || chain_type_ok( dom, yt ) )
				) {
					x.b200_device_ready();   // may flush (host-written pages)
					if( y ) { y->b200_device_ready(); }
					const int xs = c.nsteps > 0 ? chain_slot( c, x.b200_values(), xt ) : -1;
					const int ys = ( c.nsteps > 0 && y ) ? chain_slot( c, y->b200_values(), yt ) : -1;
					if( c.nsteps > 0 && xs >= 0 && ( !y || ys >= 0 ) ) {
						alpb_vec_step &st = c.step[ c.nsteps ];
						st.kind = ALPB_VEC_REDUCE;
						st.op = add_op;
						st.mul_op = y ? mul_op : ALPB_OP_ADD;
						st.descr = descr;
						st.z = 0;
						st.x = xs;
						st.y = ys;
						st.reserved = 0;
						st.alpha = 0;
						st.beta = 0;
						st.identity = domain_bits( identity, dom );
						const int steps = c.nsteps + 1;
						c.nsteps = 0;   // the chain is consumed here, whatever the outcome
						const RC rc = check( alpb_vec_chain( dom, c.n, c.nslots, c.val, c.type, steps,
							c.step, &r, nullptr ), "reduce (fused)" );
						++c.runs;
						c.fused_steps += steps;
						c.nslots = 0;
						c.domain = -1;
						c.n = 0;
						if( rc == SUCCESS ) { out = from_domain_bits< OutT >( r, dom ); }
						return rc;
					}
				}
				x.b200_device_ready();
				if( y ) { y->b200_device_ready(); }
				if( masked ) { mask->b200_device_ready(); }
				const RC rc = check( alpb_vec_reduce_dom( &r, add_op, domain_bits( identity, dom ),
					mul_op, descr, dom, n, x.b200_values(), xt, x.b200_flags_or_dense(),
					y ? y->b200_values() : nullptr, yt, y ? y->b200_flags_or_dense() : nullptr,
					masked ? mask->b200_values() : nullptr, masked ? mask->b200_flags_or_dense() : nullptr,
					mt, masked ? 1 : 0, stream() ), "reduce" );
				if( rc == SUCCESS ) { out = from_domain_bits< OutT >( r, dom ); }
				return rc;
			}

		}
	}

	// ------------------------------------------------------------------ dot --
	template< Descriptor descr = descriptors::no_operation, class AddMonoid, class AnyOp,
		typename OutputType, typename InputType1, typename InputType2, typename Coords >
	RC dot( OutputType &z, const Vector< InputType1, b200, Coords > &x,
		const Vector< InputType2, b200, Coords > &y, const AddMonoid &addMonoid = AddMonoid(),
		const AnyOp &anyOp = AnyOp(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_monoid< AddMonoid >::value && grb::is_operator< AnyOp >::value,
			void >::type * const = nullptr
	) {
		(void) addMonoid;
		(void) anyOp;
		if( phase == RESIZE ) { return size( x ) == size( y ) ? SUCCESS : MISMATCH; }
		using namespace internal::b200rt;
		return vec_reduce< descr, OutputType, InputType1, InputType2, bool >( z,
			monoid_code< AddMonoid >::value, monoid_code< AddMonoid >::identity(),
			op_code< AnyOp >::value, x, &y, nullptr );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename IOType,
		typename InputType1, typename InputType2, typename Coords >
	RC dot( IOType &x, const Vector< InputType1, b200, Coords > &left,
		const Vector< InputType2, b200, Coords > &right, const Ring &ring = Ring(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value && !grb::is_object< IOType >::value &&
			grb::is_semiring< Ring >::value, void >::type * const = nullptr
	) {
		return dot< descr >( x, left, right, ring.getAdditiveMonoid(),
			ring.getMultiplicativeOperator(), phase );
	}

	// ------------------------------------------------- vector -> scalar fold --
	template< Descriptor descr = descriptors::no_operation, class Monoid, typename IOType,
		typename InputType, typename MaskType, typename Coords >
	RC foldl( IOType &x, const Vector< InputType, b200, Coords > &y,
		const Vector< MaskType, b200, Coords > &mask, const Monoid &monoid = Monoid(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< IOType >::value &&
			!grb::is_object< InputType >::value && !grb::is_object< MaskType >::value &&
			grb::is_monoid< Monoid >::value, void >::type * const = nullptr
	) {
		(void) monoid;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_reduce< descr, IOType, InputType, InputType, MaskType >( x,
			monoid_code< Monoid >::value, monoid_code< Monoid >::identity(), ALPB_OP_LEFT_ASSIGN, y,
			nullptr, &mask );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename IOType,
		typename InputType, typename Coords >
	RC foldl( IOType &x, const Vector< InputType, b200, Coords > &y,
		const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< IOType >::value &&
			!grb::is_object< InputType >::value && grb::is_monoid< Monoid >::value,
			void >::type * const = nullptr
	) {
		(void) monoid;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_reduce< descr, IOType, InputType, InputType, bool >( x,
			monoid_code< Monoid >::value, monoid_code< Monoid >::identity(), ALPB_OP_LEFT_ASSIGN, y,
			nullptr, nullptr );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename InputType,
		typename IOType, typename Coords >
	RC foldr( const Vector< InputType, b200, Coords > &x, IOType &beta,
		const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< InputType >::value &&
			!grb::is_object< IOType >::value && grb::is_monoid< Monoid >::value,
			void >::type * const = nullptr
	) {
		return foldl< descr >( beta, x, monoid, phase );
	}

	// ------------------------------------------------- scalar -> vector fold --
	template< Descriptor descr = descriptors::no_operation, class Op, typename IOType,
		typename InputType, typename Coords >
	RC foldl( Vector< IOType, b200, Coords > &x, const InputType beta, const Op &op = Op(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< IOType >::value &&
			!grb::is_object< InputType >::value && grb::is_operator< Op >::value,
			void >::type * = nullptr
	) {
		(void) op;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, IOType, IOType, IOType, bool >( ALPB_VEC_FOLDL,
			internal::b200rt::op_code< Op >::value, false, 0.0, 0, x, nullptr, nullptr,
			static_cast< internal::b200rt::scalar_t >( beta ), nullptr, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename IOType,
		typename InputType, typename Coords >
	RC foldl( Vector< IOType, b200, Coords > &x, const InputType beta,
		const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< IOType >::value &&
			!grb::is_object< InputType >::value && grb::is_monoid< Monoid >::value,
			void >::type * = nullptr
	) {
		(void) monoid;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		// absent entries take beta (reference/blas1.hpp:957-981)
		return vec_op< descr, IOType, IOType, IOType, bool >( ALPB_VEC_FOLDL,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, x, nullptr,
			nullptr, static_cast< internal::b200rt::scalar_t >( beta ), nullptr, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Op, typename IOType,
		typename MaskType, typename InputType, typename Coords >
	RC foldl( Vector< IOType, b200, Coords > &x, const Vector< MaskType, b200, Coords > &m,
		const InputType beta, const Op &op = Op(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< IOType >::value &&
			!grb::is_object< MaskType >::value && !grb::is_object< InputType >::value &&
			grb::is_operator< Op >::value, void >::type * = nullptr
	) {
		(void) op;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, IOType, IOType, IOType, MaskType >( ALPB_VEC_FOLDL,
			internal::b200rt::op_code< Op >::value, false, 0.0, 0, x, &m, nullptr,
			static_cast< internal::b200rt::scalar_t >( beta ), nullptr, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename IOType,
		typename MaskType, typename InputType, typename Coords >
	RC foldl( Vector< IOType, b200, Coords > &x, const Vector< MaskType, b200, Coords > &m,
		const InputType beta, const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< IOType >::value &&
			!grb::is_object< MaskType >::value && !grb::is_object< InputType >::value &&
			grb::is_monoid< Monoid >::value, void >::type * = nullptr
	) {
		(void) monoid;
		if( size( m ) == 0 ) { return foldl< descr >( x, beta, monoid, phase ); }
		if( size( m ) != size( x ) ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, IOType, IOType, IOType, MaskType >( ALPB_VEC_FOLDL,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, x, &m, nullptr,
			static_cast< internal::b200rt::scalar_t >( beta ), nullptr, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename IOType,
		typename InputType, typename Coords >
	RC foldr( const InputType &alpha, Vector< IOType, b200, Coords > &y,
		const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< InputType >::value &&
			!grb::is_object< IOType >::value && grb::is_monoid< Monoid >::value,
			void >::type * const = nullptr
	) {
		(void) monoid;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, IOType, IOType, IOType, bool >( ALPB_VEC_FOLDR,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, y, nullptr,
			nullptr, static_cast< internal::b200rt::scalar_t >( alpha ), nullptr, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class OP, typename IOType,
		typename InputType, typename Coords >
	RC foldr( const InputType &alpha, Vector< IOType, b200, Coords > &y, const OP &op = OP(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< InputType >::value &&
			!grb::is_object< IOType >::value && grb::is_operator< OP >::value,
			void >::type * const = nullptr
	) {
		(void) op;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, IOType, IOType, IOType, bool >( ALPB_VEC_FOLDR,
			internal::b200rt::op_code< OP >::value, false, 0.0, 0, y, nullptr, nullptr,
			static_cast< internal::b200rt::scalar_t >( alpha ), nullptr, 0.0 );
	}

	// ------------------------------------------------- vector -> vector fold --
	template< Descriptor descr = descriptors::no_operation, class OP, typename IOType,
		typename InputType, typename Coords >
	RC foldl( Vector< IOType, b200, Coords > &x, const Vector< InputType, b200, Coords > &y,
		const OP &op = OP(), const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_operator< OP >::value &&
			!grb::is_object< IOType >::value && !grb::is_object< InputType >::value,
			void >::type * = nullptr
	) {
		(void) op;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, IOType, InputType, InputType, bool >( ALPB_VEC_FOLDL,
			internal::b200rt::op_code< OP >::value, false, 0.0, 0, x, nullptr, &y, 0.0, nullptr, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename IOType,
		typename InputType, typename Coords >
	RC foldl( Vector< IOType, b200, Coords > &x, const Vector< InputType, b200, Coords > &y,
		const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_monoid< Monoid >::value &&
			!grb::is_object< IOType >::value && !grb::is_object< InputType >::value,
			void >::type * = nullptr
	) {
		(void) monoid;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, IOType, InputType, InputType, bool >( ALPB_VEC_FOLDL,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, x, nullptr, &y,
			0.0, nullptr, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class OP, typename IOType,
		typename MaskType, typename InputType, typename Coords >
	RC foldl( Vector< IOType, b200, Coords > &x, const Vector< MaskType, b200, Coords > &m,
		const Vector< InputType, b200, Coords > &y, const OP &op = OP(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_operator< OP >::value &&
			!grb::is_object< IOType >::value && !grb::is_object< MaskType >::value &&
			!grb::is_object< InputType >::value, void >::type * = nullptr
	) {
		(void) op;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, IOType, InputType, InputType, MaskType >(
			ALPB_VEC_FOLDL, internal::b200rt::op_code< OP >::value, false, 0.0, 0, x, &m, &y, 0.0,
			nullptr, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename IOType,
		typename MaskType, typename InputType, typename Coords >
	RC foldl( Vector< IOType, b200, Coords > &x, const Vector< MaskType, b200, Coords > &m,
		const Vector< InputType, b200, Coords > &y, const Monoid &monoid = Monoid(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_monoid< Monoid >::value &&
			!grb::is_object< IOType >::value && !grb::is_object< MaskType >::value &&
			!grb::is_object< InputType >::value, void >::type * = nullptr
	) {
		(void) monoid;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, IOType, InputType, InputType, MaskType >( ALPB_VEC_FOLDL,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, x, &m, &y, 0.0,
			nullptr, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class OP, typename IOType,
		typename InputType, typename Coords >
	RC foldr( const Vector< InputType, b200, Coords > &x, Vector< IOType, b200, Coords > &y,
		const OP &op = OP(), const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_operator< OP >::value &&
			!grb::is_object< InputType >::value && !grb::is_object< IOType >::value,
			void >::type * = nullptr
	) {
		(void) op;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, IOType, InputType, InputType, bool >( ALPB_VEC_FOLDR,
			internal::b200rt::op_code< OP >::value, false, 0.0, 0, y, nullptr, &x, 0.0, nullptr, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename IOType,
		typename InputType, typename Coords >
	RC foldr( const Vector< InputType, b200, Coords > &x, Vector< IOType, b200, Coords > &y,
		const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< grb::is_monoid< Monoid >::value &&
			!grb::is_object< InputType >::value && !grb::is_object< IOType >::value,
			void >::type * = nullptr
	) {
		(void) monoid;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, IOType, InputType, InputType, bool >( ALPB_VEC_FOLDR,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, y, nullptr, &x,
			0.0, nullptr, 0.0 );
	}

	// ----------------------------------------------------------- eWiseApply --
	template< Descriptor descr = descriptors::no_operation, class OP, typename OutputType,
		typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< InputType1, b200, Coords > &x, const Vector< InputType2, b200, Coords > &y,
		const OP &op = OP(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_operator< OP >::value, void >::type * const = nullptr
	) {
		(void) op;
		// aliased operands as the reference resolves them (reference/blas1.hpp:5260-5270)
		if( static_cast< const void * >( &x ) == static_cast< const void * >( &y ) &&
			grb::is_idempotent< OP >::value
		) {
			return set< descr >( z, x, phase );
		}
		if( static_cast< const void * >( &x ) == static_cast< const void * >( &z ) ) {
			return foldl< descr >( z, y, op, phase );
		}
		if( static_cast< const void * >( &y ) == static_cast< const void * >( &z ) ) {
			return foldr< descr >( x, z, op, phase );
		}
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, OutputType, InputType1, InputType2, bool >(
			ALPB_VEC_APPLY, internal::b200rt::op_code< OP >::value, false, 0.0, 0, z, nullptr, &x, 0.0,
			&y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename OutputType,
		typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< InputType1, b200, Coords > &x, const Vector< InputType2, b200, Coords > &y,
		const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_monoid< Monoid >::value, void >::type * const = nullptr
	) {
		(void) monoid;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType1, InputType2, bool >( ALPB_VEC_APPLY,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, z, nullptr, &x,
			0.0, &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class OP, typename OutputType,
		typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< InputType1, b200, Coords > &x, const InputType2 beta, const OP &op = OP(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_operator< OP >::value, void >::type * const = nullptr
	) {
		(void) op;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, OutputType, InputType1, InputType1, bool >(
			ALPB_VEC_APPLY, internal::b200rt::op_code< OP >::value, false, 0.0, 0, z, nullptr, &x, 0.0,
			nullptr, static_cast< internal::b200rt::scalar_t >( beta ) );
	}

	template< Descriptor descr = descriptors::no_operation, class OP, typename OutputType,
		typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z, const InputType1 alpha,
		const Vector< InputType2, b200, Coords > &y, const OP &op = OP(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_operator< OP >::value, void >::type * const = nullptr
	) {
		(void) op;
		// z aliasing y folds alpha into it (reference/blas1.hpp:5045-5047)
		if( static_cast< const void * >( &y ) == static_cast< const void * >( &z ) ) {
			return foldr< descr >( alpha, z, op, phase );
		}
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, OutputType, InputType2, InputType2, bool >(
			ALPB_VEC_APPLY, internal::b200rt::op_code< OP >::value, false, 0.0, 0, z, nullptr, nullptr,
			static_cast< internal::b200rt::scalar_t >( alpha ), &y, 0.0 );
	}

	// two scalars: z is set to alpha (.) beta, everywhere or under the mask
	// (reference/blas1.hpp:4083-4300)
	template< Descriptor descr = descriptors::no_operation, class OP, typename OutputType,
		typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z, const InputType1 alpha,
		const InputType2 beta, const OP &op = OP(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_operator< OP >::value, void >::type * const = nullptr
	) {
		if( ( descr & descriptors::dense ) && nnz( z ) < size( z ) ) { return ILLEGAL; }
		if( phase == RESIZE ) { return SUCCESS; }
		typename OP::D3 val;
		const RC rc = apply< descr >( val, alpha, beta, op );
		return rc != SUCCESS ? rc : set< descr >( z, val );
	}

	template< Descriptor descr = descriptors::no_operation, class OP, typename OutputType,
		typename MaskType, typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &mask, const InputType1 alpha,
		const InputType2 beta, const OP &op = OP(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< MaskType >::value && !grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value && grb::is_operator< OP >::value,
			void >::type * const = nullptr
	) {
		if( size( mask ) == 0 ) { return eWiseApply< descr >( z, alpha, beta, op, phase ); }
		if( size( mask ) != size( z ) ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		typename OP::D3 val;
		const RC rc = apply< descr >( val, alpha, beta, op );
		return rc != SUCCESS ? rc : set< descr >( z, mask, val );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename OutputType,
		typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z, const InputType1 alpha,
		const InputType2 beta, const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_monoid< Monoid >::value, void >::type * const = nullptr
	) {
		return eWiseApply< descr >( z, alpha, beta, monoid.getOperator(), phase );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename OutputType,
		typename MaskType, typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &mask, const InputType1 alpha,
		const InputType2 beta, const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< MaskType >::value && !grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value && grb::is_monoid< Monoid >::value,
			void >::type * const = nullptr
	) {
		return eWiseApply< descr >( z, mask, alpha, beta, monoid.getOperator(), phase );
	}

	// masked eWiseApply: z is cleared, then z_i = x_i (.) y_i wherever the mask
	// holds (reference/blas1.hpp:4307-4400, 5090-5180, 5343-5440); an empty mask
	// is the unmasked primitive.  Operators take the intersection of the inputs'
	// structures, monoids their union (reference/blas1.hpp:4658-4780).
	template< Descriptor descr = descriptors::no_operation, class OP, typename OutputType,
		typename MaskType, typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &mask, const Vector< InputType1, b200, Coords > &x,
		const InputType2 beta, const OP &op = OP(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< MaskType >::value && !grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value && grb::is_operator< OP >::value,
			void >::type * const = nullptr
	) {
		if( size( mask ) == 0 ) { return eWiseApply< descr >( z, x, beta, op, phase ); }
		if( size( mask ) != size( z ) ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, OutputType, InputType1, InputType1, MaskType >(
			ALPB_VEC_APPLY, internal::b200rt::op_code< OP >::value, false, 0.0, 0, z, &mask, &x, 0.0,
			nullptr, static_cast< internal::b200rt::scalar_t >( beta ) );
	}

	template< Descriptor descr = descriptors::no_operation, class OP, typename OutputType,
		typename MaskType, typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &mask, const InputType1 alpha,
		const Vector< InputType2, b200, Coords > &y, const OP &op = OP(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< MaskType >::value && !grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value && grb::is_operator< OP >::value,
			void >::type * const = nullptr
	) {
		if( size( mask ) == 0 ) { return eWiseApply< descr >( z, alpha, y, op, phase ); }
		if( size( mask ) != size( z ) ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, OutputType, InputType2, InputType2, MaskType >(
			ALPB_VEC_APPLY, internal::b200rt::op_code< OP >::value, false, 0.0, 0, z, &mask, nullptr,
			static_cast< internal::b200rt::scalar_t >( alpha ), &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class OP, typename OutputType,
		typename MaskType, typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &mask, const Vector< InputType1, b200, Coords > &x,
		const Vector< InputType2, b200, Coords > &y, const OP &op = OP(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< MaskType >::value && !grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value && grb::is_operator< OP >::value,
			void >::type * const = nullptr
	) {
		if( size( mask ) == 0 ) { return eWiseApply< descr >( z, x, y, op, phase ); }
		if( size( mask ) != size( z ) ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::vec_op< descr, OutputType, InputType1, InputType2, MaskType >(
			ALPB_VEC_APPLY, internal::b200rt::op_code< OP >::value, false, 0.0, 0, z, &mask, &x, 0.0,
			&y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename OutputType,
		typename MaskType, typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &mask, const Vector< InputType1, b200, Coords > &x,
		const Vector< InputType2, b200, Coords > &y, const Monoid &monoid = Monoid(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< MaskType >::value && !grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value && grb::is_monoid< Monoid >::value,
			void >::type * const = nullptr
	) {
		if( size( mask ) == 0 ) { return eWiseApply< descr >( z, x, y, monoid, phase ); }
		if( size( mask ) != size( z ) ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType1, InputType2, MaskType >( ALPB_VEC_APPLY,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, z, &mask, &x,
			0.0, &y, 0.0 );
	}

	// monoid with a scalar operand: an absent x_i takes the identity, so the
	// output is dense (reference/blas1.hpp:4502-4640), or dense under the mask
	// (reference/blas1.hpp:4793-4960)
	template< Descriptor descr = descriptors::no_operation, class Monoid, typename OutputType,
		typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< InputType1, b200, Coords > &x, const InputType2 beta,
		const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_monoid< Monoid >::value, void >::type * const = nullptr
	) {
		(void) monoid;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType1, InputType1, bool >( ALPB_VEC_APPLY,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, z, nullptr, &x,
			0.0, nullptr, static_cast< internal::b200rt::scalar_t >( beta ) );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename OutputType,
		typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z, const InputType1 alpha,
		const Vector< InputType2, b200, Coords > &y, const Monoid &monoid = Monoid(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_monoid< Monoid >::value, void >::type * const = nullptr
	) {
		(void) monoid;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType2, InputType2, bool >( ALPB_VEC_APPLY,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, z, nullptr,
			nullptr, static_cast< internal::b200rt::scalar_t >( alpha ), &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename OutputType,
		typename MaskType, typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &mask, const Vector< InputType1, b200, Coords > &x,
		const InputType2 beta, const Monoid &monoid = Monoid(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< MaskType >::value && !grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value && grb::is_monoid< Monoid >::value,
			void >::type * const = nullptr
	) {
		if( size( mask ) == 0 ) { return eWiseApply< descr >( z, x, beta, monoid, phase ); }
		if( size( mask ) != size( z ) ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType1, InputType1, MaskType >( ALPB_VEC_APPLY,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, z, &mask, &x,
			0.0, nullptr, static_cast< internal::b200rt::scalar_t >( beta ) );
	}

	template< Descriptor descr = descriptors::no_operation, class Monoid, typename OutputType,
		typename MaskType, typename InputType1, typename InputType2, typename Coords >
	RC eWiseApply( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &mask, const InputType1 alpha,
		const Vector< InputType2, b200, Coords > &y, const Monoid &monoid = Monoid(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< MaskType >::value && !grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value && grb::is_monoid< Monoid >::value,
			void >::type * const = nullptr
	) {
		if( size( mask ) == 0 ) { return eWiseApply< descr >( z, alpha, y, monoid, phase ); }
		if( size( mask ) != size( z ) ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType2, InputType2, MaskType >( ALPB_VEC_APPLY,
			monoid_code< Monoid >::value, true, monoid_code< Monoid >::identity(), 0, z, &mask,
			nullptr, static_cast< internal::b200rt::scalar_t >( alpha ), &y, 0.0 );
	}

	// ------------------------------------------------------------- eWiseMul --
	/** z = z (+) ( alpha (*) y ) over the ring (reference/blas1.hpp:8610-9172). */
	template< Descriptor descr = descriptors::no_operation, class Ring, typename InputType1,
		typename InputType2, typename OutputType, typename Coords >
	RC eWiseMul( Vector< OutputType, b200, Coords > &z, const InputType1 alpha,
		const Vector< InputType2, b200, Coords > &y, const Ring &ring = Ring(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_semiring< Ring >::value, void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType2, InputType2, bool >( ALPB_VEC_MULADD,
			op_code< typename Ring::AdditiveOperator >::value, false, 0.0,
			op_code< typename Ring::MultiplicativeOperator >::value, z, nullptr, nullptr,
			static_cast< internal::b200rt::scalar_t >( alpha ), &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename InputType1,
		typename InputType2, typename OutputType, typename Coords >
	RC eWiseMul( Vector< OutputType, b200, Coords > &z,
		const Vector< InputType1, b200, Coords > &x, const Vector< InputType2, b200, Coords > &y,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_semiring< Ring >::value, void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType1, InputType2, bool >( ALPB_VEC_MULADD,
			op_code< typename Ring::AdditiveOperator >::value, false, 0.0,
			op_code< typename Ring::MultiplicativeOperator >::value, z, nullptr, &x, 0.0, &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename InputType1,
		typename InputType2, typename OutputType, typename Coords >
	RC eWiseMul( Vector< OutputType, b200, Coords > &z,
		const Vector< InputType1, b200, Coords > &x, const InputType2 beta,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_semiring< Ring >::value, void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType1, InputType1, bool >( ALPB_VEC_MULADD,
			op_code< typename Ring::AdditiveOperator >::value, false, 0.0,
			op_code< typename Ring::MultiplicativeOperator >::value, z, nullptr, &x, 0.0, nullptr,
			static_cast< internal::b200rt::scalar_t >( beta ) );
	}

	/** z = z (+) (alpha (*) beta): nothing when either is the ring's zero, else
	 *  a fold of the product into z (reference/blas1.hpp:8824-8897). */
	template< Descriptor descr = descriptors::no_operation, class Ring, typename InputType1,
		typename InputType2, typename OutputType, typename Coords >
	RC eWiseMul( Vector< OutputType, b200, Coords > &z, const InputType1 alpha,
		const InputType2 beta, const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			grb::is_semiring< Ring >::value, void >::type * const = nullptr
	) {
		if( ( descr & descriptors::dense ) && nnz( z ) < size( z ) ) { return ILLEGAL; }
		if( phase == RESIZE ) { return SUCCESS; }
		if( alpha == ring.template getZero< typename Ring::D1 >() ) { return SUCCESS; }
		if( beta == ring.template getZero< typename Ring::D2 >() ) { return SUCCESS; }
		typename Ring::D3 temp;
		(void) grb::apply( temp, alpha, beta, ring.getMultiplicativeOperator() );
		return foldl< descr >( z, temp, ring.getAdditiveMonoid(), phase );
	}

	/** Masked eWiseMul: z_i = z_i (+) (x_i (*) y_i) where the mask admits i and
	 *  both operands are present (reference/blas1.hpp:8899-9260). */
	template< Descriptor descr = descriptors::no_operation, class Ring, typename InputType1,
		typename InputType2, typename OutputType, typename MaskType, typename Coords >
	RC eWiseMul( Vector< OutputType, b200, Coords > &z, const Vector< MaskType, b200, Coords > &m,
		const Vector< InputType1, b200, Coords > &x, const Vector< InputType2, b200, Coords > &y,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			!grb::is_object< MaskType >::value && grb::is_semiring< Ring >::value,
			void >::type * const = nullptr
	) {
		if( size( m ) == 0 ) { return eWiseMul< descr >( z, x, y, ring, phase ); }
		const size_t n = size( z );
		if( size( m ) != n || size( x ) != n || size( y ) != n ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		if( nnz( x ) == 0 || nnz( y ) == 0 ) { return SUCCESS; }
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType1, InputType2, MaskType >( ALPB_VEC_MULADD,
			op_code< typename Ring::AdditiveOperator >::value, false, 0.0,
			op_code< typename Ring::MultiplicativeOperator >::value, z, &m, &x, 0.0, &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename InputType1,
		typename InputType2, typename OutputType, typename MaskType, typename Coords >
	RC eWiseMul( Vector< OutputType, b200, Coords > &z, const Vector< MaskType, b200, Coords > &m,
		const InputType1 alpha, const Vector< InputType2, b200, Coords > &y,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			!grb::is_object< MaskType >::value && grb::is_semiring< Ring >::value,
			void >::type * const = nullptr
	) {
		if( size( m ) == 0 ) { return eWiseMul< descr >( z, alpha, y, ring, phase ); }
		const size_t n = size( z );
		if( size( m ) != n || size( y ) != n ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		if( nnz( y ) == 0 || alpha == ring.template getZero< typename Ring::D1 >() ) {
			return SUCCESS;
		}
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType2, InputType2, MaskType >( ALPB_VEC_MULADD,
			op_code< typename Ring::AdditiveOperator >::value, false, 0.0,
			op_code< typename Ring::MultiplicativeOperator >::value, z, &m, nullptr,
			static_cast< internal::b200rt::scalar_t >( alpha ), &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename InputType1,
		typename InputType2, typename OutputType, typename MaskType, typename Coords >
	RC eWiseMul( Vector< OutputType, b200, Coords > &z, const Vector< MaskType, b200, Coords > &m,
		const Vector< InputType1, b200, Coords > &x, const InputType2 beta,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			!grb::is_object< MaskType >::value && grb::is_semiring< Ring >::value,
			void >::type * const = nullptr
	) {
		if( size( m ) == 0 ) { return eWiseMul< descr >( z, x, beta, ring, phase ); }
		const size_t n = size( z );
		if( size( m ) != n || size( x ) != n ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		if( nnz( x ) == 0 || beta == ring.template getZero< typename Ring::D2 >() ) {
			return SUCCESS;
		}
		using namespace internal::b200rt;
		return vec_op< descr, OutputType, InputType1, InputType1, MaskType >( ALPB_VEC_MULADD,
			op_code< typename Ring::AdditiveOperator >::value, false, 0.0,
			op_code< typename Ring::MultiplicativeOperator >::value, z, &m, &x, 0.0, nullptr,
			static_cast< internal::b200rt::scalar_t >( beta ) );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename InputType1,
		typename InputType2, typename OutputType, typename MaskType, typename Coords >
	RC eWiseMul( Vector< OutputType, b200, Coords > &z, const Vector< MaskType, b200, Coords > &m,
		const InputType1 alpha, const InputType2 beta, const Ring &ring = Ring(),
		const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			!grb::is_object< InputType1 >::value && !grb::is_object< InputType2 >::value &&
			!grb::is_object< MaskType >::value && grb::is_semiring< Ring >::value,
			void >::type * const = nullptr
	) {
		if( size( m ) == 0 ) { return eWiseMul< descr >( z, alpha, beta, ring, phase ); }
		if( size( m ) != size( z ) ) { return MISMATCH; }
		if( phase == RESIZE ) { return SUCCESS; }
		if( alpha == ring.template getZero< typename Ring::D1 >() ) { return SUCCESS; }
		if( beta == ring.template getZero< typename Ring::D2 >() ) { return SUCCESS; }
		typename Ring::D3 temp;
		(void) grb::apply( temp, alpha, beta, ring.getMultiplicativeOperator() );
		return foldl< descr >( z, m, temp, ring.getAdditiveMonoid(), phase );
	}

	// ---------------------------------------------------------- eWiseMulAdd --
	namespace internal {
		namespace b200rt {
			/** z = z (+) (a (*) x) (+) y over the ring (reference/blas1.hpp:6347-6770):
			 *  the product folds into z where a and x are present, then y folds in as
			 *  a monoid (absent z entries start from the identity); a scalar y reaches
			 *  every entry. */
			template< Descriptor descr, class Ring, typename Z, typename A, typename X, typename Y,
				typename M, typename Coords >
			RC muladd( Vector< Z, grb::b200, Coords > &z,
				const Vector< M, grb::b200, typename nd< Coords >::type > * const mask,
				const Vector< A, grb::b200, typename nd< Coords >::type > * const a, const scalar_t alpha,
				const Vector< X, grb::b200, typename nd< Coords >::type > * const x, const scalar_t chi,
				const Vector< Y, grb::b200, typename nd< Coords >::type > * const y, const scalar_t gamma
			) {
				const int add = op_code< typename Ring::AdditiveOperator >::value;
				const int mul = op_code< typename Ring::MultiplicativeOperator >::value;
				const scalar_t zero = static_cast< scalar_t >( Ring().template getZero< Z >() );
				RC rc;
				if( !a && !x ) {
					// both scalars: fold the constant product into every entry
					rc = vec_op< descr, Z, Z, Z, M >( ALPB_VEC_FOLDL, add, false, zero, 0, z, mask,
						nullptr, 0.0, nullptr, 0.0 );
					if( rc == SUCCESS ) {
						// the constant product, formed in Z as the ring's operator would
						Z prod;
						if( std::is_floating_point< Z >::value ) {
							prod = static_cast< Z >( static_cast< double >( alpha ) *
								static_cast< double >( chi ) );
						} else {
							const uint64_t pa = domain_bits( alpha, ALPB_UINT64 ),
								pc = domain_bits( chi, ALPB_UINT64 );
							prod = static_cast< Z >( pa * pc );   // wraps, as integer products do
						}
						Vector< Z, grb::b200, Coords > c( z.b200_size() );
						rc = set< descriptors::no_operation >( c, prod );
						if( rc == SUCCESS ) {
							rc = vec_op< descr, Z, Z, Z, M >( ALPB_VEC_FOLDL, add, true, zero, 0, z, mask,
								&c, 0.0, nullptr, 0.0 );
						}
					}
				} else {
					rc = vec_op< descr, Z, A, X, M >( ALPB_VEC_MULADD, add, false, zero, mul, z, mask,
						a, alpha, x, chi );
				}
				if( rc != SUCCESS ) { return rc; }
				if( y ) {
					return vec_op< descr, Z, Y, Y, M >( ALPB_VEC_FOLDL, add, true, zero, 0, z, mask, y,
						0.0, nullptr, 0.0 );
				}
				Vector< Z, grb::b200, Coords > g( z.b200_size() );
				rc = set< descriptors::no_operation >( g, static_cast< Z >( gamma ) );
				if( rc != SUCCESS ) { return rc; }
				return vec_op< descr, Z, Z, Z, M >( ALPB_VEC_FOLDL, add, true, zero, 0, z, mask, &g,
					0.0, nullptr, 0.0 );
			}
		}
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const InputType1 alpha,
		const InputType2 chi,
		const InputType3 gamma,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value &&
			!grb::is_object< InputType3 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, OutputType, OutputType, OutputType, bool >( z, nullptr,
			nullptr, static_cast< internal::b200rt::scalar_t >( alpha ), nullptr, static_cast< internal::b200rt::scalar_t >( chi ), nullptr, static_cast< internal::b200rt::scalar_t >( gamma ) );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const InputType1 alpha,
		const InputType2 chi,
		const Vector< InputType3, b200, Coords > &y,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, OutputType, OutputType, InputType3, bool >( z, nullptr,
			nullptr, static_cast< internal::b200rt::scalar_t >( alpha ), nullptr, static_cast< internal::b200rt::scalar_t >( chi ), &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const InputType1 alpha,
		const Vector< InputType2, b200, Coords > &x,
		const InputType3 gamma,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType3 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, OutputType, InputType2, OutputType, bool >( z, nullptr,
			nullptr, static_cast< internal::b200rt::scalar_t >( alpha ), &x, 0.0, nullptr, static_cast< internal::b200rt::scalar_t >( gamma ) );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const InputType1 alpha,
		const Vector< InputType2, b200, Coords > &x,
		const Vector< InputType3, b200, Coords > &y,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< InputType1 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, OutputType, InputType2, InputType3, bool >( z, nullptr,
			nullptr, static_cast< internal::b200rt::scalar_t >( alpha ), &x, 0.0, &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< InputType1, b200, Coords > &a,
		const InputType2 chi,
		const InputType3 gamma,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< InputType2 >::value &&
			!grb::is_object< InputType3 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, InputType1, OutputType, OutputType, bool >( z, nullptr,
			&a, 0.0, nullptr, static_cast< internal::b200rt::scalar_t >( chi ), nullptr, static_cast< internal::b200rt::scalar_t >( gamma ) );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< InputType1, b200, Coords > &a,
		const InputType2 chi,
		const Vector< InputType3, b200, Coords > &y,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< InputType2 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, InputType1, OutputType, InputType3, bool >( z, nullptr,
			&a, 0.0, nullptr, static_cast< internal::b200rt::scalar_t >( chi ), &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< InputType1, b200, Coords > &a,
		const Vector< InputType2, b200, Coords > &x,
		const InputType3 gamma,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< InputType3 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, InputType1, InputType2, OutputType, bool >( z, nullptr,
			&a, 0.0, &x, 0.0, nullptr, static_cast< internal::b200rt::scalar_t >( gamma ) );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< InputType1, b200, Coords > &a,
		const Vector< InputType2, b200, Coords > &x,
		const Vector< InputType3, b200, Coords > &y,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, InputType1, InputType2, InputType3, bool >( z, nullptr,
			&a, 0.0, &x, 0.0, &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename MaskType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &m,
		const InputType1 alpha,
		const InputType2 chi,
		const InputType3 gamma,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< MaskType >::value &&
			!grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value &&
			!grb::is_object< InputType3 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, OutputType, OutputType, OutputType, MaskType >( z, &m,
			nullptr, static_cast< internal::b200rt::scalar_t >( alpha ), nullptr, static_cast< internal::b200rt::scalar_t >( chi ), nullptr, static_cast< internal::b200rt::scalar_t >( gamma ) );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename MaskType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &m,
		const InputType1 alpha,
		const InputType2 chi,
		const Vector< InputType3, b200, Coords > &y,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< MaskType >::value &&
			!grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType2 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, OutputType, OutputType, InputType3, MaskType >( z, &m,
			nullptr, static_cast< internal::b200rt::scalar_t >( alpha ), nullptr, static_cast< internal::b200rt::scalar_t >( chi ), &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename MaskType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &m,
		const InputType1 alpha,
		const Vector< InputType2, b200, Coords > &x,
		const InputType3 gamma,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< MaskType >::value &&
			!grb::is_object< InputType1 >::value &&
			!grb::is_object< InputType3 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, OutputType, InputType2, OutputType, MaskType >( z, &m,
			nullptr, static_cast< internal::b200rt::scalar_t >( alpha ), &x, 0.0, nullptr, static_cast< internal::b200rt::scalar_t >( gamma ) );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename MaskType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &m,
		const InputType1 alpha,
		const Vector< InputType2, b200, Coords > &x,
		const Vector< InputType3, b200, Coords > &y,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< MaskType >::value &&
			!grb::is_object< InputType1 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, OutputType, InputType2, InputType3, MaskType >( z, &m,
			nullptr, static_cast< internal::b200rt::scalar_t >( alpha ), &x, 0.0, &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename MaskType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &m,
		const Vector< InputType1, b200, Coords > &a,
		const InputType2 chi,
		const InputType3 gamma,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< MaskType >::value &&
			!grb::is_object< InputType2 >::value &&
			!grb::is_object< InputType3 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, InputType1, OutputType, OutputType, MaskType >( z, &m,
			&a, 0.0, nullptr, static_cast< internal::b200rt::scalar_t >( chi ), nullptr, static_cast< internal::b200rt::scalar_t >( gamma ) );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename MaskType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &m,
		const Vector< InputType1, b200, Coords > &a,
		const InputType2 chi,
		const Vector< InputType3, b200, Coords > &y,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< MaskType >::value &&
			!grb::is_object< InputType2 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, InputType1, OutputType, InputType3, MaskType >( z, &m,
			&a, 0.0, nullptr, static_cast< internal::b200rt::scalar_t >( chi ), &y, 0.0 );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename MaskType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &m,
		const Vector< InputType1, b200, Coords > &a,
		const Vector< InputType2, b200, Coords > &x,
		const InputType3 gamma,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< MaskType >::value &&
			!grb::is_object< InputType3 >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, InputType1, InputType2, OutputType, MaskType >( z, &m,
			&a, 0.0, &x, 0.0, nullptr, static_cast< internal::b200rt::scalar_t >( gamma ) );
	}

	template< Descriptor descr = descriptors::no_operation, class Ring, typename OutputType, typename MaskType, typename InputType1, typename InputType2, typename InputType3, typename Coords >
	RC eWiseMulAdd( Vector< OutputType, b200, Coords > &z,
		const Vector< MaskType, b200, Coords > &m,
		const Vector< InputType1, b200, Coords > &a,
		const Vector< InputType2, b200, Coords > &x,
		const Vector< InputType3, b200, Coords > &y,
		const Ring &ring = Ring(), const Phase &phase = EXECUTE,
		const typename std::enable_if< !grb::is_object< OutputType >::value &&
			grb::is_semiring< Ring >::value &&
			!grb::is_object< MaskType >::value,
			void >::type * const = nullptr
	) {
		(void) ring;
		if( phase == RESIZE ) { return SUCCESS; }
		return internal::b200rt::muladd< descr, Ring, OutputType, InputType1, InputType2, InputType3, MaskType >( z, &m,
			&a, 0.0, &x, 0.0, &y, 0.0 );
	}

	// ---------------------------------------------------------- eWiseLambda --
	namespace internal {
		namespace b200rt {
			inline void touch() {}
			template< typename T, typename C, typename... Args >
			void touch( const Vector< T, grb::b200, C > &v, const Args &... args ) {
				(void) v.raw();  // synchronised host access; pages return on next device use
				touch( args... );
			}
			template< typename First, typename... Args >
			void touch( const First &, const Args &... args ) { touch( args... ); }
		}
	}

	/** Runs f(i) on the host for every assigned index of x (all when dense). */
	template< Descriptor descr = descriptors::no_operation, class Func, typename DataType1,
		typename Coords, typename... Args >
	RC eWiseLambda( const Func f, const Vector< DataType1, b200, Coords > &x,
		const Args &... args
	) {
		x.b200_host_ready();
		internal::b200rt::touch( x, args... );
		const size_t n = size( x );
		const uint8_t * const fl = x.b200_flags();
		const bool dense = x.b200_dense() || ( descr & descriptors::dense );
		for( size_t i = 0; i < n; ++i ) {
			if( dense || fl[ i ] ) { f( i ); }
		}
		return SUCCESS;
	}

}

#endif
