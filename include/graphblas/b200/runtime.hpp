/*
 * Glue between ALP's C++ types and the C-ABI of libalp_b200.so
 * (include/alp_b200.h): element type codes, operator codes of ALP's
 * operator classes (graphblas/ops.hpp), semiring codes, device buffers and
 * the stream every b200 primitive is ordered on.
 *
 * Host code of the b200 backend is compiled by the host compiler only (no
 * CUDA headers needed): it calls the C-ABI, which launches the kernels.
 */
#ifndef _H_GRB_B200_RUNTIME
#define _H_GRB_B200_RUNTIME

#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <type_traits>

#include <alp_b200.h>

#include <graphblas/backends.hpp>
#include <graphblas/ops.hpp>
#include <graphblas/rc.hpp>

namespace grb {

	namespace internal {

		namespace b200rt {

			/**
			 * Pending chain of dense level-1 steps (alpb_vec_chain): set, foldl,
			 * foldr, eWiseMul and eWiseMulAdd calls on dense vectors without a mask
			 * are recorded instead of run, and the chain runs as ONE device pass
			 * when anything else needs the device or a vector's values -- a dot or
			 * fold to a scalar closes it inside that pass.  This is the lazy fusion
			 * of ALP's nonblocking backend (include/graphblas/nonblocking/), done
			 * on the device; results are those of the steps run one by one, bit
			 * for bit.  ALPB_FUSE=0 in the environment runs every step at once.
			 */
			struct Chain {
				int domain = -1;
				int64_t n = 0;
				int nslots = 0, nsteps = 0;
				void * val[ ALPB_CHAIN_SLOTS ];
				int type[ ALPB_CHAIN_SLOTS ];
				alpb_vec_step step[ ALPB_CHAIN_STEPS ];
				int enabled = -1;   // -1: ALPB_FUSE not read yet
				long runs = 0, fused_steps = 0;   // passes run, steps they held
			};
			inline Chain & chain() noexcept { static Chain c; return c; }

			inline bool fusion_enabled() noexcept {
				Chain &c = chain();
				if( c.enabled < 0 ) {
					const char * const e = std::getenv( "ALPB_FUSE" );
					c.enabled = ( e && e[ 0 ] == '0' ) ? 0 : 1;
				}
				return c.enabled == 1;
			}

			/** Runs the pending chain, if any (enqueued on the default stream). */
			inline void flush() noexcept {
				Chain &c = chain();
				if( c.nsteps == 0 ) { return; }
				const int rc = alpb_vec_chain( c.domain, c.n, c.nslots, c.val, c.type, c.nsteps,
					c.step, nullptr, nullptr );
				++c.runs;
				c.fused_steps += c.nsteps;
				c.nsteps = 0;
				c.nslots = 0;
				c.domain = -1;
				c.n = 0;
				if( rc != ALPB_SUCCESS ) {
#ifndef _GRB_NO_STDIO
					std::cerr << "grb::b200: fused level-1 chain: " << alpb_last_error() << "\n";
#endif
				}
			}

			/** Stream all primitives are ordered on (NULL: the legacy default
			 *  stream); asking for it runs the pending chain first. */
			inline void * stream() noexcept {
				flush();
				return nullptr;
			}

			/** The C-ABI returns grb::RC numbering; map it and keep the message. */
			inline RC check( const int rc, const char * const where ) {
				if( rc != ALPB_SUCCESS ) {
#ifndef _GRB_NO_STDIO
					std::cerr << "grb::b200: " << where << ": " << alpb_last_error() << "\n";
#endif
				}
				return static_cast< RC >( rc );
			}

			/** Element type code of a C++ domain; -1 when the device cannot hold it. */
			template< typename T, typename Enable = void >
			struct type_code { static constexpr int value = -1; };
			template<> struct type_code< double > { static constexpr int value = ALPB_FP64; };
			template<> struct type_code< bool > { static constexpr int value = ALPB_BOOL; };
			template<> struct type_code< int > { static constexpr int value = ALPB_INT32; };
			template<> struct type_code< unsigned int > { static constexpr int value = ALPB_UINT32; };
			template<> struct type_code< long > { static constexpr int value = ALPB_INT64; };
			template<> struct type_code< long long > { static constexpr int value = ALPB_INT64; };
			template<> struct type_code< unsigned long > { static constexpr int value = ALPB_INT64; };
			template<> struct type_code< unsigned char > { static constexpr int value = ALPB_UINT8; };
			template<> struct type_code< signed char > { static constexpr int value = ALPB_INT8; };
			template<> struct type_code< char > { static constexpr int value = ALPB_INT8; };
			template<> struct type_code< void > { static constexpr int value = ALPB_VOID; };

			/** Device storage type of a domain (bool is held as one byte). */
			template< typename T >
			struct storage { typedef T type; };
			template<>
			struct storage< bool > { typedef uint8_t type; };

			/** Operator code of an ALP operator class; -1 when not on the device. */
			template< class OP >
			struct op_code { static constexpr int value = -1; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::add< A, B, C, X > > { static constexpr int value = ALPB_OP_ADD; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::subtract< A, B, C, X > > { static constexpr int value = ALPB_OP_SUB; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::mul< A, B, C, X > > { static constexpr int value = ALPB_OP_MUL; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::divide< A, B, C, X > > { static constexpr int value = ALPB_OP_DIV; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::min< A, B, C, X > > { static constexpr int value = ALPB_OP_MIN; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::max< A, B, C, X > > { static constexpr int value = ALPB_OP_MAX; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::abs_diff< A, B, C, X > > { static constexpr int value = ALPB_OP_ABS_DIFF; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::left_assign< A, B, C, X > > { static constexpr int value = ALPB_OP_LEFT_ASSIGN; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::right_assign< A, B, C, X > > { static constexpr int value = ALPB_OP_RIGHT_ASSIGN; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::logical_or< A, B, C, X > > { static constexpr int value = ALPB_OP_LOR; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::logical_and< A, B, C, X > > { static constexpr int value = ALPB_OP_LAND; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::equal< A, B, C, X > > { static constexpr int value = ALPB_OP_EQUAL; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::not_equal< A, B, C, X > > {
				static constexpr int value = ALPB_OP_NOT_EQUAL;
			};
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::less_than< A, B, C, X > > { static constexpr int value = ALPB_OP_LESS; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::leq< A, B, C, X > > { static constexpr int value = ALPB_OP_LEQ; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::greater_than< A, B, C, X > > {
				static constexpr int value = ALPB_OP_GREATER;
			};
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::geq< A, B, C, X > > { static constexpr int value = ALPB_OP_GEQ; };
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::left_assign_if< A, B, C, X > > {
				static constexpr int value = ALPB_OP_LEFT_ASSIGN_IF;
			};
			// on real domains the conjugating multiplications are plain products
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::conjugate_right_mul< A, B, C, X > > {
				static constexpr int value = std::is_floating_point< A >::value ? ALPB_OP_MUL : -1;
			};
			template< typename A, typename B, typename C, Backend X >
			struct op_code< operators::conjugate_left_mul< A, B, C, X > > {
				static constexpr int value = std::is_floating_point< A >::value ? ALPB_OP_MUL : -1;
			};

			/** Semiring code of a (additive, multiplicative) operator pair; -1 otherwise. */
			template< class ADD, class MUL >
			struct ring_code { static constexpr int value = -1; };
			template< Backend X, Backend Y >
			struct ring_code< operators::add< double, double, double, X >,
				operators::mul< double, double, double, Y > > {
				static constexpr int value = ALPB_RING_PLUS_TIMES_F64;
			};
			template< Backend X, Backend Y >
			struct ring_code< operators::logical_or< bool, bool, bool, X >,
				operators::logical_and< bool, bool, bool, Y > > {
				static constexpr int value = ALPB_RING_LOR_LAND_BOOL;
			};
			template< Backend X, Backend Y >
			struct ring_code< operators::min< int, int, int, X >,
				operators::add< int, int, int, Y > > {
				static constexpr int value = ALPB_RING_MIN_PLUS_I32;
			};
			template< Backend X, Backend Y >
			struct ring_code< operators::add< double, double, double, X >,
				operators::left_assign_if< double, bool, double, Y > > {
				static constexpr int value = ALPB_RING_PLUS_PATTERN_F64;
			};
			template< Backend X, Backend Y >
			struct ring_code< operators::add< int, int, int, X >,
				operators::mul< int, int, int, Y > > {
				static constexpr int value = ALPB_RING_PLUS_TIMES_I32;
			};

			// the degree ring of the Pregel interface (interfaces/pregel.hpp:381-386)
			template< Backend X, Backend Y >
			struct ring_code< operators::add< size_t, size_t, size_t, X >,
				operators::right_assign_if< bool, size_t, size_t, Y > > {
				static constexpr int value = ALPB_RING_PLUS_RIGHT_IF_U64;
			};
			// Pregel messages under max (pregel.hpp:714-720 with operators::max<size_t>)
			template< Backend X, Backend Y >
			struct ring_code< operators::max< size_t, size_t, size_t, X >,
				operators::left_assign_if< size_t, bool, size_t, Y > > {
				static constexpr int value = ALPB_RING_MAX_LEFT_IF_U64;
			};

			template< Backend X, Backend Y >
			struct ring_code< operators::mul< double, double, double, X >,
				operators::add< double, double, double, Y > > {
				static constexpr int value = ALPB_RING_TIMES_PLUS_F64;
			};

			/** Host scalar that holds every double and every 64-bit integer
			 *  exactly (a 64-bit or wider significand), so that scalars reach the
			 *  device unrounded in whichever domain the primitive computes. */
			typedef long double scalar_t;
			static_assert( std::numeric_limits< long double >::digits >= 64,
				"the b200 backend needs a long double with a 64-bit significand" );

			/** Compute domain of an element-wise primitive over operands of these
			 *  C++ types, as the reference's operators cast to their domain:
			 *  ALPB_FP64 when any is floating point; else the widest integer
			 *  width among them (64 or 32 bits, bool and narrower types count as
			 *  32), unsigned when an operand of that width is unsigned. */
			template< typename... T >
			struct domain_of {
				static constexpr bool fp = false, wide = false, u64 = false, u32 = false;
				static constexpr int value = ALPB_INT32;
			};
			template< typename H, typename... T >
			struct domain_of< H, T... > {
				typedef domain_of< T... > rest;
				static constexpr bool is_int = std::is_integral< H >::value;
				static constexpr bool fp = std::is_floating_point< H >::value || rest::fp;
				static constexpr bool wide = ( is_int && sizeof( H ) == 8 ) || rest::wide;
				static constexpr bool u64 = ( is_int && std::is_unsigned< H >::value &&
					sizeof( H ) == 8 ) || rest::u64;
				static constexpr bool u32 = ( is_int && std::is_unsigned< H >::value &&
					sizeof( H ) == 4 ) || rest::u32;
				static constexpr int value = fp ? ALPB_FP64 : wide ? ( u64 ? ALPB_UINT64 : ALPB_INT64 ) :
					( u32 ? ALPB_UINT32 : ALPB_INT32 );
			};

			/** The bits of v as a value of domain `dom`.  Integer domains clamp to
			 *  their range: an infinite identity (of min or max) becomes the
			 *  domain's extreme, which is that identity there. */
			inline uint64_t domain_bits( const scalar_t v, const int dom ) {
				uint64_t b = 0;
				if( dom == ALPB_FP64 ) {
					const double d = static_cast< double >( v );
					std::memcpy( &b, &d, 8 );
				} else if( dom == ALPB_INT64 ) {
					const scalar_t lo = static_cast< scalar_t >( std::numeric_limits< int64_t >::min() );
					const scalar_t hi = static_cast< scalar_t >( std::numeric_limits< int64_t >::max() );
					const int64_t i = v != v ? 0 : v <= lo ? std::numeric_limits< int64_t >::min() :
						v >= hi ? std::numeric_limits< int64_t >::max() : static_cast< int64_t >( v );
					std::memcpy( &b, &i, 8 );
				} else if( dom == ALPB_INT32 ) {
					const int32_t i = v != v ? 0 : v <= -2147483648.0L ? std::numeric_limits< int32_t >::min() :
						v >= 2147483647.0L ? std::numeric_limits< int32_t >::max() :
						static_cast< int32_t >( v );
					std::memcpy( &b, &i, 4 );
				} else if( dom == ALPB_UINT32 ) {
					// a negative scalar wraps, as its conversion to an unsigned type does
					const uint32_t u = v != v ? 0 : v >= 4294967295.0L ? 4294967295u :
						v < 0 ? static_cast< uint32_t >( static_cast< int64_t >( v ) ) :
						static_cast< uint32_t >( v );
					std::memcpy( &b, &u, 4 );
				} else {
					const scalar_t hi = static_cast< scalar_t >( std::numeric_limits< uint64_t >::max() );
					// a negative scalar wraps, as its conversion to an unsigned type does
					b = v != v ? 0 : v >= hi ? std::numeric_limits< uint64_t >::max() :
						v < 0 ? static_cast< uint64_t >( static_cast< int64_t >( v ) ) :
						static_cast< uint64_t >( v );
				}
				return b;
			}

			/** A value of domain `dom` (its bits) as T, converted the way C++
			 *  converts from the domain's type (integers wrap). */
			template< typename T >
			T from_domain_bits( const uint64_t b, const int dom ) {
				if( dom == ALPB_FP64 ) {
					double d;
					std::memcpy( &d, &b, 8 );
					return static_cast< T >( d );
				}
				if( dom == ALPB_INT64 ) { return static_cast< T >( static_cast< int64_t >( b ) ); }
				if( dom == ALPB_INT32 ) {
					int32_t i;
					std::memcpy( &i, &b, 4 );
					return static_cast< T >( i );
				}
				if( dom == ALPB_UINT32 ) { return static_cast< T >( static_cast< uint32_t >( b ) ); }
				return static_cast< T >( b );
			}

			/** Device allocation that reports OUTOFMEM through the C-ABI. */
			template< typename T >
			T * alloc( const size_t n ) {
				void * p = nullptr;
				if( n == 0 ) { return nullptr; }
				const int rc = alpb_malloc( &p, n * sizeof( T ) );
				if( rc != ALPB_SUCCESS ) {
					throw std::runtime_error( std::string( "grb::b200: device allocation of " ) +
						std::to_string( n * sizeof( T ) ) + " bytes failed: " + alpb_last_error() );
				}
				return static_cast< T * >( p );
			}

			inline void release( void * p ) noexcept {
				if( p ) {
					flush();   // the pending chain may name this buffer
					(void) alpb_free( p );
				}
			}

			/** Whether a vector of type code t joins a chain in domain dom (the
			 *  domain's own type: no value is rounded between fused steps). */
			inline bool chain_type_ok( const int dom, const int t ) noexcept {
				return t == dom || ( dom == ALPB_UINT64 && t == ALPB_INT64 ) ||
					( dom == ALPB_INT64 && t == ALPB_UINT64 );
			}

			/** Slot of buffer p in the pending chain (added if new); -1 when full. */
			inline int chain_slot( Chain &c, void * const p, const int t ) noexcept {
				for( int q = 0; q < c.nslots; ++q ) {
					if( c.val[ q ] == p ) { return q; }
				}
				if( c.nslots == ALPB_CHAIN_SLOTS ) { return -1; }
				c.val[ c.nslots ] = p;
				c.type[ c.nslots ] = t;
				return c.nslots++;
			}

			/**
			 * Appends a step on dense vectors (z; x and y, or NULL for the
			 * scalars alpha and beta) to the pending chain, after running what is
			 * pending if the domain or length differs or the chain is full.  The
			 * caller has checked that the step is one alpb_vec_chain accepts and
			 * that every vector is dense and of the domain's type.
			 */
			inline bool record_step( const int kind, const int op, const int mul_op,
				const uint32_t descr, const int dom, const size_t n, void * const z, const int zt,
				void * const x, const int xt, const scalar_t alpha, void * const y, const int yt,
				const scalar_t beta
			) {
				Chain &c = chain();
				if( c.nsteps > 0 && ( c.domain != dom || c.n != static_cast< int64_t >( n ) ||
					c.nsteps >= ALPB_CHAIN_STEPS - 1 ) ) { flush(); }
				for( int attempt = 0; attempt < 2; ++attempt ) {
					const int zs = chain_slot( c, z, zt );
					const int xs = x ? chain_slot( c, x, xt ) : -1;
					const int ys = y ? chain_slot( c, y, yt ) : -1;
					if( zs < 0 || ( x && xs < 0 ) || ( y && ys < 0 ) ) {
						flush();   // out of slots: run what is pending, then start anew
						continue;
					}
					alpb_vec_step &st = c.step[ c.nsteps++ ];
					st.kind = kind;
					st.op = op;
					st.mul_op = mul_op;
					st.descr = descr;
					st.z = zs;
					st.x = xs;
					st.y = ys;
					st.reserved = 0;
					st.alpha = domain_bits( alpha, dom );
					st.beta = domain_bits( beta, dom );
					st.identity = 0;
					c.domain = dom;
					c.n = static_cast< int64_t >( n );
					return true;
				}
				return false;
			}

		} // namespace b200rt

	} // namespace internal

} // namespace grb

#endif
