/*
 * Differential test driver: one ALP/GraphBLAS program, compiled once against
 * the reference backend (the checker, into oracle/_ref/cpp/) and once against
 * the b200 backend (into _build/cpp/), by tests/cpp/Makefile.  It reads a
 * case file, runs ALP's public API on it and prints every result with 17
 * significant digits, so the two builds can be compared line by line.
 *
 *   alp_driver <case file>
 *
 * Case file (little-endian): int64 op, int64 ring, int64 descr_id, int64 m,
 * int64 n, int64 nnz, uint32 I[nnz], uint32 J[nnz], double V[nnz], then for
 * each of u, v, umask, vmask: int64 length, double values[length],
 * uint8 assigned[length] (length 0 = absent).
 *   op 0: mxv, 1: vxm, 2: conjugate_gradient (u = x0, v = b), 3: simple_pagerank,
 *   op 4: BLAS1 script on u, v (dot, folds, eWiseApply, eWiseMul, eWiseMulAdd, set)
 *   op 5: matrix-to-matrix set and ALP's capacity contract (default capacity,
 *         too small a capacity, the RESIZE phase, an empty source)
 *   op 6: integer BLAS1 on m entries with values from a seeded hash (size_t
 *         values above 2^53, int values near the ends of their range): dot,
 *         folds, eWiseApply, eWiseMul(Add) and set over size_t and int, printed
 *         as hexadecimal so that both builds are compared bit for bit
 *   ring 0: plus-times double, 1: lor-land bool, 2: min-plus int
 */
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include <graphblas.hpp>
#include <graphblas/algorithms/conjugate_gradient.hpp>
#include <graphblas/algorithms/simple_pagerank.hpp>

using namespace grb;

struct Arr {
	std::vector< double > v;
	std::vector< uint8_t > a;
};

struct Case {
	int64_t op, ring, descr, m, n, nnz;
	std::vector< uint32_t > I, J;
	std::vector< double > V;
	Arr u, v, um, vm;
};

static bool read_case( const char *path, Case &c ) {
	std::ifstream f( path, std::ios::binary );
	if( !f ) { return false; }
	auto rd = [ &f ]( void *p, size_t b ) { f.read( static_cast< char * >( p ), b ); };
	rd( &c.op, 8 ); rd( &c.ring, 8 ); rd( &c.descr, 8 ); rd( &c.m, 8 ); rd( &c.n, 8 ); rd( &c.nnz, 8 );
	c.I.resize( c.nnz ); c.J.resize( c.nnz ); c.V.resize( c.nnz );
	rd( c.I.data(), 4 * c.nnz ); rd( c.J.data(), 4 * c.nnz ); rd( c.V.data(), 8 * c.nnz );
	for( Arr *a : { &c.u, &c.v, &c.um, &c.vm } ) {
		int64_t len = 0;
		rd( &len, 8 );
		a->v.resize( len );
		a->a.resize( len );
		rd( a->v.data(), 8 * len );
		rd( a->a.data(), len );
	}
	return bool( f );
}

template< typename T >
static RC load( Vector< T > &x, const Arr &a ) {
	RC rc = clear( x );
	for( size_t i = 0; rc == SUCCESS && i < a.v.size(); ++i ) {
		if( a.a[ i ] ) { rc = setElement( x, static_cast< T >( a.v[ i ] ), i ); }
	}
	return rc;
}

template< typename T >
static void print( const char *tag, const Vector< T > &x ) {
	const size_t n = size( x );
	std::vector< double > val( n, 0.0 );
	std::vector< int > has( n, 0 );
	for( const auto &p : x ) {
		val[ p.first ] = static_cast< double >( p.second );
		has[ p.first ] = 1;
	}
	std::printf( "%s nnz %zu\n", tag, nnz( x ) );
	for( size_t i = 0; i < n; ++i ) {
		if( has[ i ] ) { std::printf( "%s %zu %.17g\n", tag, i, val[ i ] ); }
	}
}

template< Descriptor d, typename T, class Ring >
static RC spmv( bool vxm_form, Vector< T > &u, const Vector< bool > &um, const Matrix< T > &A,
	const Vector< T > &v, const Vector< bool > &vm, const Ring &ring
) {
	if( vxm_form ) { return grb::vxm< d >( u, um, v, vm, A, ring ); }
	return grb::mxv< d >( u, um, A, v, vm, ring );
}

template< typename T, class Ring >
static RC run_spmv( const Case &c, const Ring &ring ) {
	const bool vx = c.op == 1;
	Matrix< T > A( c.m, c.n );
	// std::vector< bool > has no data(): keep the values in a plain array
	std::unique_ptr< T[] > vals( new T[ c.nnz > 0 ? c.nnz : 1 ] );
	for( int64_t k = 0; k < c.nnz; ++k ) { vals[ k ] = static_cast< T >( c.V[ k ] ); }
	RC rc = buildMatrixUnique( A, c.I.data(), c.J.data(), vals.get(), c.nnz, SEQUENTIAL );
	Vector< T > u( c.u.v.size() ), v( c.v.v.size() );
	Vector< bool > um( c.um.v.size() ), vm( c.vm.v.size() );
	rc = rc ? rc : load( u, c.u );
	rc = rc ? rc : load( v, c.v );
	rc = rc ? rc : load( um, c.um );
	rc = rc ? rc : load( vm, c.vm );
	if( rc != SUCCESS ) { return rc; }
	using namespace descriptors;
	switch( c.descr ) {
		case 0: rc = spmv< no_operation >( vx, u, um, A, v, vm, ring ); break;
		case 1: rc = spmv< invert_mask >( vx, u, um, A, v, vm, ring ); break;
		case 2: rc = spmv< structural >( vx, u, um, A, v, vm, ring ); break;
		case 3: rc = spmv< structural | invert_mask >( vx, u, um, A, v, vm, ring ); break;
		case 4: rc = spmv< add_identity >( vx, u, um, A, v, vm, ring ); break;
		case 5: rc = spmv< explicit_zero >( vx, u, um, A, v, vm, ring ); break;
		case 6: rc = spmv< transpose_matrix >( vx, u, um, A, v, vm, ring ); break;
		case 7: rc = spmv< dense >( vx, u, um, A, v, vm, ring ); break;
		default: return ILLEGAL;
	}
	std::printf( "rc %d\n", int( rc ) );
	print( "u", u );
	return SUCCESS;
}

static RC run_cg( const Case &c ) {
	Matrix< double > A( c.m, c.n );
	RC rc = buildMatrixUnique( A, c.I.data(), c.J.data(), c.V.data(), c.nnz, SEQUENTIAL );
	Vector< double > x( c.m ), b( c.m ), r( c.m ), u( c.m ), t( c.m );
	rc = rc ? rc : load( x, c.u );
	rc = rc ? rc : load( b, c.v );
	size_t iters = 0;
	double res = 0;
	rc = rc ? rc : algorithms::conjugate_gradient( x, A, b, 500, 1e-10, iters, res, r, u, t );
	std::printf( "rc %d\niterations %zu\nresidual %.17g\n", int( rc ), iters, res );
	print( "x", x );
	return SUCCESS;
}

static RC run_pagerank( const Case &c ) {
	Matrix< double > L( c.m, c.n );
	RC rc = buildMatrixUnique( L, c.I.data(), c.J.data(), c.V.data(), c.nnz, SEQUENTIAL );
	Vector< double > pr( c.m ), a( c.m ), b( c.m ), rs( c.m );
	Vector< bool > dang( c.m );
	size_t iters = 0;
	double quality = 0;
	rc = rc ? rc : algorithms::simple_pagerank< descriptors::no_operation >( pr, L, a, b, rs, dang,
		0.85, 1e-9, 1000, &iters, &quality );
	std::printf( "rc %d\niterations %zu\n", int( rc ), iters );
	print( "pr", pr );
	return SUCCESS;
}

static RC run_blas1( const Case &c ) {
	const size_t n = c.u.v.size();
	Semiring< operators::add< double >, operators::mul< double >, identities::zero,
		identities::one > ring;
	Monoid< operators::add< double >, identities::zero > addM;
	Monoid< operators::max< double >, identities::negative_infinity > maxM;
	Vector< double > u( n ), v( n ), z( n ), w( n );
	Vector< bool > m( c.um.v.size() );
	RC rc = load( u, c.u );
	rc = rc ? rc : load( v, c.v );
	rc = rc ? rc : load( m, c.um );
	double d = 0.5;
	std::printf( "rc_dot %d\n", int( dot( d, u, v, ring ) ) );
	std::printf( "dot %.17g\n", d );
	double mx = -1;
	std::printf( "rc_fold %d\n", int( foldl( mx, u, maxM ) ) );
	std::printf( "fold_max %.17g\n", mx );
	double sm = 0;
	if( size( m ) == n ) {
		std::printf( "rc_mfold %d\n", int( foldl< descriptors::structural >( sm, v, m, addM ) ) );
		std::printf( "mfold %.17g\n", sm );
	}
	rc = set( z, u ) ? FAILED : foldl( z, v, operators::subtract< double >() );
	std::printf( "rc_foldl_op %d\n", int( rc ) );
	print( "foldl_op", z );
	rc = set( z, u ) ? FAILED : foldl( z, v, addM );
	std::printf( "rc_foldl_monoid %d\n", int( rc ) );
	print( "foldl_monoid", z );
	rc = set( z, u ) ? FAILED : foldr( v, z, operators::mul< double >() );
	std::printf( "rc_foldr_op %d\n", int( rc ) );
	print( "foldr_op", z );
	// on a dense vector: the sequential reference's unmasked scalar-into-vector
	// fold walks past the assigned count of a sparse vector (its
	// fold_from_scalar_to_vector_generic loop runs to n) and asserts
	rc = set( z, 1.5 ) ? FAILED : foldl( z, 2.5, operators::mul< double >() );
	std::printf( "rc_foldl_scalar %d\n", int( rc ) );
	print( "foldl_scalar", z );
	// the second operand is dense: with an operator, the reference's
	// sparse_apply_generic assigns every index of its tail block of the
	// sparser input even where the other input has no entry, and leaves the
	// value there unset (reference/blas1.hpp:3309-3352), which nothing can match
	rc = set( z, 0.25 ) ? FAILED : foldl( z, v, operators::right_assign< double >() );
	rc = rc ? rc : eWiseApply( w, u, z, operators::mul< double >() );
	std::printf( "rc_apply_op %d\n", int( rc ) );
	print( "apply_op", w );
	// again a dense second operand: with a monoid, an index held only by the
	// input that the reference loops over gets the OTHER input's (absent) raw
	// value (reference/blas1.hpp:3203-3211), which nothing can match
	rc = eWiseApply( w, u, z, addM );
	std::printf( "rc_apply_monoid %d\n", int( rc ) );
	print( "apply_monoid", w );
	rc = set( z, u ) ? FAILED : eWiseMul( z, 3.0, v, ring );
	std::printf( "rc_ewisemul %d\n", int( rc ) );
	print( "ewisemul", z );
	rc = set( z, 1.0 ) ? FAILED : eWiseMulAdd( z, 2.0, u, v, ring );
	std::printf( "rc_muladd %d\n", int( rc ) );
	print( "muladd", z );
	if( size( m ) == n ) {
		rc = set( z, u ) ? FAILED : set( z, m, 7.0 );
		std::printf( "rc_mset %d\n", int( rc ) );
		print( "mset", z );
		rc = clear( z ) ? FAILED : set( z, m, v );
		std::printf( "rc_mset_vec %d\n", int( rc ) );
		print( "mset_vec", z );
	}
	return SUCCESS;
}

template< typename T >
static void print_matrix( const char *tag, const Matrix< T > &A ) {
	std::vector< std::pair< std::pair< size_t, size_t >, double > > e;
	for( const auto &t : A ) {
		e.push_back( std::make_pair( std::make_pair( t.first.first, t.first.second ),
			static_cast< double >( t.second ) ) );
	}
	std::sort( e.begin(), e.end() );
	std::printf( "%s nnz %zu\n", tag, e.size() );
	for( size_t k = 0; k < e.size(); ++k ) {
		std::printf( "%s %zu %.17g\n", tag, k, e[ k ].second );
		std::printf( "%s_row %zu %zu\n", tag, k, e[ k ].first.first );
		std::printf( "%s_col %zu %zu\n", tag, k, e[ k ].first.second );
	}
}

static RC run_matrix_set( const Case &c ) {
	Matrix< double > A( c.m, c.n, c.nnz > 0 ? c.nnz : 1 );
	RC rc = buildMatrixUnique( A, c.I.data(), c.J.data(), c.V.data(), c.nnz, SEQUENTIAL );
	std::printf( "rc_build %d\nnnz_A %zu\n", int( rc ), nnz( A ) );
	// the default capacity is max( rows, columns )
	Matrix< double > D( c.m, c.n );
	std::printf( "cap_default_ok %d\n", int( capacity( D ) >= std::max( c.m, c.n ) ) );
	// too small a capacity: ILLEGAL, and the target is cleared
	Matrix< double > C( c.m, c.n, 1 );
	rc = buildMatrixUnique( C, c.I.data(), c.J.data(), c.V.data(), 1, SEQUENTIAL );
	std::printf( "rc_build_C %d\nnnz_C0 %zu\n", int( rc ), nnz( C ) );
	std::printf( "rc_set_small %d\n", int( set( C, A ) ) );
	std::printf( "nnz_C_small %zu\n", nnz( C ) );
	// RESIZE reserves; EXECUTE then copies
	std::printf( "rc_set_resize %d\n", int( set( C, A, RESIZE ) ) );
	std::printf( "cap_C_ok %d\n", int( capacity( C ) >= nnz( A ) ) );
	std::printf( "rc_set %d\n", int( set( C, A ) ) );
	print_matrix( "C", C );
	// an empty source clears the target
	Matrix< double > E( c.m, c.n );
	std::printf( "rc_set_empty %d\n", int( set( C, E ) ) );
	std::printf( "nnz_C_empty %zu\n", nnz( C ) );
	return SUCCESS;
}

static uint64_t mix64( uint64_t z ) {   // splitmix64 finaliser
	z += 0x9e3779b97f4a7c15ull;
	z = ( z ^ ( z >> 30 ) ) * 0xbf58476d1ce4e5b9ull;
	z = ( z ^ ( z >> 27 ) ) * 0x94d049bb133111ebull;
	return z ^ ( z >> 31 );
}

template< typename T >
static void print_hex( const char *tag, const T v ) {
	std::printf( "%s 0x%016llx\n", tag, static_cast< unsigned long long >(
		static_cast< uint64_t >( v ) ) );
}

template< typename T >
static void print_hex_vector( const char *tag, const Vector< T > &x ) {
	std::vector< std::pair< size_t, T > > e;
	for( const auto &p : x ) { e.push_back( p ); }
	std::sort( e.begin(), e.end() );
	std::printf( "%s_nnz %zu\n", tag, e.size() );
	for( const auto &p : e ) {
		std::printf( "%s_%zu 0x%016llx\n", tag, p.first, static_cast< unsigned long long >(
			static_cast< uint64_t >( p.second ) ) );
	}
}

static RC run_integer_blas1( const Case &c ) {
	const size_t n = static_cast< size_t >( c.m );
	Vector< size_t > u( n ), v( n ), z( n );
	Vector< int > a( n ), b( n ), w( n );
	RC rc = SUCCESS;
	for( size_t i = 0; rc == SUCCESS && i < n; ++i ) {
		// size_t values well above 2^53; ints within 1000 of INT_MAX / INT_MIN
		rc = setElement( u, mix64( 3 * i + 1 ) | ( size_t( 1 ) << 60 ), i );
		rc = rc ? rc : setElement( v, mix64( 3 * i + 2 ), i );
		const int64_t r = static_cast< int64_t >( mix64( 3 * i + 3 ) % 2000 );
		rc = rc ? rc : setElement( a, static_cast< int >( i % 2 ? 2147483647 - r : -2147483647 + r ), i );
		rc = rc ? rc : setElement( b, static_cast< int >( r - 1000 ), i );
	}
	std::printf( "rc_load %d\n", int( rc ) );
	Semiring< operators::add< size_t >, operators::mul< size_t >, identities::zero,
		identities::one > ringU;
	Semiring< operators::add< int >, operators::mul< int >, identities::zero,
		identities::one > ringI;
	Semiring< operators::min< int >, operators::add< int >, identities::infinity,
		identities::zero > minPlus;
	Monoid< operators::add< size_t >, identities::zero > addU;
	Monoid< operators::max< size_t >, identities::negative_infinity > maxU;
	Monoid< operators::min< size_t >, identities::infinity > minU;
	Monoid< operators::add< int >, identities::zero > addI;
	size_t du = 7;
	std::printf( "rc_dot_u64 %d\n", int( dot( du, u, v, ringU ) ) );
	print_hex( "dot_u64", du );
	size_t su = 0, mu = 0, nu = 0;
	std::printf( "rc_fold_u64 %d\n", int( foldl( su, u, addU ) ) );
	print_hex( "fold_add_u64", su );
	std::printf( "rc_fold_max_u64 %d\n", int( foldl( mu, v, maxU ) ) );
	print_hex( "fold_max_u64", mu );
	nu = ~size_t( 0 );
	std::printf( "rc_fold_min_u64 %d\n", int( foldl( nu, v, minU ) ) );
	print_hex( "fold_min_u64", nu );
	int di = 0, si = 0;
	std::printf( "rc_dot_i32 %d\n", int( dot( di, a, b, ringI ) ) );
	print_hex( "dot_i32", di );
	std::printf( "rc_fold_i32 %d\n", int( foldl( si, a, addI ) ) );
	print_hex( "fold_add_i32", si );
	rc = eWiseApply( z, u, v, operators::add< size_t >() );
	std::printf( "rc_apply_u64 %d\n", int( rc ) );
	print_hex_vector( "apply_u64", z );
	rc = set( z, u ) ? FAILED : foldl( z, v, operators::mul< size_t >() );
	std::printf( "rc_foldl_u64 %d\n", int( rc ) );
	print_hex_vector( "foldl_u64", z );
	rc = set( z, ~size_t( 0 ) - 5 );
	std::printf( "rc_set_u64 %d\n", int( rc ) );
	print_hex_vector( "set_u64", z );
	rc = set( z, u ) ? FAILED : eWiseMul( z, v, u, ringU );
	std::printf( "rc_mul_u64 %d\n", int( rc ) );
	print_hex_vector( "mul_u64", z );
	rc = eWiseApply( w, a, b, operators::add< int >() );
	std::printf( "rc_apply_i32 %d\n", int( rc ) );
	print_hex_vector( "apply_i32", w );
	Vector< int > c3( n );
	rc = set( w, a ) ? FAILED : ( set( c3, b ) ? FAILED : eWiseMulAdd( w, a, b, c3, minPlus ) );
	std::printf( "rc_minplus_i32 %d\n", int( rc ) );
	print_hex_vector( "minplus_i32", w );
	return SUCCESS;
}

int main( int argc, char **argv ) {
	if( argc != 2 ) {
		std::cerr << "usage: " << argv[ 0 ] << " <case file>\n";
		return 2;
	}
	Case c;
	if( !read_case( argv[ 1 ], c ) ) {
		std::cerr << "cannot read " << argv[ 1 ] << "\n";
		return 2;
	}
	if( grb::init() != SUCCESS ) { return 3; }
	RC rc = SUCCESS;
	if( c.op <= 1 ) {
		if( c.ring == 0 ) {
			rc = run_spmv< double >( c, Semiring< operators::add< double >, operators::mul< double >,
				identities::zero, identities::one >() );
		} else if( c.ring == 1 ) {
			rc = run_spmv< bool >( c, Semiring< operators::logical_or< bool >,
				operators::logical_and< bool >, identities::logical_false, identities::logical_true >() );
		} else {
			rc = run_spmv< int >( c, Semiring< operators::min< int >, operators::add< int >,
				identities::infinity, identities::zero >() );
		}
	} else if( c.op == 2 ) {
		rc = run_cg( c );
	} else if( c.op == 3 ) {
		rc = run_pagerank( c );
	} else if( c.op == 5 ) {
		rc = run_matrix_set( c );
	} else if( c.op == 6 ) {
		rc = run_integer_blas1( c );
	} else {
		rc = run_blas1( c );
	}
	(void) grb::finalize();
	return rc == SUCCESS ? 0 : 1;
}
