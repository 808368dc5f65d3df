/*
 * MatrixMarket ingest checker: reads one file through ALP's own reader
 * (grb::utils::MatrixFileReader + buildMatrixUnique) on the backend it is
 * compiled for, and on b200 also through buildMatrixUniqueFromFile (the
 * file parsed by every host core, the storage built on the device); prints
 * each matrix's entries in sorted order and one product y = A x, so that the
 * two paths and the reference build can be compared line by line.
 *
 *   mm_driver <file.mtx> <pattern: 0|1>
 */
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include <graphblas.hpp>
#include <graphblas/utils/parser.hpp>

using namespace grb;

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

template< typename T >
static void product( const char *tag, const Matrix< T > &A ) {
	const size_t m = nrows( A ), n = ncols( A );
	Vector< double > x( n ), y( m );
	for( size_t j = 0; j < n; ++j ) { (void) setElement( x, 0.5 * double( j + 1 ), j ); }
	(void) set( y, 0.0 );
	Semiring< operators::add< double >, operators::mul< double >, identities::zero,
		identities::one > ring;
	const RC rc = mxv( y, A, x, ring );
	std::printf( "%s_rc %d\n", tag, int( rc ) );
	for( const auto &p : y ) { std::printf( "%s_y %zu %.17g\n", tag, p.first, p.second ); }
}

int main( int argc, char **argv ) {
	if( argc != 3 ) {
		std::fprintf( stderr, "usage: %s <file.mtx> <pattern: 0|1>\n", argv[ 0 ] );
		return 2;
	}
	const std::string path = argv[ 1 ];
	if( grb::init() != SUCCESS ) { return 3; }
	grb::utils::MatrixFileReader< double, size_t > parser( path, true );
	Matrix< double > A( parser.m(), parser.n() );
	RC rc = buildMatrixUnique( A, parser.begin( SEQUENTIAL ), parser.end( SEQUENTIAL ), SEQUENTIAL );
	std::printf( "rc_reader %d\n", int( rc ) );
	print_matrix( "A", A );
	product( "A", A );
#ifdef _GRB_WITH_B200
	Matrix< double > B( parser.m(), parser.n() );
	rc = buildMatrixUniqueFromFile( B, path );
	std::fprintf( stderr, "rc_file %d\n", int( rc ) );
	// the device-ingested matrix, under the same tags as ALP's reader path
	// on the other build, on stderr
	std::vector< std::pair< std::pair< size_t, size_t >, double > > e;
	for( const auto &t : B ) {
		e.push_back( std::make_pair( std::make_pair( t.first.first, t.first.second ), t.second ) );
	}
	std::sort( e.begin(), e.end() );
	std::fprintf( stderr, "A nnz %zu\n", e.size() );
	for( size_t k = 0; k < e.size(); ++k ) {
		std::fprintf( stderr, "A %zu %.17g\nA_row %zu %zu\nA_col %zu %zu\n", k, e[ k ].second, k,
			e[ k ].first.first, k, e[ k ].first.second );
	}
	{
		const size_t m = nrows( B ), n = ncols( B );
		Vector< double > x( n ), y( m );
		for( size_t j = 0; j < n; ++j ) { (void) setElement( x, 0.5 * double( j + 1 ), j ); }
		(void) set( y, 0.0 );
		Semiring< operators::add< double >, operators::mul< double >, identities::zero,
			identities::one > ring;
		const RC r2 = mxv( y, B, x, ring );
		std::fprintf( stderr, "A_rc %d\n", int( r2 ) );
		for( const auto &p : y ) { std::fprintf( stderr, "A_y %zu %.17g\n", p.first, p.second ); }
	}
	std::fprintf( stderr, "rc_reader %d\n", int( rc == SUCCESS ? SUCCESS : rc ) );
	if( argv[ 2 ][ 0 ] == '1' ) {
		Matrix< void > P( parser.m(), parser.n() );
		const RC r3 = buildMatrixUniqueFromFile( P, path );
		std::fprintf( stderr, "pattern_rc %d\npattern_nnz %zu\n", int( r3 ), nnz( P ) );
	}
#endif
	(void) grb::finalize();
	return 0;
}
