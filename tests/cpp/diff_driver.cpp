/*
 * Driver of the differentiated solvers in the b200 C++ API
 * (graphblas/b200/algorithms.hpp), for the parity tests.  The forward CG is
 * ALP's own algorithms::conjugate_gradient, compiled unchanged for b200.
 *
 *   diff_driver cg  <dir>   A.bin, b.bin, xstar.bin  ->  x.bin, lambda.bin, grad.bin, order.bin
 *   diff_driver ppr <dir>   W.bin, seeds.bin, g.bin  ->  X.bin, Lambda.bin, grad.bin, order.bin
 *
 * Matrix files: int64 n, int64 nnz, uint32 I[nnz], uint32 J[nnz], double V[nnz].
 * seeds.bin: int64 S, int64 seeds[S].  Vectors: raw doubles.  order.bin holds
 * the (uint32 i, uint32 j) of each stored entry in the order the matrix
 * iterator visits them (the order of grad.bin).  CG: L = 0.5 ||x - x*||^2,
 * tolerance 1e-12; PageRank: alpha 0.85, conv 1e-10, dL/dX = g.
 */
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include <graphblas.hpp>
#include <graphblas/algorithms/conjugate_gradient.hpp>
#include <graphblas/b200/algorithms.hpp>

using namespace grb;

template< typename T >
static bool read_raw( const std::string &path, std::vector< T > &v, size_t count ) {
	std::ifstream f( path, std::ios::binary );
	v.resize( count );
	f.read( reinterpret_cast< char * >( v.data() ), count * sizeof( T ) );
	return bool( f );
}

struct Coo {
	int64_t n = 0, nnz = 0;
	std::vector< uint32_t > I, J;
	std::vector< double > V;
};

static bool read_coo( const std::string &path, Coo &c ) {
	std::ifstream f( path, std::ios::binary );
	f.read( reinterpret_cast< char * >( &c.n ), 8 );
	f.read( reinterpret_cast< char * >( &c.nnz ), 8 );
	c.I.resize( c.nnz );
	c.J.resize( c.nnz );
	c.V.resize( c.nnz );
	f.read( reinterpret_cast< char * >( c.I.data() ), 4 * c.nnz );
	f.read( reinterpret_cast< char * >( c.J.data() ), 4 * c.nnz );
	f.read( reinterpret_cast< char * >( c.V.data() ), 8 * c.nnz );
	return bool( f );
}

static void write_vec( const std::string &path, const Vector< double > &x ) {
	std::vector< double > h( size( x ), 0.0 );
	for( const auto &p : x ) { h[ p.first ] = p.second; }
	std::ofstream f( path, std::ios::binary );
	f.write( reinterpret_cast< const char * >( h.data() ), h.size() * 8 );
}

static void write_order( const std::string &path, const Matrix< double > &A ) {
	std::vector< uint32_t > ij;
	for( const auto &p : A ) {
		ij.push_back( static_cast< uint32_t >( p.first.first ) );
		ij.push_back( static_cast< uint32_t >( p.first.second ) );
	}
	std::ofstream f( path, std::ios::binary );
	f.write( reinterpret_cast< const char * >( ij.data() ), ij.size() * 4 );
}

static RC load( Vector< double > &x, const std::vector< double > &v ) {
	return buildVector( x, v.begin(), v.end(), SEQUENTIAL );
}

static int run_cg( const std::string &dir ) {
	Coo c;
	if( !read_coo( dir + "/A.bin", c ) ) { return 2; }
	const size_t n = c.n;
	std::vector< double > hb, hxs;
	if( !read_raw( dir + "/b.bin", hb, n ) || !read_raw( dir + "/xstar.bin", hxs, n ) ) { return 2; }
	Matrix< double > A( n, n );
	RC rc = buildMatrixUnique( A, c.I.data(), c.J.data(), c.V.data(), c.nnz, SEQUENTIAL );
	Vector< double > x( n ), b( n ), xs( n ), g( n ), r( n ), u( n ), t( n ), lam( n ),
		grad( nnz( A ) );
	rc = rc ? rc : load( b, hb );
	rc = rc ? rc : load( xs, hxs );
	rc = rc ? rc : set( x, 0.0 );
	size_t itf = 0, ita = 0;
	double res = 0;
	rc = rc ? rc : algorithms::conjugate_gradient( x, A, b, 5000, 1e-12, itf, res, r, u, t );
	rc = rc ? rc : set( g, 0.0 );
	rc = rc ? rc : eWiseApply( g, x, xs, operators::subtract< double >() );
	rc = rc ? rc : algorithms::conjugate_gradient_adjoint( lam, grad, A, x, g, 5000, 1e-12, ita,
		res );
	std::printf( "rc %d\niterations_fwd %zu\niterations_adj %zu\n", int( rc ), itf, ita );
	if( rc != SUCCESS ) { return 1; }
	write_vec( dir + "/x.bin", x );
	write_vec( dir + "/lambda.bin", lam );
	write_vec( dir + "/grad.bin", grad );
	write_order( dir + "/order.bin", A );
	return 0;
}

static int run_ppr( const std::string &dir ) {
	Coo c;
	if( !read_coo( dir + "/W.bin", c ) ) { return 2; }
	const size_t n = c.n;
	std::ifstream fs( dir + "/seeds.bin", std::ios::binary );
	int64_t S = 0;
	fs.read( reinterpret_cast< char * >( &S ), 8 );
	std::vector< int64_t > sd( S );
	fs.read( reinterpret_cast< char * >( sd.data() ), 8 * S );
	std::vector< double > hg;
	if( !fs || !read_raw( dir + "/g.bin", hg, n * S ) ) { return 2; }
	Matrix< double > W( n, n );
	RC rc = buildMatrixUnique( W, c.I.data(), c.J.data(), c.V.data(), c.nnz, SEQUENTIAL );
	if( rc != SUCCESS ) { return 1; }
	Vector< double > X( n * S ), G( n * S ), L( n * S ), grad( nnz( W ) );
	rc = load( G, hg );
	algorithms::PersonalisedPageRank<> ppr( W, S );
	rc = rc ? rc : ppr.status();
	std::vector< size_t > seeds( sd.begin(), sd.end() ), itf, ita;
	rc = rc ? rc : ppr.solve( X, seeds, 0.85, 1e-10, 1000, false, &itf );
	rc = rc ? rc : ppr.adjoint( L, G, 1e-10, 1000, &ita );
	rc = rc ? rc : ppr.gradient( grad, X, L );
	std::printf( "rc %d\n", int( rc ) );
	for( size_t s = 0; s < itf.size(); ++s ) { std::printf( "iterations_fwd %zu\n", itf[ s ] ); }
	for( size_t s = 0; s < ita.size(); ++s ) { std::printf( "iterations_adj %zu\n", ita[ s ] ); }
	if( rc != SUCCESS ) { return 1; }
	write_vec( dir + "/X.bin", X );
	write_vec( dir + "/Lambda.bin", L );
	write_vec( dir + "/grad.bin", grad );
	write_order( dir + "/order.bin", W );
	return 0;
}

int main( int argc, char **argv ) {
	if( argc != 3 ) {
		std::cerr << "usage: " << argv[ 0 ] << " cg|ppr <dir>\n";
		return 2;
	}
	if( grb::init() != SUCCESS ) { return 3; }
	const std::string what = argv[ 1 ];
	int ret = 2;
	{
		if( what == "cg" ) { ret = run_cg( argv[ 2 ] ); }
		else if( what == "ppr" ) { ret = run_ppr( argv[ 2 ] ); }
	}
	(void) grb::finalize();
	return ret;
}
