/*
 * HPCG checker: runs grb::algorithms::hpcg unchanged on the backend it is
 * compiled for (the reference backend for the parity tests), on the system
 * build_hpcg_system makes, and prints the outcome for the device solver to be
 * compared with.
 *
 *   hpcg_driver nx ny nz max_levels colors pre post max_iter tol precondition
 *               rhs_file|- x_out_file
 *
 * rhs_file holds nx*ny*nz doubles (native byte order); "-" takes b = A 1.
 * x starts at zero.  Prints "iterations N" and "residual R" (||r||), and
 * writes x to x_out_file.
 */
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include <graphblas.hpp>
#include <graphblas/algorithms/hpcg/hpcg.hpp>
#include <graphblas/algorithms/hpcg/system_building_utils.hpp>

using namespace grb;
using namespace grb::algorithms;

struct Args {
	size_t nx, ny, nz, levels, colors, pre, post, max_iter;
	double tol;
	bool precondition;
	const char *rhs, *xout;
};

struct Out {
	int rc = 0;
	size_t iterations = 0;
	double residual = 0;
};

static void program( const Args &in, Out &out ) {
	const std::array< size_t, 3 > sizes = { in.nx, in.ny, in.nz };
	hpcg_system_params< 3, double > params {
		sizes, 1, in.colors, 26.0, -1.0, 4, in.levels, 2
	};
	std::unique_ptr< hpcg_data< double, double, double > > data;
	RC rc = build_hpcg_system< 3, double >( data, params );
	const size_t n = in.nx * in.ny * in.nz;
	Semiring< operators::add< double >, operators::mul< double >, identities::zero,
		identities::one > ring;
	if( rc == SUCCESS ) {
		if( in.rhs[ 0 ] == '-' && in.rhs[ 1 ] == 0 ) {
			rc = set( data->x, 1.0 );
			rc = rc ? rc : set( data->b, 0.0 );
			rc = rc ? rc : mxv( data->b, data->A, data->x, ring );
		} else {
			std::vector< double > b( n );
			FILE *f = std::fopen( in.rhs, "rb" );
			if( !f || std::fread( b.data(), sizeof( double ), n, f ) != n ) { rc = FAILED; }
			if( f ) { std::fclose( f ); }
			for( size_t i = 0; rc == SUCCESS && i < n; ++i ) { rc = setElement( data->b, b[ i ], i ); }
		}
	}
	rc = rc ? rc : set( data->x, 0.0 );
	size_t iterations = 0;
	double residual = 0.0;
	rc = rc ? rc : hpcg( *data, in.precondition, in.pre, in.post, in.max_iter, in.tol, iterations,
		residual );
	out.rc = int( rc );
	out.iterations = iterations;
	out.residual = residual;
	if( rc == SUCCESS ) {
		std::vector< double > x( n, 0.0 );
		for( const auto &pair : data->x ) { x[ pair.first ] = pair.second; }
		FILE *f = std::fopen( in.xout, "wb" );
		if( f ) {
			std::fwrite( x.data(), sizeof( double ), n, f );
			std::fclose( f );
		} else {
			out.rc = int( FAILED );
		}
	}
}

int main( int argc, char **argv ) {
	if( argc != 13 ) {
		std::fprintf( stderr, "usage: %s nx ny nz max_levels colors pre post max_iter tol "
			"precondition rhs_file|- x_out_file\n", argv[ 0 ] );
		return 2;
	}
	Args in;
	in.nx = std::strtoul( argv[ 1 ], nullptr, 10 );
	in.ny = std::strtoul( argv[ 2 ], nullptr, 10 );
	in.nz = std::strtoul( argv[ 3 ], nullptr, 10 );
	in.levels = std::strtoul( argv[ 4 ], nullptr, 10 );
	in.colors = std::strtoul( argv[ 5 ], nullptr, 10 );
	in.pre = std::strtoul( argv[ 6 ], nullptr, 10 );
	in.post = std::strtoul( argv[ 7 ], nullptr, 10 );
	in.max_iter = std::strtoul( argv[ 8 ], nullptr, 10 );
	in.tol = std::strtod( argv[ 9 ], nullptr );
	in.precondition = std::strtoul( argv[ 10 ], nullptr, 10 ) != 0;
	in.rhs = argv[ 11 ];
	in.xout = argv[ 12 ];
	Out out;
	Launcher< AUTOMATIC > launcher;
	if( launcher.exec( &program, in, out, true ) != SUCCESS ) {
		std::fprintf( stderr, "launch failed\n" );
		return 1;
	}
	std::printf( "rc %d\niterations %zu\nresidual %.17g\n", out.rc, out.iterations, out.residual );
	return out.rc == 0 ? 0 : 1;
}
