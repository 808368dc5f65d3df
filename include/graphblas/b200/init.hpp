/* grb::init / grb::finalize for the b200 backend: select and initialise the
 * CUDA device (the reference's are src/graphblas/reference/init.cpp:45-113). */
#ifndef _H_GRB_B200_INIT
#define _H_GRB_B200_INIT

#include <cstdlib>

#include <graphblas/base/init.hpp>
#include <graphblas/b200/runtime.hpp>

namespace grb {

	/** Uses the device named by ALPB_DEVICE (default 0); s = 0, P = 1 only. */
	template<>
	inline RC init< b200 >( const size_t s, const size_t P, void * const data ) {
		(void) data;
		if( s != 0 || P != 1 ) { return UNSUPPORTED; }
		const char * const dev = std::getenv( "ALPB_DEVICE" );
		return internal::b200rt::check( alpb_init( dev ? std::atoi( dev ) : 0 ), "grb::init" );
	}

	template<>
	inline RC finalize< b200 >() {
		return internal::b200rt::check( alpb_finalize(), "grb::finalize" );
	}

}

#endif
