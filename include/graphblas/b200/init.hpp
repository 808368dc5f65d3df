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

	/** Runs pending fused level-1 steps; with ALPB_TRACE set, one line on
	 *  stderr with the fusion count and the kernels launched. */
	template<>
	inline RC finalize< b200 >() {
		(void) alpb_stream_sync( internal::b200rt::stream() );
		if( std::getenv( "ALPB_TRACE" ) != nullptr ) {
			const internal::b200rt::Chain &c = internal::b200rt::chain();
			std::cerr << "grb::b200: fused level-1 passes " << c.runs << " for " << c.fused_steps
				<< " steps, kernel launches " << alpb_launch_count() << "\n";
		}
		return internal::b200rt::check( alpb_finalize(), "grb::finalize" );
	}

}

#endif
