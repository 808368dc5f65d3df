/* Compile-time configuration of the b200 backend (the reference's is
 * graphblas/reference/config.hpp:145-190). */
#ifndef _H_GRB_B200_CONFIG
#define _H_GRB_B200_CONFIG

#include <graphblas/base/config.hpp>

namespace grb {

	namespace config {

		template<>
		class IMPLEMENTATION< b200 > {
			public:
				/** Vector capacities equal their sizes. */
				static constexpr bool fixedVectorCapacities() { return true; }
				static constexpr size_t vectorBufferSize( const size_t, const size_t ) { return 0; }
				static constexpr Backend coordinatesBackend() { return b200; }
		};

	}

}

#endif
