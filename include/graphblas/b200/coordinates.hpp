/*
 * Sparsity bookkeeping of a b200 vector (reference:
 * graphblas/reference/coordinates.hpp:61-1500, a bool array plus a stack of
 * assigned indices).  On the device the b200 vector keeps one assigned flag
 * per entry and a device counter of assigned entries; the order of assigned
 * indices is not observable through the API, so no stack is kept.  This
 * class is the Coords template argument of Vector<D, b200, Coords>.
 */
#ifndef _H_GRB_B200_COORDINATES
#define _H_GRB_B200_COORDINATES

#include <cstddef>
#include <cstdint>

#include <graphblas/backends.hpp>
#include <graphblas/base/coordinates.hpp>

namespace grb {

	namespace internal {

		template<>
		class Coordinates< b200 > {
			public:
				/** The b200 vector holds its own flags; this type is a tag. */
				static constexpr bool device_resident = true;
		};

	}

}

#endif
