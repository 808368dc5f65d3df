/* Properties of the b200 backend (reference: graphblas/reference/properties.hpp:36-56).
 * Lambdas given to eWiseLambda run on the host over mirrored values, so they
 * may not write captured scalars that the algorithm then reads as reductions:
 * writableCaptured is false, which sends simple_pagerank down its
 * primitive-only branch. */
#ifndef _H_GRB_B200_PROPERTIES
#define _H_GRB_B200_PROPERTIES

#include <graphblas/base/properties.hpp>

namespace grb {

	template<>
	class Properties< b200 > {
		public:
			static constexpr const bool writableCaptured = false;
			static constexpr const bool isBlockingExecution = true;
			static constexpr const bool isNonblockingExecution = false;
	};

}

#endif
