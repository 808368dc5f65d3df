/* Single user process per GPU (reference: graphblas/reference/spmd.hpp). */
#ifndef _H_GRB_B200_SPMD
#define _H_GRB_B200_SPMD

#include <graphblas/base/spmd.hpp>

namespace grb {

	template<>
	class spmd< b200 > {
		public:
			static inline size_t nprocs() noexcept { return 1; }
			static inline size_t pid() noexcept { return 0; }
			static RC sync( const size_t = 0, const size_t = 0 ) noexcept { return SUCCESS; }
			static RC barrier() noexcept { return SUCCESS; }
	};

}

#endif
