/* Collectives over one process are identities (reference:
 * graphblas/reference/collectives.hpp:82-140). */
#ifndef _H_GRB_B200_COLLECTIVES
#define _H_GRB_B200_COLLECTIVES

#include <graphblas/base/collectives.hpp>

namespace grb {

	template<>
	class collectives< b200 > {
		private:
			collectives() {}
		public:
			template< Descriptor descr = descriptors::no_operation, class Operator, typename IOType >
			static RC allreduce( IOType &, const Operator = Operator() ) { return SUCCESS; }
			template< Descriptor descr = descriptors::no_operation, class Operator, typename IOType >
			static RC reduce( IOType &, const size_t root = 0, const Operator = Operator() ) {
				return root == 0 ? SUCCESS : ILLEGAL;
			}
			template< typename IOType >
			static RC broadcast( IOType &, const size_t root = 0 ) {
				return root == 0 ? SUCCESS : ILLEGAL;
			}
			template< Descriptor descr = descriptors::no_operation, typename IOType >
			static RC broadcast( IOType *, const size_t, const size_t root = 0 ) {
				return root == 0 ? SUCCESS : ILLEGAL;
			}
	};

}

#endif
