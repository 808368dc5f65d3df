/* Benchmarker of the b200 backend (reference: graphblas/reference/benchmark.hpp). */
#ifndef _H_GRB_B200_BENCHMARK
#define _H_GRB_B200_BENCHMARK

#include <graphblas/base/benchmark.hpp>
#include <graphblas/b200/exec.hpp>

namespace grb {

	template< EXEC_MODE mode >
	class Benchmarker< mode, b200 > :
		public Launcher< mode, b200 >, protected internal::BenchmarkerBase
	{
		public:
			using Launcher< mode, b200 >::Launcher;

			template< typename U >
			RC exec( AlpUntypedFunc< U > alp_program, const void * data_in,
				const size_t in_size, U &data_out, const size_t inner, const size_t outer,
				const bool broadcast = false
			) const {
				if( in_size > 0 && data_in == nullptr ) { return ILLEGAL; }
				auto fun = [ data_in, in_size, &data_out, alp_program, inner, outer ] {
					benchmark< U, b200 >( alp_program, data_in, in_size, data_out, inner, outer, 0 );
				};
				return Launcher< mode, b200 >::init_and_run( fun, broadcast );
			}

			template< typename T, typename U >
			RC exec( AlpTypedFunc< T, U > alp_program, const T &data_in, U &data_out,
				const size_t inner, const size_t outer, const bool broadcast = false
			) {
				auto fun = [ &data_in, &data_out, alp_program, inner, outer ] {
					benchmark< T, U, b200 >( alp_program, data_in, data_out, inner, outer, 0 );
				};
				return Launcher< mode, b200 >::init_and_run( fun, broadcast );
			}

			using Launcher< mode, b200 >::finalize;
	};

}

#endif
