/* Launcher of the b200 backend: one user process, the program runs on the
 * host and drives the device (reference: graphblas/reference/exec.hpp:38-132). */
#ifndef _H_GRB_B200_EXEC
#define _H_GRB_B200_EXEC

#include <stdexcept>
#include <string>

#include <graphblas/base/exec.hpp>
#include <graphblas/init.hpp>

namespace grb {

	template< EXEC_MODE mode >
	class Launcher< mode, b200 > {

		protected:

			template< typename Runner >
			RC init_and_run( Runner &runner, const bool ) const {
				RC ret = grb::init< b200 >();
				if( ret == SUCCESS ) {
					runner();
					ret = grb::finalize< b200 >();
				}
				return ret;
			}

		public:

			Launcher( const size_t process_id = 0, const size_t nprocs = 1,
				const std::string hostname = "localhost", const std::string port = "0"
			) {
				(void) hostname;
				(void) port;
				if( nprocs != 1 || process_id != 0 ) {
					throw std::invalid_argument( "the b200 backend runs one user process per GPU" );
				}
			}

			template< typename U >
			RC exec( AlpUntypedFunc< U > alp_program, const void * const data_in,
				const size_t in_size, U &data_out, const bool broadcast = false
			) const {
				if( in_size > 0 && data_in == nullptr ) { return ILLEGAL; }
				auto fun = [ data_in, in_size, &data_out, alp_program ] {
					(*alp_program)( data_in, in_size, data_out );
				};
				return init_and_run( fun, broadcast );
			}

			template< typename T, typename U >
			RC exec( AlpTypedFunc< T, U > alp_program, const T &data_in, U &data_out,
				const bool broadcast = false
			) {
				auto fun = [ &data_in, &data_out, alp_program ] {
					(*alp_program)( data_in, data_out );
				};
				return init_and_run( fun, broadcast );
			}

			static RC finalize() { return SUCCESS; }
	};

}

#endif
