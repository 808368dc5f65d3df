/* No b200-specific blas0 specialisations: ALP's scalar operations are generic. */
#ifndef _H_GRB_B200_BLAS0
#define _H_GRB_B200_BLAS0
#endif
