/* Level-3 primitives (SpGEMM, matrix eWiseApply, select) are outside the
 * b200 hot path: they keep the base specification, which returns UNSUPPORTED. */
#ifndef _H_GRB_B200_BLAS3
#define _H_GRB_B200_BLAS3
#endif
