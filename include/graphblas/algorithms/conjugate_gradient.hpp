/*
 * Overlay of ALP's graphblas/algorithms/conjugate_gradient.hpp: ALP's header is included
 * unchanged (include_next finds it in the ALP include tree, which follows
 * this directory on the include path), then, with -D_GRB_WITH_B200, the b200
 * overload of conjugate_gradient, which runs the fused device solver for
 * b200 containers (graphblas/b200/fused_cg.hpp).
 */
#ifndef ALPB_OVERLAY_ALGORITHMS_CG_HPP
#define ALPB_OVERLAY_ALGORITHMS_CG_HPP

#include_next <graphblas/algorithms/conjugate_gradient.hpp>

#ifdef _GRB_WITH_B200
 #include <graphblas/b200/fused_cg.hpp>
#endif

#endif
