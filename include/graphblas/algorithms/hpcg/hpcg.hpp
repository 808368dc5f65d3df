/*
 * Overlay of ALP's graphblas/algorithms/hpcg/hpcg.hpp: ALP's header is
 * included unchanged (include_next finds it in the ALP include tree, which
 * follows this directory on the include path), then, with -D_GRB_WITH_B200,
 * the b200 overload of hpcg, which runs the fused device HPCG for systems
 * that build_hpcg_system made (graphblas/b200/fused_hpcg.hpp).
 */
#ifndef ALPB_OVERLAY_ALGORITHMS_HPCG_HPP
#define ALPB_OVERLAY_ALGORITHMS_HPCG_HPP

#include_next <graphblas/algorithms/hpcg/hpcg.hpp>

#ifdef _GRB_WITH_B200
 #include <graphblas/b200/fused_hpcg.hpp>
#endif

#endif
