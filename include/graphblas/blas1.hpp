/*
 * Overlay of the ALP/GraphBLAS dispatcher header graphblas/blas1.hpp for the
 * B200 backend: the reference header is included unchanged (include_next
 * finds it in the ALP include tree, which follows this directory on the
 * include path), then, when the backend is enabled with -D_GRB_WITH_B200,
 * the b200 specialisation -- the same pattern the reference dispatchers use
 * for their own backends (e.g. graphblas/blas2.hpp:30-47).
 */
#ifndef ALPB_OVERLAY_BLAS1_HPP
#define ALPB_OVERLAY_BLAS1_HPP

#include <graphblas/config.hpp>
#include_next <graphblas/blas1.hpp>

#ifdef _GRB_WITH_B200
 #include <graphblas/b200/blas1.hpp>
#endif

#endif
