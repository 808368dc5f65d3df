/*
 * Overlay of the ALP/GraphBLAS dispatcher header graphblas/config.hpp for the
 * B200 backend: the reference header is included unchanged (include_next
 * finds it in the ALP include tree, which follows this directory on the
 * include path), then, when the backend is enabled with -D_GRB_WITH_B200,
 * the b200 specialisation -- the same pattern the reference dispatchers use
 * for their own backends (e.g. graphblas/blas2.hpp:30-47).
 */
#ifndef ALPB_OVERLAY_CONFIG_HPP
#define ALPB_OVERLAY_CONFIG_HPP

#include <graphblas/backends.hpp>
#include_next <graphblas/config.hpp>

#ifdef _GRB_WITH_B200
 #include <graphblas/b200/config.hpp>
#endif

#endif
