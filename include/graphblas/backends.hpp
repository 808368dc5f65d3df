/*
 * Backend enumeration of ALP/GraphBLAS with the B200 backend added.
 *
 * grb::Backend is a closed enum (graphblas/backends.hpp of ALP), so adding a
 * backend means providing the enum: the enumerators below are ALP's own, in
 * ALP's order (so every existing specialisation keeps its meaning), followed
 * by `b200`.  The include guard is ALP's, so ALP's own backends.hpp -- which
 * other ALP headers include by relative path -- is never parsed twice.
 */
#ifndef _H_GRB_BACKENDS
#define _H_GRB_BACKENDS

#include <iostream>
#include <string>

namespace grb {

	enum Backend {
		reference,
		reference_omp,
		hyperdags,
		nonblocking,
		shmem1D,
		NUMA1D,
		GENERIC_BSP,
		BSP1D,
		doublyBSP1D,
		BSP2D,
		autoBSP,
		optBSP,
		hybrid,
		hybridSmall,
		hybridMid,
		hybridLarge,
		minFootprint,
		banshee,
		banshee_ssr,
		/** One NVIDIA B200 (sm_100a): device-resident containers, CUDA kernels. */
		b200
	};

	static inline std::string toString( const enum grb::Backend backend ) {
		switch( backend ) {
			case reference: return "reference";
			case reference_omp: return "reference_omp";
			case hyperdags: return "hyperdags";
			case nonblocking: return "nonblocking";
			case shmem1D: return "shmem1D";
			case NUMA1D: return "NUMA1D";
			case GENERIC_BSP: return "GENERIC_BSP";
			case BSP1D: return "BSP1D";
			case doublyBSP1D: return "doublyBSP1D";
			case BSP2D: return "BSP2D";
			case autoBSP: return "autoBSP";
			case optBSP: return "optBSP";
			case hybrid: return "hybrid";
			case hybridSmall: return "hybridSmall";
			case hybridMid: return "hybridMid";
			case hybridLarge: return "hybridLarge";
			case minFootprint: return "minFootprint";
			case banshee: return "banshee";
			case banshee_ssr: return "banshee_ssr";
			case b200: return "b200";
		}
		std::cerr << "Warning, grb::toString: unknown backend " << static_cast< int >( backend )
			<< "\n";
		return "unknown";
	}

}

#endif
