// Build configuration for compiling the reference's multicomponent sources as a test
// oracle (oracle/_ref/libref_mc.so; with REACTION defined on the command line,
// oracle/_ref/libref_mcr.so).  Test infrastructure only: nothing in the
// product links this.
//
// This header is force-included (-include) ahead of every reference translation unit.
// It defines the reference's include guard DEFINES_H, so the reference's own
// src/headers/defines.hpp is skipped and the macros below take its place.  The
// values mirror the reference's compile-time switches (src/headers/defines.hpp):
//   * the velocity set (D3Q27, NDIM 3; defines.hpp:120-131),
//   * OpenMP loops on (PARALLEL; defines.hpp:73-75),
//   * cell-type codes TYPE_F..TYPE_Q (defines.hpp:140-149) -- an interface that must
//     stay identical, since setups and restart files store them,
//   * NSCBC constants (defines.hpp:100-111), SPECIES_MIN (defines.hpp:96).
// MULTICOMP is defined (species populations f_a plus the energy population g);
// ISOTHERM, CONJUGATE, SMOOTHING stay undefined; REACTION is set by the build recipe.
#ifndef DEFINES_H
#define DEFINES_H
#include <math.h>

#define PARALLEL
#define NUM_THREADS 8
#define OUTPUT_SI
#define OUTPUT_MASSFRAC
#define LIMITER_TYPE limiterVanleer
#define SPECIES_MIN 1E-8

#define NSCBC_SIGMA_OUT 0.25
#define NSCBC_RELAX_U 0.20
#define NSCBC_RELAX_T 0.20
#define NSCBC_RELAX_Y 0.20

#define VEL0 0.1
#define RHO0 1.0
#define TEMP0 0.025

#define D3Q27
#define NDIM 3
#define MULTICOMP

#define TYPE_F 0
#define TYPE_S 1
#define TYPE_P 2
#define TYPE_A 3
#define TYPE_FS 4
#define TYPE_I 5
#define TYPE_O 6
#define TYPE_I_C 7
#define TYPE_O_C 8
#define TYPE_Q 9

#endif
