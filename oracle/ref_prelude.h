/*
 * ref_prelude.h -- force-included (-include) ahead of every reference GASAL2
 * translation unit that the oracle recipe compiles in place.
 *
 * TEST INFRASTRUCTURE ONLY: used by oracle/Makefile to build the reference
 * library into oracle/_ref/; nothing in the product includes it.
 *
 * The reference's src/gasal.h:9 includes the CUDA runtime header through an
 * absolute CUDA-10.1 path that does not exist here.  This prelude supplies the
 * same declarations from include/gasal.h (identical layouts) and defines the
 * reference header's include guard, so that src/gasal.h is opened but skipped
 * and the reference sources compile unmodified.
 */
#include "../include/gasal.h"
#define __GASAL_H__
