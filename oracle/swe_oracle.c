/*
 * swe_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 * Builds the float and double restatements of the reference step from
 * swe_oracle_impl.h.  Compile without FMA contraction or fast-math:
 *   gcc -O2 -fno-fast-math -ffp-contract=off -fopenmp -shared -fPIC
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "swe_oracle.h"

#define R float
#define SFX f32
#include "swe_oracle_impl.h"
#undef R
#undef SFX

#define R double
#define SFX f64
#include "swe_oracle_impl.h"
#undef R
#undef SFX

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
