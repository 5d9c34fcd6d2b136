/*
 * CPU oracle (test infrastructure, never shipped in the product path).
 * Builds the float (_f) and double (_d) restatements of the reference
 * elastic FD path from oracle_impl.h.  See oracle_impl.h for the citations.
 */
#define _USE_MATH_DEFINES
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_FAT 4          /* varDeclare.h:8 */
#define ORC_SUB_MAX 100    /* varDeclare.h:11 */
#define ORC_PAD_MAX 500    /* varDeclare.h:10 */
/* 8th-order staggered first-derivative coefficients (times 1/d),
 * F/prop/src/nonlinearPropElasticGpuFunctions.cu:159-167 */
#define ORC_C0 1.196289062541883
#define ORC_C1 -0.079752604188901
#define ORC_C2 0.009570312506634
#define ORC_C3 -6.975446437140719e-04

#define REAL float
#define SUFFIX _f
#define ORC_IS_FLOAT 1
#include "oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef ORC_IS_FLOAT

#define REAL double
#define SUFFIX _d
#define ORC_IS_FLOAT 0
#include "oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef ORC_IS_FLOAT

int orc_num_threads(void)
{
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}
