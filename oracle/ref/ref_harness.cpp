/*
 * Harness around the reference's OWN CUDA driver layer (test infrastructure).
 *
 * The reference host layer (fdParamElastic, spaceInterpGpu, SEP vectors,
 * Boost, TBB) is not buildable here, but its L1 GPU drivers
 *   elastic_iso_lib/elastic_iso_{float,double}/prop/src/nonlinearPropElasticGpuFunctions.cu
 *   elastic_iso_lib/elastic_iso_{float,double}/prop/src/BornElasticGpuFunctions.cu
 * compile unchanged with nvcc.  This file is compiled next to one of them
 * (from where it lies in the reference tree, see Makefile) and exposes a
 * C entry point that runs one shot exactly the way the reference's per-shot
 * operators do: init -> allocate -> propagate -> deallocate
 * (nonlinearPropElasticGpu.cpp:6-28,155-217; BornElasticGpu.cpp:8-29,82-105).
 *
 * Compile-time switches: REF_REAL (float|double), REF_BORN (0|1).
 */
#include <cstdio>
#if REF_BORN
#include "BornElasticGpuFunctions.h"
#else
#include "nonlinearPropElasticGpuFunctions.h"
#endif

typedef REF_REAL real;

#define EXPORT extern "C" __attribute__((visibility("default")))

#if !REF_BORN
/* model: 5 regular-grid source arrays [nSrcReg][nts]; data: 5 [nRecReg][nts]. */
EXPORT int ref_nl_prop(int adj, int nz, int nx, real dz, real dx, int nts, real dts, int sub_int,
                       int minPad, real alphaCos, real **medium, real **model, real **data,
                       int **srcPos, const int *nSrc, int **recPos, const int *nRec, int surface)
{
    initNonlinearElasticGpu(dz, dx, nz, nx, nts, dts, sub_int, minPad, 16, alphaCos, 1, 0, 0);
    allocateNonlinearElasticGpu(medium[0], medium[1], medium[2], medium[3], medium[4], 0, 0);
    if (!adj)
        propShotsElasticFwdGpu(model[0], model[1], model[2], model[3], model[4],
                               data[0], data[1], data[2], data[3], data[4],
                               srcPos[0], nSrc[0], srcPos[1], nSrc[1], srcPos[2], nSrc[2], srcPos[3], nSrc[3],
                               recPos[0], nRec[0], recPos[1], nRec[1], recPos[2], nRec[2], recPos[3], nRec[3],
                               0, 0, surface);
    else
        propShotsElasticAdjGpu(model[0], model[1], model[2], model[3], model[4],
                               data[0], data[1], data[2], data[3], data[4],
                               srcPos[0], nSrc[0], srcPos[1], nSrc[1], srcPos[2], nSrc[2], srcPos[3], nSrc[3],
                               recPos[0], nRec[0], recPos[1], nRec[1], recPos[2], nRec[2], recPos[3], nRec[3],
                               0, 0, surface);
    deallocateNonlinearElasticGpu(0, 0);
    return 0;
}

/* As ref_nl_prop, through the drivers that also save the wavefield
 * (propShotsElastic{Fwd,Adj}GpuWavefield); wavefield [nts][5][nx][nz]. */
EXPORT int ref_nl_prop_wf(int adj, int nz, int nx, real dz, real dx, int nts, real dts, int sub_int,
                          int minPad, real alphaCos, real **medium, real **model, real **data,
                          int **srcPos, const int *nSrc, int **recPos, const int *nRec, real *wavefield)
{
    /* the drivers size the device wavefield with the 32-bit product 5*nz*nx*nts */
    if ((long long)5 * nts * nz * nx >= (1LL << 31)) return -2;
    initNonlinearElasticGpu(dz, dx, nz, nx, nts, dts, sub_int, minPad, 16, alphaCos, 1, 0, 0);
    allocateNonlinearElasticGpu(medium[0], medium[1], medium[2], medium[3], medium[4], 0, 0);
    if (!adj)
        propShotsElasticFwdGpuWavefield(model[0], model[1], model[2], model[3], model[4],
                                        data[0], data[1], data[2], data[3], data[4],
                                        srcPos[0], nSrc[0], srcPos[1], nSrc[1], srcPos[2], nSrc[2], srcPos[3], nSrc[3],
                                        recPos[0], nRec[0], recPos[1], nRec[1], recPos[2], nRec[2], recPos[3], nRec[3],
                                        wavefield, 0, 0, 0);
    else
        propShotsElasticAdjGpuWavefield(model[0], model[1], model[2], model[3], model[4],
                                        data[0], data[1], data[2], data[3], data[4],
                                        srcPos[0], nSrc[0], srcPos[1], nSrc[1], srcPos[2], nSrc[2], srcPos[3], nSrc[3],
                                        recPos[0], nRec[0], recPos[1], nRec[1], recPos[2], nRec[2], recPos[3], nRec[3],
                                        wavefield, 0, 0);
    deallocateNonlinearElasticGpu(0, 0);
    return 0;
}
#else
/* srcDtw: 5 fine-time source arrays [nSrcReg][ntw]; dm: 5 [nx][nz]; data: 5 [nRecReg][nts].
 * Forward overwrites data; adjoint accumulates into dm. */
EXPORT int ref_born_prop(int adj, int nz, int nx, real dz, real dx, int nts, real dts, int sub_int,
                         int minPad, real alphaCos, real **medium, real **srcDtw, real **dm, real **data,
                         int **srcPos, const int *nSrc, int **recPos, const int *nRec)
{
    /* The reference indexes its coarse Vx/Vz history with the 32-bit product
     * its * nz * nx (interpWavefieldSingleComp, kernelsGpuElastic.cu:1342), which
     * overflows once nts * nz * nx reaches 2^31 and then faults with an illegal
     * address.  Refuse those sizes instead of running them. */
    if ((long long)nts * nz * nx >= (1LL << 31)) return -2;
    initBornGpu(dz, dx, nz, nx, nts, dts, sub_int, minPad, 16, alphaCos, 1, 0, 0);
    allocateBornElasticGpu(medium[0], medium[1], medium[2], medium[3], medium[4], 0, 0, 0);
    if (!adj)
        BornShotsFwdGpu(srcDtw[0], srcDtw[1], srcDtw[2], srcDtw[3], srcDtw[4],
                        dm[0], dm[1], dm[2], dm[3], dm[4],
                        data[0], data[1], data[2], data[3], data[4],
                        srcPos[0], nSrc[0], srcPos[1], nSrc[1], srcPos[2], nSrc[2], srcPos[3], nSrc[3],
                        recPos[0], nRec[0], recPos[1], nRec[1], recPos[2], nRec[2], recPos[3], nRec[3],
                        0, 0, 0, 0);
    else
        BornShotsAdjGpu(srcDtw[0], srcDtw[1], srcDtw[2], srcDtw[3], srcDtw[4],
                        dm[0], dm[1], dm[2], dm[3], dm[4],
                        data[0], data[1], data[2], data[3], data[4],
                        srcPos[0], nSrc[0], srcPos[1], nSrc[1], srcPos[2], nSrc[2], srcPos[3], nSrc[3],
                        recPos[0], nRec[0], recPos[1], nRec[1], recPos[2], nRec[2], recPos[3], nRec[3],
                        0, 0, 0, 0);
    deallocateBornElasticGpu(0, 0, 0);
    return 0;
}
#endif
