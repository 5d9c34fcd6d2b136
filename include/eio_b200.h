/*
 * eio_b200.h -- C ABI of the B200 (sm_100a) 2-D isotropic elastic
 * velocity-stress staggered-grid finite-difference engine.
 *
 * This is the drop-in boundary for the reference's elastic propagation path
 * (biondiettore/elastic_isotropic_operators).  Paths in the citations are
 * relative to that project:
 *   F  = elastic_iso_lib/elastic_iso_float/prop
 *   PF = elastic_iso_lib/python/python_float
 *
 * Conventions
 *   - Every function returns an int status: EIO_OK (0) or a negative error
 *     code; eio_last_error() returns the message of the last failure on the
 *     calling thread.  Nothing here calls exit() (the reference's cudaErrors.cu
 *     does); QC failures that the reference reports with std::runtime_error
 *     ("" + stderr message) come back as EIO_ERR_QC with the same message.
 *   - Arrays use the reference layouts, z fastest:
 *       elastic parameters  [3][nx][nz]   (rho, lambda, mu)
 *       wavefield fields    [nx][nz]      (vx, vz, sigmaxx, sigmazz, sigmaxz)
 *       regular-grid traces [nPoints][nt] (time fastest)
 *     Field order is always vx, vz, sigmaxx, sigmazz, sigmaxz.  Position
 *     lists come in grid order center (sigmaxx, sigmazz), x-shifted (vx),
 *     z-shifted (vz), xz-shifted (sigmaxz).
 *   - Host-pointer entry points copy in and out themselves; *_dev entry points
 *     take device pointers (plus host position lists) and run on the
 *     context's stream; every entry point synchronizes that stream before
 *     it returns.
 *   - A context is bound to one GPU and is not re-entrant (like the
 *     reference operator objects); different contexts may be used from
 *     different host threads.
 */
#ifndef EIO_B200_H
#define EIO_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define EIO_OK 0
#define EIO_ERR_ARG -1     /* invalid argument / inconsistent sizes */
#define EIO_ERR_QC -2      /* finite-difference QC failed (stability, dispersion, size) */
#define EIO_ERR_CUDA -3    /* CUDA runtime error (message has the CUDA error string) */
#define EIO_ERR_BOUNDS -4  /* acquisition device outside the usable grid */
#define EIO_ERR_UNSUPPORTED -5
#define EIO_ERR_NOMEM -6
#define EIO_ERR_TIMEOUT -7 /* a bounded device wait gave up: that call's output is incomplete; the kernel
                              drained its copies before returning, so the context stays usable (the
                              reference exits the process on any CUDA error, F/src/cudaErrors.cu:4-29) */
#define EIO_ERR_NONFINITE -8 /* a call's output holds NaN / Inf (an unstable propagation); only with
                              eio_ctx_set_check_finite on */

typedef struct eio_sinterp eio_sinterp;
typedef struct eio_ctx eio_ctx;

/* Finite-difference parameters: the par-file keys read by
 * fdParamElastic::fdParamElastic (F/src/fdParamElastic.cpp:12-77). */
typedef struct eio_fd_params {
    int nts;            /* coarse (data) time samples */
    float dts;          /* coarse sampling [s] */
    float ots;
    int sub;            /* par-file sub; doubled internally (fdParamElastic.cpp:28) */
    int nz, nx;         /* total grid incl. padding and FAT */
    float oz, ox;       /* origin of the padded grid */
    float dz, dx;
    int zPadMinus, zPadPlus, xPadMinus, xPadPlus;
    float fMax;         /* default 1000 */
    int blockSize;      /* must be 16 (reference constraint) */
    int fat;            /* must be 4 */
    float alphaCos;     /* default 0.99 */
    int surfaceCondition; /* 0, or 1: free surface at z = 2*fat (nonlinear operators) */
    int mod_par;        /* 1: metres (default), 2: km in the par file */
    float errorTolerance; /* default 1e-6 */
} eio_fd_params;

/* Fills p with the reference defaults (fMax 1000, blockSize 16, fat 4,
 * alphaCos 0.99, surfaceCondition 0, mod_par 1, errorTolerance 1e-6). */
void eio_fd_params_default(eio_fd_params *p);

const char *eio_last_error(void);
int eio_version(void);

/* ---------------------------------------------------------------------------
 * Spatial interpolation of acquisition devices (spaceInterpGpu)
 * replaces spaceInterpGpu::spaceInterpGpu / forward / adjoint / getRegPosUnique
 * (F/src/spaceInterpGpu.cpp:11-362; pybind PF/pyElastic_iso_float_nl.cpp:19-30)
 * method: "linear" (bilinear 2x2; nFilt forced to 1), "sinc" (normalised
 * (2 nFilt)^2 sinc stencil; equals the reference exactly for nFilt = 1),
 * "gauss".  dipole = 1 is supported for "linear" only, as in the reference.
 * ------------------------------------------------------------------------ */
int eio_sinterp_create(const float *zCoord, const float *xCoord, int nDevice,
                       int nz, float oz, float dz, int nx, float ox, float dx,
                       int nt, const char *method, int nFilt, int dipole,
                       float zDipoleShift, float xDipoleShift, eio_sinterp **out);
void eio_sinterp_destroy(eio_sinterp *s);
/* nIrreg devices, nReg unique regular grid points, nFiltTotal points per device */
int eio_sinterp_sizes(const eio_sinterp *s, int *nIrreg, int *nReg, int *nFiltTotal);
int eio_sinterp_positions(const eio_sinterp *s, int *regPos /* [nReg] */);
int eio_sinterp_weights(const eio_sinterp *s, int *gridPointIndex, float *weight /* [nIrreg*nFiltTotal] */);
/* forward: regular [nReg][nt] -> irregular [nIrreg][nt]; adjoint: the transpose */
int eio_sinterp_forward(const eio_sinterp *s, int add, const float *signalReg, float *signalIrreg);
int eio_sinterp_adjoint(const eio_sinterp *s, int add, float *signalReg, const float *signalIrreg);

/* ---------------------------------------------------------------------------
 * Medium preparation + QC (fdParamElastic), host only
 * replaces fdParamElastic::fdParamElastic (F/src/fdParamElastic.cpp:12-157)
 * outputs the five scaled staggered coefficient grids [nx][nz]:
 * rhoxDtw, rhozDtw, lamb2MuDtw, lambDtw, muxzDtw
 * ------------------------------------------------------------------------ */
int eio_medium_prepare(const eio_fd_params *p, const float *elasticParam,
                       float *rhoxDtw, float *rhozDtw, float *lamb2MuDtw, float *lambDtw, float *muxzDtw);

/* Staggering operators (staggerX / staggerZ, F/src/stagger.cpp:18-114), [nx][nz] */
int eio_stagger(int axis /*0 = x, 1 = z*/, int adj, int add, int nz, int nx, float *model, float *data);

/* Linear coarse<->fine time interpolation (interpTimeLinTbb, F/src/interpTimeLinTbb.cpp:26-102)
 * sub_internal = 2*sub.  fwd: coarse [nDev][nts] -> fine [nDev][ntw] */
int eio_time_interp(int adj, int add, int nts, float dts, float ots, int sub_internal, int nDev,
                    float *coarse, float *fine);

/* ---------------------------------------------------------------------------
 * Device context = fdParamElastic + init/allocate on one GPU
 * replaces initNonlinearElasticGpu + allocateNonlinearElasticGpu and
 * initBornGpu + allocateBornElasticGpu
 * (F/src/nonlinearPropElasticGpuFunctions.cu:85-264,
 *  F/src/BornElasticGpuFunctions.cu:88-338), plus the QC of fdParamElastic.
 * ------------------------------------------------------------------------ */
int eio_ctx_create(const eio_fd_params *p, const float *elasticParam, int device, eio_ctx **out);
/* setBackground: rebuild the medium (QC may fail) (PF/pyElastic_iso_float_nl.cpp:48) */
int eio_ctx_set_background(eio_ctx *c, const float *elasticParam);
void eio_ctx_destroy(eio_ctx *c);
/* Where the Born operators' source-wavefield history lives (the reference
 * streams it to host RAM when it is large, useStreams = 1,
 * F/src/BornElasticGpuFunctions.cu:850-1096): 0 (default) = device memory, or,
 * when the device allocation fails, pinned host memory mapped into the device
 * address space (the kernels write and read it across the host link: slower,
 * same results); 1 = device only (EIO_ERR_NOMEM when it does not fit);
 * 2 = mapped host memory.  eio_ctx_get_history_location: 0 = none held yet,
 * 1 = device, 2 = host. */
int eio_ctx_set_history_location(eio_ctx *c, int where);
int eio_ctx_get_history_location(const eio_ctx *c, int *where);
/* NaN / Inf checks.  The elastic parameters are always checked at
 * eio_ctx_create / eio_ctx_set_background (EIO_ERR_ARG naming the parameter and
 * cell).  With on != 0 every eio_nl_forward / eio_nl_adjoint / eio_born_forward /
 * eio_born_adjoint / eio_fwi_gradient call also scans its host inputs
 * (EIO_ERR_ARG before any work) and its outputs (EIO_ERR_NONFINITE after the
 * propagation, e.g. an unstable model); off by default (a pass over the
 * arrays on the host). */
int eio_ctx_set_check_finite(eio_ctx *c, int on);
/* A process-wide cap on the device memory the library's own buffers may hold
 * (bytes; 0 = none), and the bytes they hold now: an allocation above the cap
 * fails as if the device were full (EIO_ERR_NOMEM, or the host-memory history
 * above), so callers can reserve memory for others and tests can produce
 * out-of-memory on purpose. */
int eio_set_device_memory_cap(long long bytes);
int eio_get_device_memory_used(long long *bytes);
/* Source-wavefield snapshot storage for the Born operators (no reference
 * counterpart; the reference keeps FP32 snapshots): 0 = FP32 (bit-faithful to
 * the reference), 1 = BF16, 2 = FP16, both as 16-bit codes with one scale per
 * snapshot and field (BF16: the snapshot's max |value|, FP16: max / 2^15), half
 * the history memory.  16-bit modes need sub = 1 (else EIO_ERR_UNSUPPORTED at
 * the next Born call). */
int eio_ctx_set_checkpoint_precision(eio_ctx *c, int mode);
/* Scaled coefficient grids of the context (for inspection / tests). */
int eio_ctx_get_medium(const eio_ctx *c, float *rhoxDtw, float *rhozDtw, float *lamb2MuDtw,
                       float *lambDtw, float *muxzDtw);
/* Fine time steps and updated cells of one propagation (for throughput accounting). */
int eio_ctx_counts(const eio_ctx *c, long long *fineSteps, long long *cellsPerStep);
/* CUDA stream of the context (cudaStream_t as void*). */
void *eio_ctx_stream(eio_ctx *c);
/* Step-kernel selection (no reference counterpart; the reference has one
 * 16x16-tile kernel).  kind 0: shared-memory tile kernel; kind 1: TMA-pipelined
 * x-sweep with strip height tz (64 or 128), chunk width cw (8 or 16) and cpr
 * chunks per CTA; kind 2: persistent TMA tile kernel; kind 3: tile kernel at
 * 4 CTAs per SM; kind 4: two threads per float4; kind 5: two fine steps per
 * launch (the tile widened by the stencil radius, four wavefield levels), kind 3
 * for the steps that run alone (free surface, saved wavefields, the last
 * coarse interval of a Born source wavefield, running-sum epilogues).  By
 * default the first propagation of a context times every candidate on its
 * grid (eio_ctx_autotune) and keeps the fastest. */
int eio_ctx_set_kernel(eio_ctx *c, int kind, int tz, int cw, int cpr);
int eio_ctx_get_kernel(const eio_ctx *c, int *kind, int *tz, int *cw, int *cpr);
int eio_ctx_autotune(eio_ctx *c, int *kind, int *tz, int *cw, int *cpr);
/* Bound of the TMA-pipeline waits of the sweep (kind 1) and tile (kind 2)
 * kernels, in mbarrier try_wait polls (no reference counterpart: the
 * reference's kernels have no device-side waits).  A wait that runs out sets
 * the context's error flag; the CTA then waits for its copies still in flight
 * (with a fixed long bound that this setting does not shorten) and returns,
 * and the call fails with EIO_ERR_TIMEOUT.  polls < 0 restores the default
 * (2^20); 0 makes every pipeline wait give up at once (used by the tests of
 * the timeout path). */
int eio_ctx_set_wait_limit(eio_ctx *c, long long polls);
/* Persistent time loop (no reference counterpart; the reference launches 4-12
 * kernels per fine step, BornElasticGpuFunctions.cu:744-849): the shot groups
 * of the Born operators (eio_ctx_set_born_batch) run every fine step of a
 * propagation phase in one cooperative launch, the CTAs advancing tile by tile
 * behind per-tile step counters instead of a grid-wide boundary per step, the
 * forward's secondary sources computed per tile inside the loop.  Results are
 * bitwise those of the per-step launches.  A tile whose neighbours do not
 * arrive within 4 x the wait limit (eio_ctx_set_wait_limit) polls sets the
 * error flag and the call fails with EIO_ERR_TIMEOUT.  mask: the phases that
 * run as persistent loops, 1 the source wavefield, 2 the Born forward's
 * scattered wavefield, 4 the Born adjoint; 0 (default) launches per step, which
 * measured faster on the 600x1800 benchmark (the per-tile completion fence and
 * neighbour polls cost more than the launch boundaries they remove). */
int eio_ctx_set_persistent(eio_ctx *c, int mask);
int eio_ctx_get_persistent(const eio_ctx *c, int *mask);
int eio_ctx_get_wait_limit(const eio_ctx *c, long long *polls);
/* Instrumentation (no reference counterpart): kernel launch counters and,
 * when enabled, CUDA-event timing of every 16th fused step-kernel launch;
 * stepMs is the sampled mean duration times stepLaunches.
 * enable: 1 on, 0 off, -1 unchanged; reset: zero the counters after reading. */
int eio_ctx_stats(eio_ctx *c, int enable, int reset, long long *launches, long long *stepLaunches,
                  double *stepMs);
/* Cell updates of the single-step launches since the last eio_ctx_stats reset,
 * summed over the lanes (a launch that advances several shots counts each
 * shot's interior cells); call it before eio_ctx_stats resets the counters. */
int eio_ctx_step_cells(const eio_ctx *c, long long *cells);
/* Shot batching of the nonlinear operators (no reference counterpart; the
 * reference runs one shot per GPU at a time, nonlinearPropElasticShotsGpu.cpp:80-422):
 * with shots > 1 (default 8), eio_nl_forward and eio_nl_adjoint advance up to
 * `shots` (<= 8) shots in lockstep, one engine each, with one step launch per
 * fine step for all of them (the shots of a tile next to each other in the
 * launch, every shot reading one copy of the medium; each shot on its own
 * window and point lists); 1 runs the shots one at a time on the lanes.
 * Results equal the one-shot propagation with the tile kernel bit for bit.
 * Not used with the free surface or when a wavefield is saved. */
int eio_ctx_set_shot_batch(eio_ctx *c, int shots);
/* Shot batching of the Born operators (eio_born_forward / eio_born_adjoint /
 * eio_born_shots_dev; no reference counterpart, BornElasticShotsGpu.cpp:178-207
 * runs one shot per GPU): with shots > 1 the shots of a call run in groups of
 * up to min(shots, lanes) that the free device memory holds (each shot needs
 * its own source-wavefield history), sizes as even as possible, one engine per
 * shot, one step launch per fine step for the group and the imaging of the
 * group in one launch per coarse sample (sub = 1 and FP32 histories; otherwise
 * the lanes run the shots).  Per-shot traces equal the one-shot propagation
 * with the tile kernel (kind 3) bit for bit; the image adds the shots in
 * another order.  Default 1 (the shots on the lanes): on the 600x1800 Born
 * benchmark two concurrent lanes measured faster than groups of 2-5. */
int eio_ctx_set_born_batch(eio_ctx *c, int shots);
/* Shot lanes (no reference counterpart; the reference runs one shot per GPU at
 * a time). The multi-shot operators (eio_nl_forward/adjoint,
 * eio_born_forward/adjoint, eio_born_shots_dev) run their shots on up to
 * `lanes` engines of the same GPU concurrently. Each lane has its own
 * streams, wavefields and Born history. Lane k takes shots k, k + n, ... in
 * order, and the lanes' images and stacked adjoint sources are added in lane
 * order, so results do not depend on timing. A new lane is created only while
 * the free device memory holds its buffers (for Born, the source-wavefield
 * history). Default 2, range 1 .. 8; lowering the count releases lanes.
 * eio_ctx_get_lanes reports the setting and the lanes that exist. */
int eio_ctx_set_lanes(eio_ctx *c, int lanes);
int eio_ctx_get_lanes(const eio_ctx *c, int *lanes, int *active);
/* Many Born shots with device-resident inputs (no reference counterpart).
 * Shot s: fine-time regular sources srcDtw[5*s + f] and receiver traces
 * data[5*s + f] (device pointers, as eio_born_fwd_reg_dev), positions
 * srcPos[4*s + k] / nSrc[4*s + k] and recPos[4*s + k] / nRec[4*s + k] (host).
 * dm[5]: the device perturbation (adj = 0) or the device image every shot
 * adds into (adj = 1). The shots run on the context's lanes. */
int eio_born_shots_dev(eio_ctx *c, int adj, int nShots, float *const *srcDtw, float *const dm[5],
                       float *const *data, const int *const *srcPos, const int *nSrc,
                       const int *const *recPos, const int *nRec);
/* FWI misfit and gradient in one pass per shot (no reference counterpart:
 * the reference runs nonlinearFwiPropElasticShotsGpu, then BornElasticShotsGpu
 * adjoint, three propagations per shot). Per shot, the nonlinear forward of
 * the source traces `model` (irregular, as eio_nl_forward) records the Born
 * source-wavefield history. The sampled residual r = S d - dObs follows, then
 * the Born adjoint of S^T r on that history: two propagations per shot. The
 * nonlinear forward injects the coarse traces with the time filter, where the
 * Born operators inject host-interpolated fine traces of the same signal, so
 * the history agrees with theirs to rounding. S picks nComp components, codes
 * 0..4 = vx, vz, sxx, szz, sxz and 5 = pressure 0.5 (sxx + szz) (the data
 * component sampler of the FWI scripts).
 * dObs: [nExp][nComp][nRecIrreg][nts]; data (optional, may be NULL):
 * [nExp][5][nRecIrreg][nts] modelled; grad: [3][nx][nz], overwritten with
 * the Born adjoint image of the residual; misfit: 0.5 r.r (FP64 sum, shots in order).
 * Runs on the context's lanes and shot windows; no free surface. */
int eio_fwi_gradient(eio_ctx *c, int nExp, int nModelExp, const float *model, const float *dObs, int nComp,
                     const int *comps, eio_sinterp *const *src, eio_sinterp *const *rec, int nRecGeom,
                     float *data, float *grad, double *misfit);
/* Cropped shots (no reference counterpart; the reference propagates every shot
 * on the whole grid). Shot i of the next multi-shot calls (eio_nl_forward,
 * eio_nl_adjoint, eio_born_forward, eio_born_adjoint with nExp == nShots)
 * propagates on columns [ix0[i], ix0[i] + nxw[i]) of the grid only: the
 * medium, the Born perturbation and the gradient are viewed through the
 * window. Its first and last fat columns are the frozen frame, and the
 * grid's cosine taper runs from the window's edges. Each window must lie in
 * the grid, hold 2*fat + a multiple of 16 columns, and contain the shot's
 * sources and receivers in its updated interior (EIO_ERR_BOUNDS otherwise).
 * Wavefield saving is not available on windows. nShots = 0 restores
 * whole-grid shots. */
int eio_ctx_set_shot_windows(eio_ctx *c, int nShots, const int *ix0, const int *nxw);
/* FP64 reductions on the GPU (no reference counterpart; the reference sums on
 * the host in pySolver, operator.h:50-89 for the dot-product test).
 * op 0: sum x[i]*y[i] (dot product, or squared norm with y == x);
 * op 1: sum (x[i]-y[i])^2 (data misfit). x, y: n values of type dtype
 * (0: float, 1: double), device pointers when onDevice != 0, else host arrays
 * staged through the device in chunks. The summation order is fixed, so the
 * result is reproducible. */
int eio_reduce64(int device, int op, int dtype, const void *x, const void *y, long long n, int onDevice,
                 double *result);
/* CUDA graphs of the time loops (no reference counterpart; off by default).
 * Each time loop is captured as a graph the first time its launch sequence
 * (kernel choice, step counts, buffer addresses, point-list sizes) is seen and
 * replayed when it recurs. Only the contents of device buffers differ between
 * replays, so shots with the same number of points share one graph. The
 * engine keeps up to 8 graphs per context. enable = 0 (the default) launches
 * every kernel directly, with programmatic dependent launch between the
 * steps; measured on B200 that is faster than the replayed graphs (600x1800
 * Born 43.3 vs 41.0-41.9 Gcell/s, 312x520 nonlinear 22.5 vs 18.7-21.4). */
int eio_ctx_set_graphs(eio_ctx *c, int enable);
/* The two-step launches (kind 5) alone, since the last reset: their count and
 * their sampled mean duration times that count (no reference counterpart).
 * They are also included in stepLaunches / stepMs of eio_ctx_stats; read this
 * before an eio_ctx_stats call that resets. */
int eio_ctx_pair_stats(eio_ctx *c, long long *pairLaunches, double *pairMs);

/* ---------------------------------------------------------------------------
 * Single-shot propagation on the regular grid
 * replaces propShotsElasticFwdGpu / propShotsElasticAdjGpu
 * (F/src/nonlinearPropElasticGpuFunctions.cu:561-648, 932-1027) and
 * BornShotsFwdGpu / BornShotsAdjGpu (F/src/BornElasticGpuFunctions.cu:719-1454).
 * model: 5 source traces [nSrcReg(grid)][nts]; data: 5 receiver traces [nRecReg(grid)][nts]
 * srcPos / recPos: 4 position lists (center, x, z, xz) with counts.
 *   nl_fwd overwrites data; nl_adj overwrites model.
 *   born_fwd: srcDtw = 5 fine-time source traces [nSrcReg][ntw] (already scaled),
 *             dm = 5 staggered+scaled perturbations [nx][nz]; overwrites data.
 *   born_adj: ACCUMULATES into dm (the reference copies dm in and back).
 * ------------------------------------------------------------------------ */
int eio_nl_fwd_reg(eio_ctx *c, float *const model[5], float *const data[5],
                   const int *const srcPos[4], const int nSrc[4], const int *const recPos[4], const int nRec[4]);
int eio_nl_adj_reg(eio_ctx *c, float *const model[5], float *const data[5],
                   const int *const srcPos[4], const int nSrc[4], const int *const recPos[4], const int nRec[4]);
int eio_born_fwd_reg(eio_ctx *c, float *const srcDtw[5], float *const dm[5], float *const data[5],
                     const int *const srcPos[4], const int nSrc[4], const int *const recPos[4], const int nRec[4]);
int eio_born_adj_reg(eio_ctx *c, float *const srcDtw[5], float *const dm[5], float *const data[5],
                     const int *const srcPos[4], const int nSrc[4], const int *const recPos[4], const int nRec[4]);
/* Same, with every float array a DEVICE pointer on the context's GPU
 * (positions stay host arrays). */
int eio_nl_fwd_reg_dev(eio_ctx *c, float *const model[5], float *const data[5],
                       const int *const srcPos[4], const int nSrc[4], const int *const recPos[4], const int nRec[4]);
int eio_nl_adj_reg_dev(eio_ctx *c, float *const model[5], float *const data[5],
                       const int *const srcPos[4], const int nSrc[4], const int *const recPos[4], const int nRec[4]);
int eio_born_fwd_reg_dev(eio_ctx *c, float *const srcDtw[5], float *const dm[5], float *const data[5],
                         const int *const srcPos[4], const int nSrc[4], const int *const recPos[4], const int nRec[4]);
int eio_born_adj_reg_dev(eio_ctx *c, float *const srcDtw[5], float *const dm[5], float *const data[5],
                         const int *const srcPos[4], const int nSrc[4], const int *const recPos[4], const int nRec[4]);

/* ---------------------------------------------------------------------------
 * Multi-shot operators (the pybind11 targets)
 * replace nonlinearPropElasticShotsGpu::forward/adjoint
 * (F/src/nonlinearPropElasticShotsGpu.cpp:80-183, 304-422; pybind
 * PF/pyElastic_iso_float_nl.cpp:32-54) and BornElasticShotsGpu::forward/adjoint
 * (F/src/BornElasticShotsGpu.cpp:85-378; pybind PF/pyElastic_iso_float_born.cpp:19-36).
 *
 * Geometry: src[4*nExp] = the four spaceInterp objects of each shot in grid
 * order (center, x, z, xz); rec[4*nRecGeom] likewise with nRecGeom = 1
 * (constant receivers) or nExp.
 * NL model  [nModelExp][5][nSrcIrreg][nts] (nModelExp = 1: same signal for all shots)
 * NL data   [nExp][5][nRecIrreg][nts]
 * Born model [3][nx][nz] (drho, dlambda, dmu); Born data like NL data;
 * Born source signals: nSignals (1 or nExp) arrays [5][nSrcIrreg][nts].
 * add = 0 zeroes the output first, add = 1 accumulates (reference semantics).
 * ------------------------------------------------------------------------ */
int eio_nl_forward(eio_ctx *c, int add, int nExp, int nModelExp, const float *model, float *data,
                   eio_sinterp *const *src, eio_sinterp *const *rec, int nRecGeom);
int eio_nl_adjoint(eio_ctx *c, int add, int nExp, int nModelExp, float *model, const float *data,
                   eio_sinterp *const *src, eio_sinterp *const *rec, int nRecGeom);
/* Nonlinear operators that also save the wavefield of one shot: replace
 * nonlinearPropElasticShotsGpu::forwardWavefield / adjointWavefield
 * (F/src/nonlinearPropElasticShotsGpu.cpp:185-300, 424-540) with the
 * saveWavefield / wavefieldShotNumber parameters, and the drivers
 * propShotsElastic{Fwd,Adj}GpuWavefield (F/src/nonlinearPropElasticGpuFunctions.cu:649-760, 1029-1110).
 * For shot wShot (0-based; < 0 saves nothing) wavefield [nts][5][nx][nz] is
 * overwritten with the coarse-time samples of every fine step's new level
 * (interpWavefield, K:1258-1291); the adjoint wavefield is then scaled like the
 * adjoint sources (nonlinearPropElasticGpu.cpp:432-446).  Every interior cell
 * is saved; the reference kernel indexes z without the FAT offset (K:1262) and
 * so leaves the last four interior rows at zero. */
int eio_nl_forward_wavefield(eio_ctx *c, int add, int nExp, int nModelExp, const float *model, float *data,
                             eio_sinterp *const *src, eio_sinterp *const *rec, int nRecGeom, int wShot,
                             float *wavefield);
int eio_nl_adjoint_wavefield(eio_ctx *c, int add, int nExp, int nModelExp, float *model, const float *data,
                             eio_sinterp *const *src, eio_sinterp *const *rec, int nRecGeom, int wShot,
                             float *wavefield);
int eio_born_forward(eio_ctx *c, int add, int nExp, const float *model, float *data,
                     const float *const *srcSignals, int nSignals,
                     eio_sinterp *const *src, eio_sinterp *const *rec, int nRecGeom);
int eio_born_adjoint(eio_ctx *c, int add, int nExp, float *model, const float *data,
                     const float *const *srcSignals, int nSignals,
                     eio_sinterp *const *src, eio_sinterp *const *rec, int nRecGeom);

/* Born host preparation of one shot, exposed so that callers can keep the
 * single-shot *_dev entry points fed from device memory:
 * - sources: seismicElasticOperator2D::setSources, Born branch
 *   (F/include/seismicElasticOperator2D.cpp:27-117): irregular signal
 *   [5][nSrcIrreg][nts] -> 5 scaled regular fine-time traces [nSrcReg(grid)][ntw];
 * - model: staggering and scaling of (drho, dlambda, dmu) [3][nx][nz] into the
 *   5 perturbation grids [nx][nz] (F/src/BornElasticShotsGpu.cpp:107-150). */
int eio_born_prepare_sources(eio_ctx *c, const float *signal, eio_sinterp *const src[4], float *const out[5]);
int eio_born_prepare_model(eio_ctx *c, const float *model, float *const out[5]);
/* Nonlinear host preparation of one shot for eio_nl_fwd_reg_dev: irregular
 * source traces [5][nSrcIrreg][nts] -> 5 regular traces [nSrcReg(grid)][nts],
 * spread by the adjoint of the source interpolators and scaled by 2*dtw (or
 * the staggered buoyancy for vx, vz) and 1/(dx*dz), as
 * nonlinearPropElasticGpu::forward does (F/src/nonlinearPropElasticGpu.cpp:116-144). */
int eio_nl_prepare_sources(eio_ctx *c, const float *model, eio_sinterp *const src[4], float *const out[5]);

/* ---------------------------------------------------------------------------
 * Allocation-free nonlinear forward propagation.  No counterpart in the
 * reference (its drivers cudaMalloc and cudaFree on every call).
 *
 * For callers that cannot call cudaMalloc -- code whose device memory belongs
 * to another allocator, processes that forbid allocation after start-up, or
 * plug-ins that must not grow their host process's device footprint.  It runs
 * the same propagation as eio_nl_fwd_reg_dev without allocating anything:
 * all scratch (both wavefield levels, taper tables, point lists, time-major
 * trace copies) lives in one fixed file-scope device array of about 28 MB
 * that every GPU loading the library holds until the process exits.
 *   - p: the par-file parameters (medium QC is the caller's: the medium
 *     arrives already prepared, e.g. with eio_medium_prepare);
 *   - medium: the 5 scaled coefficient grids [nx][nz] in device memory;
 *   - model / data: as eio_nl_fwd_reg_dev, device memory owned by the caller;
 *   - runs on `stream` (a cudaStream_t, NULL = legacy default stream) of the
 *     current device and synchronizes it before returning.
 * Limits (EIO_ERR_ARG beyond them, checked before anything runs):
 *   nz*nx <= 262144 cells, nz, nx <= 16384, source + receiver traces <=
 *   4194304 floats (sum over the 5 fields of points x nts), <= 65536 points
 *   per list.
 * Set-up: the first call on a device (and the first after a
 * cudaDeviceReset) looks up the array's device address with
 * cudaGetSymbolAddress; make that first call on each device before any
 * stream capture begins there.
 * Every call reuses the same array and clears what must start at zero;
 * calls that overlap on the GPU (other threads or streams) race on it and
 * must be serialised by the caller. */
int eio_nl_fwd_noalloc(const eio_fd_params *p, float *const medium[5], float *const model[5], float *const data[5],
                       const int *const srcPos[4], const int nSrc[4], const int *const recPos[4], const int nRec[4],
                       void *stream);

/* ---- Learned FWI preconditioner (no reference counterpart) ------------------
 * Kernels of a small convolutional network that maps an FWI gradient to an
 * approximate Gauss-Newton update, trained on (J^T J dm, dm) pairs from the
 * Born operators.  All pointers are device pointers, 16-byte aligned; work is
 * queued on `stream` (a cudaStream_t, NULL = the default stream) and nothing
 * synchronises.  Activations are NHWC BF16 with 16 or 32 channels; weights
 * [9][cout][cin] BF16, tap = 3 dy + dx; products on the tensor cores with FP32
 * accumulation. */
/* y = conv3x3(x, wt) (stride 1, zero padding 1, no bias), then ReLU when relu
 * != 0, or, when mask != NULL, y *= (mask > 0) (mask: NHWC, cout channels: the
 * ReLU derivative for the backward pass).  y: BF16 NHWC [n][h][w][cout];
 * y32 (optional): the same values in FP32. */
int eio_cnn_conv3x3(int n, int h, int w, int cin, int cout, const void *x, const void *wt, const void *mask,
                    int relu, void *y, float *y32, void *stream);
/* forward-convolution kernel of eio_cnn_conv3x3 (process-wide): 0 = mma.sync
 * (m16n8k16; default, faster at 16-32 channels), 1 = tcgen05 (M = 128 pixels,
 * TMEM accumulator, strips of rows through a cp.async ring) */
int eio_cnn_set_conv_path(int path);
int eio_cnn_get_conv_path(int *path);
/* *err = 1 when a tcgen05 kernel gave up waiting for its accumulator (the
 * output of that call is incomplete), 2 when its drain also ran out; reset !=
 * 0 clears the flag.  Synchronises the device. */
int eio_cnn_status(int reset, int *err);
/* Bound of the tcgen05 convolution's accumulator waits, in try_wait polls
 * (process-wide; < 0 restores the default 2^22; 0 makes the first wait of
 * every CTA give up).  After a timeout the CTA waits, with a fixed long
 * bound, for its MMAs and copies still in flight before it frees its tensor
 * memory and returns; eio_cnn_status then reports 1 (2 if even that drain
 * ran out). */
int eio_cnn_set_wait_limit(long long polls);
int eio_cnn_get_wait_limit(long long *polls);
/* floats of scratch the weight gradient needs for this shape */
int eio_cnn_wgrad_scratch(int n, int h, int w, int cin, int cout, long long *floats);
/* dw[tap][co][ci] = sum_p dy[p][co] x[p + (dy-1, dx-1)][ci] (FP32, overwritten;
 * fixed summation order) */
int eio_cnn_conv3x3_wgrad(int n, int h, int w, int cin, int cout, const void *x, const void *dy, float *dw,
                          float *scratch, long long scratchFloats, void *stream);
/* wt[tap][ci][co] = w[8 - tap][co][ci]: the weights of the data gradient */
int eio_cnn_flip(int cin, int cout, const void *w, void *wt, void *stream);
/* loss = 0.5 sum_{p, c < nc} (y32 - target)^2 / (npix nc) into *loss (device
 * double); dz (BF16 NHWC, c channels) = its derivative, 0 on channels >= nc.
 * target: FP32 [npix][nc]; scratch: 1024 device doubles. */
int eio_cnn_mse(long long npix, int c, int nc, const float *y32, const float *target, void *dz, double *scratch,
                double *loss, void *stream);
/* one Adam step (bias-corrected, step >= 1) on the FP32 parameters p with
 * moments m, v and gradient g; pb (optional): BF16 copy of the result */
int eio_cnn_adam(long long n, float *p, float *m, float *v, const float *g, float lr, float b1, float b2, float eps,
                 int step, void *pb, void *stream);

/* ---- U-Net preconditioner kernels (no reference counterpart) ----------------
 * The layers of precond.UNet.  Device pointers, 16-byte aligned; BF16 NHWC
 * activations, channel counts multiples of 8; queued on `stream` (NULL = the
 * default stream), nothing synchronises.  Convolution weights are
 * [cout][9][cin], tap = 3 dy + dx. */
/* C[M][N] = A[M][K] . B[N][K]^T on tcgen05: BF16 A, B stored K-major (row-major,
 * leading dimensions lda, ldb >= K, multiples of 8), FP32 accumulation.  C32
 * (optional, FP32, ldc = N) and/or C16 (optional, BF16): ReLU when relu != 0,
 * or a multiply by (mask > 0) when mask (BF16 [M][N]) is given.  splits > 1
 * splits K over at most that many slices into scratch (splits x M x N
 * floats), then adds the slices in a fixed order (no ReLU or mask then). */
int eio_gemm_bf16(long long M, long long N, long long K, const void *A, long long lda, const void *B, long long ldb,
                  float *C32, void *C16, const void *mask, int relu, int splits, float *scratch, void *stream);
/* bound of the GEMM kernel's accumulator waits (polls; < 0: default 2^22);
 * after a timeout the CTA drains its MMAs and copies and eio_gemm_status
 * reports 1 (2 if the drain ran out too); reset != 0 clears the flag
 * (synchronises) */
int eio_gemm_set_wait_limit(long long polls);
int eio_gemm_status(int reset, int *err);
/* The convolution kernels bring their operands in by TMA where the image
 * allows it (a 128-pixel tile, and a 64-pixel slice of the weight gradient,
 * form a rectangle of the image: widths that divide 128 / 64 or are
 * multiples of them, heights that the rectangle divides; input channels a
 * multiple of 16; for the weight gradient cout a multiple of 16, <= 256):
 * one 4-D tensor box per tap and channel block, the zero padding from the
 * box's out-of-bounds fill.  Other shapes use the copy-loop kernel.  on = 0
 * forces the copy loop everywhere; 1 runs the TMA kernel with one CTA per SM,
 * 2 with up to two (tiles up to 128 columns), 3 (default) with up to four
 * (three for 64-column tiles, four up to 32): fewer stages each, more copies
 * in flight per SM.  Process-wide. */
int eio_unet_set_tma(int on);
int eio_unet_get_tma(int *on);
/* 3x3 convolution (zero padding) as an implicit GEMM on tcgen05: y[p][co] =
 * sum_{tap, ci} x[p + off(tap)][ci] w[co][tap][ci], x BF16 [n][h][w][cin],
 * FP32 y32 and / or BF16 y16 [n][h][w][cout], ReLU when relu != 0.  The 3x3
 * neighbourhoods are gathered by the GEMM's copy loop (no column matrix).
 * The data gradient is the same call on the output gradient with the flipped
 * weights (eio_unet_flip). */
int eio_unet_conv3x3(int n, int h, int w, int cin, int cout, const void *x, const void *wt, float *y32, void *y16,
                     int relu, void *stream);
/* floats of scratch eio_unet_conv3x3_wgrad needs for this shape */
int eio_unet_wgrad_scratch(int n, int h, int w, int cin, int cout, long long *floats);
/* dw[co][tap][ci] = sum_p dz[p][co] x[p + off(tap)][ci] (FP32, overwritten): a
 * tcgen05 GEMM over the pixels with both operands read MN-major in place (x
 * gathered per tap, dz as stored), split over the pixels into scratch and
 * summed in a fixed order (bitwise reproducible) */
int eio_unet_conv3x3_wgrad(int n, int h, int w, int cin, int cout, const void *x, const void *dz, float *dw,
                           float *scratch, long long scratchFloats, void *stream);
/* wf[ci][tap][co] = w[co][8 - tap][ci]: the weights of the data gradient */
int eio_unet_flip(int cout, int cin, const void *w, void *wf, void *stream);
/* op 0: 2x2 average pooling of [n][h][w][c] into [n][h/2][w/2][c]; 1: its
 * adjoint into [n][h][w][c] (h, w: the fine size); 2: nearest 2x upsampling
 * of [n][h][w][c] into [n][2h][2w][c]; 3: its adjoint into [n][h][w][c].  The
 * adjoints add into `out` when add != 0 (a skip connection's gradient). */
int eio_unet_resample(int op, int n, int h, int w, int c, const void *in, void *out, int add, void *stream);
/* adj = 0: z[p] = [a[p] (ca channels), b[p] (cb channels)]; adj = 1: a[p] (+)=
 * z[p][0:ca], b[p] (+)= z[p][ca:] (accumulating where addA / addB != 0) */
int eio_unet_concat(int adj, long long pixels, int ca, int cb, void *a, int addA, void *b, int addB, void *z,
                    void *stream);
/* dst (+)= src * (mask > 0) over n BF16 values, n a multiple of 8 (the ReLU
 * derivative) */
int eio_unet_relu_adj(long long n, const void *src, const void *mask, void *dst, int add, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* EIO_B200_H */
