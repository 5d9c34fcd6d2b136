/*
 * CPU oracle for the 2-D isotropic elastic staggered-grid FD path -- TEST
 * INFRASTRUCTURE ONLY.  Nothing in the product library links or calls this
 * code; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference legs load it, and only as the checker or the timed CPU baseline.
 *
 * This header is compiled twice by eio_oracle.c: once with REAL=float
 * (suffix _f, restating elastic_iso_lib/elastic_iso_float) and once with
 * REAL=double (suffix _d, restating elastic_iso_lib/elastic_iso_double).
 * Paths below are relative to the reference project root
 * (F/ = elastic_iso_lib/elastic_iso_float/prop, K = F/src/kernelsGpuElastic.cu).
 *
 * Every routine is a plain loop restatement of the reference arithmetic,
 * including its mixed float/double promotions, so that the float build can be
 * compared with the reference float build and the double build with
 * elastic_iso_double.  Loops over x are OpenMP-parallel (deterministic: no
 * reductions cross threads) so the same code doubles as the timed CPU
 * baseline.
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SUFFIX)

/* ------------------------------------------------------------------ */
/* Constants: FD coefficients, time-interpolation filter, damping      */
/* F/prop/src/nonlinearPropElasticGpuFunctions.cu:155-202              */
/* ------------------------------------------------------------------ */
typedef struct {
    int nz, nx;          /* total grid incl. FAT */
    int nts, S, ntw;     /* S = 2*sub (internal sub-stepping) */
    int h;               /* filter half length = S+1 */
    int minPad;
    REAL zc[4], xc[4];
    REAL filt[2 * (ORC_SUB_MAX + 1)];
    REAL damp[ORC_PAD_MAX];
    REAL dts_inv;        /* Born: 1/(2 dts), F/prop/src/BornElasticGpuFunctions.cu:264 */
} FN(orc_grid_t);


/* sqrt / cos of the working precision: the float build resolves the C++
 * overloads to float (sqrtf/cosf), the double build to double. */
static REAL FN(orc_sqrt)(REAL v) { return ORC_IS_FLOAT ? (REAL)sqrtf((float)v) : (REAL)sqrt((double)v); }
static REAL FN(orc_cos)(REAL v) { return ORC_IS_FLOAT ? (REAL)cosf((float)v) : (REAL)cos((double)v); }

/* sub_int = 2*sub (already doubled, fdParamElastic.cpp:28) */
int FN(orc_grid_init)(FN(orc_grid_t) *g, int nz, int nx, float dz, float dx, int nts, float dts,
                      int sub_int, int minPad, float alphaCos)
{
    if (sub_int >= ORC_SUB_MAX || minPad >= ORC_PAD_MAX || sub_int < 1 || nts < 2) return -1;
    g->nz = nz; g->nx = nx; g->nts = nts; g->S = sub_int;
    g->ntw = (nts - 1) * sub_int + 1;
    g->h = sub_int + 1;
    g->minPad = minPad;
    REAL rdz = (REAL)dz, rdx = (REAL)dx;
    g->zc[0] = (REAL)(ORC_C0 / rdz); g->zc[1] = (REAL)(ORC_C1 / rdz);
    g->zc[2] = (REAL)(ORC_C2 / rdz); g->zc[3] = (REAL)(ORC_C3 / rdz);
    g->xc[0] = (REAL)(ORC_C0 / rdx); g->xc[1] = (REAL)(ORC_C1 / rdx);
    g->xc[2] = (REAL)(ORC_C2 / rdx); g->xc[3] = (REAL)(ORC_C3 / rdx);
    /* nonlinearPropElasticGpuFunctions.cu:172-188 */
    REAL sc = FN(orc_sqrt)((REAL)g->ntw / (REAL)g->nts);
    for (int i = 0; i < g->h; i++) {
        REAL a = (REAL)(1.0 - 1.0 * i / sub_int);
        REAL b = (REAL)(1.0 - a);
        g->filt[i] = (REAL)(a * (1.0 / sc));
        g->filt[i + g->h] = (REAL)(b * (1.0 / sc));
    }
    /* nonlinearPropElasticGpuFunctions.cu:195-202 */
    REAL ralpha = (REAL)alphaCos;
    for (int i = 0; i < minPad; i++) {
        REAL arg = (REAL)(M_PI / (1.0 * minPad) * 1.0 * (minPad - i));
        arg = (REAL)(ralpha + (1.0 - ralpha) * FN(orc_cos)(arg));
        g->damp[i] = arg;
    }
    g->dts_inv = (REAL)(1.0 / (2.0 * (REAL)dts));
    return 0;
}

/* Exported for tests: the constants computed above. */
int FN(orc_consts)(int nz, int nx, float dz, float dx, int nts, float dts, int sub_int, int minPad,
                   float alphaCos, REAL *zc, REAL *xc, REAL *filt, REAL *damp)
{
    FN(orc_grid_t) g;
    if (FN(orc_grid_init)(&g, nz, nx, dz, dx, nts, dts, sub_int, minPad, alphaCos)) return -1;
    for (int i = 0; i < 4; i++) { zc[i] = g.zc[i]; xc[i] = g.xc[i]; }
    for (int i = 0; i < 2 * g.h; i++) filt[i] = g.filt[i];
    for (int i = 0; i < minPad; i++) damp[i] = g.damp[i];
    return 0;
}

/* ------------------------------------------------------------------ */
/* Staggering operators, F/prop/src/stagger.cpp:18-114                 */
/* arrays are [nx][nz], z fastest                                     */
/* ------------------------------------------------------------------ */
void FN(orc_stagger_x)(int adj, int add, int nz, int nx, REAL *model, REAL *data)
{
    if (!adj) {
        if (!add) for (long i = 0; i < (long)nz * nx; i++) data[i] = 0;
        for (int ix = 0; ix < nx - 1; ix++)
            for (int iz = 0; iz < nz; iz++)
                data[(long)ix * nz + iz] = (REAL)(data[(long)ix * nz + iz] +
                    0.5 * (model[(long)ix * nz + iz] + model[(long)(ix + 1) * nz + iz]));
        for (int iz = 0; iz < nz; iz++)
            data[(long)(nx - 1) * nz + iz] += model[(long)(nx - 1) * nz + iz];
    } else {
        if (!add) for (long i = 0; i < (long)nz * nx; i++) model[i] = 0;
        for (int ix = 1; ix < nx - 1; ix++)
            for (int iz = 0; iz < nz; iz++)
                model[(long)ix * nz + iz] = (REAL)(model[(long)ix * nz + iz] +
                    0.5 * (data[(long)ix * nz + iz] + data[(long)(ix - 1) * nz + iz]));
        for (int iz = 0; iz < nz; iz++) {
            model[iz] = (REAL)(model[iz] + 0.5 * data[iz]);
            model[(long)(nx - 1) * nz + iz] = (REAL)(model[(long)(nx - 1) * nz + iz] +
                (data[(long)(nx - 1) * nz + iz] + 0.5 * data[(long)(nx - 2) * nz + iz]));
        }
    }
}

void FN(orc_stagger_z)(int adj, int add, int nz, int nx, REAL *model, REAL *data)
{
    if (!adj) {
        if (!add) for (long i = 0; i < (long)nz * nx; i++) data[i] = 0;
        for (int ix = 0; ix < nx; ix++)
            for (int iz = 0; iz < nz - 1; iz++)
                data[(long)ix * nz + iz] = (REAL)(data[(long)ix * nz + iz] +
                    0.5 * (model[(long)ix * nz + iz] + model[(long)ix * nz + iz + 1]));
        for (int ix = 0; ix < nx; ix++)
            data[(long)ix * nz + nz - 1] += model[(long)ix * nz + nz - 1];
    } else {
        if (!add) for (long i = 0; i < (long)nz * nx; i++) model[i] = 0;
        for (int ix = 0; ix < nx; ix++)
            for (int iz = 1; iz < nz - 1; iz++)
                model[(long)ix * nz + iz] = (REAL)(model[(long)ix * nz + iz] +
                    0.5 * (data[(long)ix * nz + iz] + data[(long)ix * nz + iz - 1]));
        for (int ix = 0; ix < nx; ix++) {
            model[(long)ix * nz] = (REAL)(model[(long)ix * nz] + 0.5 * data[(long)ix * nz]);
            model[(long)ix * nz + nz - 1] = (REAL)(model[(long)ix * nz + nz - 1] +
                (data[(long)ix * nz + nz - 1] + 0.5 * data[(long)ix * nz + nz - 2]));
        }
    }
}

/* ------------------------------------------------------------------ */
/* Medium preparation, F/prop/src/fdParamElastic.cpp:116-148           */
/* ep = [3][nx][nz] (rho, lambda, mu); dts float-rounded like getFloat */
/* ------------------------------------------------------------------ */
int FN(orc_medium)(int nz, int nx, float dts, int sub_int, const REAL *ep,
                   REAL *rhoxDtw, REAL *rhozDtw, REAL *lamb2MuDtw, REAL *lambDtw, REAL *muxzDtw)
{
    long n = (long)nz * nx;
    REAL dtw = (REAL)dts / (REAL)sub_int;
    REAL *tmp = (REAL *)malloc(sizeof(REAL) * n);
    REAL *tmp2 = (REAL *)malloc(sizeof(REAL) * n);
    if (!tmp || !tmp2) { free(tmp); free(tmp2); return -1; }
    memcpy(tmp, ep, sizeof(REAL) * n);              /* density */
    memcpy(tmp2, ep + 2 * n, sizeof(REAL) * n);     /* mu */
    FN(orc_stagger_x)(1, 0, nz, nx, rhoxDtw, tmp);
    FN(orc_stagger_z)(1, 0, nz, nx, rhozDtw, tmp);
    FN(orc_stagger_x)(1, 0, nz, nx, tmp, tmp2);     /* tmp = Sx' mu */
    FN(orc_stagger_z)(1, 0, nz, nx, muxzDtw, tmp);  /* muxz = Sz' Sx' mu */
    for (long i = 0; i < n; i++) {
        REAL lam = ep[n + i], mu = ep[2 * n + i];
        rhoxDtw[i] = (REAL)(2.0 * dtw / rhoxDtw[i]);
        rhozDtw[i] = (REAL)(2.0 * dtw / rhozDtw[i]);
        lambDtw[i] = (REAL)(2.0 * dtw * lam);
        lamb2MuDtw[i] = (REAL)(2.0 * dtw * (lam + 2 * mu));
        muxzDtw[i] = (REAL)(2.0 * dtw * muxzDtw[i]);
    }
    free(tmp); free(tmp2);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Linear time interpolation coarse<->fine, F/prop/src/interpTimeLinTbb.cpp:9-102 */
/* arrays are [ndev][nt] (time fastest).  sub_int = doubled sub.       */
/* ------------------------------------------------------------------ */
void FN(orc_tinterp)(int adj, int add, int nts, float dts_f, float ots_f, int sub_int, int ndev,
                     REAL *coarse, REAL *fine)
{
    int ntw = (nts - 1) * sub_int + 1;
    REAL dts = (REAL)dts_f, ots = (REAL)ots_f;
    REAL dtw = dts / sub_int, otw = ots;
    REAL scale = (REAL)ntw / (REAL)nts;
    scale = (REAL)(1.0 / FN(orc_sqrt)(scale));
    if (!adj) {
        if (!add) for (long i = 0; i < (long)ndev * ntw; i++) fine[i] = 0;
        for (int d = 0; d < ndev; d++) {
            REAL *m = coarse + (long)d * nts, *f = fine + (long)d * ntw;
            for (int itw = 0; itw < ntw - 1; itw++) {
                REAL tw = otw + itw * dtw;
                REAL w = (tw - ots) / dts;
                int i0 = (int)w;
                w = w - i0;
                f[itw] = (REAL)(f[itw] + (m[i0] * (1.0 - w) + m[i0 + 1] * w) * scale);
            }
            f[ntw - 1] += scale * m[nts - 1];
        }
    } else {
        if (!add) for (long i = 0; i < (long)ndev * nts; i++) coarse[i] = 0;
        for (int d = 0; d < ndev; d++) {
            REAL *m = coarse + (long)d * nts, *f = fine + (long)d * ntw;
            for (int itw = 0; itw < ntw - 1; itw++) {
                REAL tw = otw + itw * dtw;
                REAL w = (tw - ots) / dts;
                int i0 = (int)w;
                w = w - i0;
                m[i0] = (REAL)(m[i0] + scale * f[itw] * (1.0 - w));
                m[i0 + 1] += scale * f[itw] * w;
            }
            m[nts - 1] += scale * f[ntw - 1];
        }
    }
}

/* ------------------------------------------------------------------ */
/* Spatial interpolation weights, F/prop/src/spaceInterpGpu.cpp:11-283 */
/* method: 0 linear, 1 sinc, 2 gauss.  Outputs gpi/w of length        */
/* nDev*nFiltTotal, the unique regular positions (in first-seen order) */
/* and, for every (device, filter) entry, its unique slot.            */
/* ------------------------------------------------------------------ */
static double FN(orc_sinc_pi)(double x)
{
    /* Boost.Math sinc_pi: Taylor series near 0, sin(x)/x elsewhere */
    const double eps = 2.220446049250313e-16;
    const double t0 = eps, t2 = sqrt(eps), tn = sqrt(t2);
    double ax = fabs(x);
    if (ax >= tn) return sin(x) / x;
    double r = 1.0;
    if (ax >= t0) {
        double x2 = x * x;
        r -= x2 / 6.0;
        if (ax >= t2) r += (x2 * x2) / 120.0;
    }
    return r;
}

static double FN(orc_normal_pdf)(double mean, double sd, double x)
{
    double z = (x - mean) / sd;
    return exp(-0.5 * z * z) / (sd * sqrt(2.0 * M_PI));
}

int FN(orc_sinterp_build)(const REAL *zCoord, const REAL *xCoord, int nDev,
                          int nz, float oz_f, float dz_f, int nx, float ox_f, float dx_f,
                          int method, int nFilt, int dipole, float zDipShift, float xDipShift,
                          int *gpi, REAL *w, int *slot, int *uniq, int *nUniq, int *nFiltTotalOut)
{
    REAL oz = (REAL)oz_f, dz = (REAL)dz_f, ox = (REAL)ox_f, dx = (REAL)dx_f;
    if (method == 0) nFilt = 1;
    int nFilt2D = 2 * nFilt;
    int nft;
    if (method == 0) nft = dipole ? 8 : 4;
    else nft = nFilt2D * nFilt2D;   /* intended (2N)^2 stencil; equals the built 4 for nFilt=1 */
    if (method != 0 && dipole) return -2;
    /* checkOutOfBounds, spaceInterpGpu.cpp:364-388 */
    REAL zMax = oz + (nz - 1) * dz, xMax = ox + (nx - 1) * dx;
    REAL zBuf = dz * nFilt, xBuf = dx * nFilt;
    for (int i = 0; i < nDev; i++) {
        if (zCoord[i] >= zMax - zBuf || zCoord[i] <= oz + zBuf) return -3;
        if (xCoord[i] >= xMax - xBuf || xCoord[i] <= ox + xBuf) return -3;
    }
    REAL zDS = (REAL)zDipShift * dz, xDS = (REAL)xDipShift * dx;
    for (int d = 0; d < nDev; d++) {
        int o = d * nft;
        if (method == 0) {
            /* calcLinearWeights, spaceInterpGpu.cpp:78-138 */
            REAL wz = (zCoord[d] - oz) / dz;
            REAL wx = (xCoord[d] - ox) / dx;
            int zr = (int)wz; wz = wz - zr; wz = (REAL)(1.0 - wz);
            int xr = (int)wx; wx = wx - xr; wx = (REAL)(1.0 - wx);
            gpi[o] = xr * nz + zr;           w[o] = wz * wx;
            gpi[o + 1] = gpi[o] + 1;         w[o + 1] = (REAL)((1.0 - wz) * wx);
            gpi[o + 2] = gpi[o] + nz;        w[o + 2] = (REAL)(wz * (1.0 - wx));
            gpi[o + 3] = gpi[o] + nz + 1;    w[o + 3] = (REAL)((1.0 - wz) * (1.0 - wx));
            if (dipole) {
                REAL wzd = (zCoord[d] + zDS - oz) / dz;
                REAL wxd = (xCoord[d] + xDS - ox) / dx;
                int zrd = (int)wzd; wzd = wzd - zrd; wzd = (REAL)(1.0 - wzd);
                int xrd = (int)wxd; wxd = wxd - xrd; wxd = (REAL)(1.0 - wxd);
                gpi[o + 4] = xrd * nz + zrd;      w[o + 4] = (REAL)((-1.0) * wzd * wxd);
                gpi[o + 5] = gpi[o + 4] + 1;      w[o + 5] = (REAL)((-1.0) * (1.0 - wzd) * wxd);
                gpi[o + 6] = gpi[o + 4] + nz;     w[o + 6] = (REAL)((-1.0) * wzd * (1.0 - wxd));
                gpi[o + 7] = gpi[o + 4] + nz + 1; w[o + 7] = (REAL)((-1.0) * (1.0 - wzd) * (1.0 - wxd));
            }
        } else {
            /* calcSincWeights / calcGaussWeights, spaceInterpGpu.cpp:139-211 */
            REAL zi = zCoord[d], xi = xCoord[d];
            int zr = (int)((zi - oz) / dz), xr = (int)((xi - ox) / dx);
            REAL sum = 0;
            for (int ix = 0; ix < nFilt2D; ix++) {
                for (int iz = 0; iz < nFilt2D; iz++) {
                    REAL xc = (xr + ix - nFilt + 1) * dx + ox;
                    REAL zc = (zr + iz - nFilt + 1) * dz + oz;
                    REAL xin = (xi - xc) / dx, zin = (zi - zc) / dz;
                    REAL v;
                    if (method == 1)
                        v = (REAL)(FN(orc_sinc_pi)(M_PI * zin) * FN(orc_sinc_pi)(M_PI * xin));
                    else
                        v = (REAL)(FN(orc_normal_pdf)(xi, 2 * dx, xc) * FN(orc_normal_pdf)(zi, 2 * dz, zc));
                    w[o + nFilt2D * ix + iz] = v;
                    gpi[o + nFilt2D * ix + iz] = nz * (xr + ix - nFilt + 1) + (zr + iz - nFilt + 1);
                    sum += v;
                }
            }
            for (int i = 0; i < nft; i++) w[o + i] = w[o + i] / sum;
        }
    }
    /* convertIrregToReg, spaceInterpGpu.cpp:288-311: unique points in first-seen order */
    int nu = 0;
    for (int i = 0; i < nDev * nft; i++) {
        int s = -1;
        for (int j = 0; j < nu; j++) if (uniq[j] == gpi[i]) { s = j; break; }
        if (s < 0) { uniq[nu] = gpi[i]; s = nu++; }
        slot[i] = s;
    }
    *nUniq = nu;
    *nFiltTotalOut = nft;
    return 0;
}

/* spaceInterpGpu::forward (reg -> irreg) / adjoint, spaceInterpGpu.cpp:313-362 */
void FN(orc_sinterp_apply)(int adj, int add, int nDev, int nft, int nReg, int nt, const int *slot,
                           const REAL *w, REAL *reg, REAL *irreg)
{
    if (!adj) {
        if (!add) for (long i = 0; i < (long)nDev * nt; i++) irreg[i] = 0;
        for (int d = 0; d < nDev; d++)
            for (int f = 0; f < nft; f++) {
                int i1 = d * nft + f, i2 = slot[i1];
                for (int t = 0; t < nt; t++) irreg[(long)d * nt + t] += w[i1] * reg[(long)i2 * nt + t];
            }
    } else {
        if (!add) for (long i = 0; i < (long)nReg * nt; i++) reg[i] = 0;
        for (int d = 0; d < nDev; d++)
            for (int f = 0; f < nft; f++) {
                int i1 = d * nft + f, i2 = slot[i1];
                for (int t = 0; t < nt; t++) reg[(long)i2 * nt + t] += w[i1] * irreg[(long)d * nt + t];
            }
    }
}

/* ------------------------------------------------------------------ */
/* One fine time step (forward / adjoint), K:234-529                   */
/* p0 = o (overwritten with n), p1 = c                                 */
/* ------------------------------------------------------------------ */
#define ORC_DM(f, i, s, cc) (cc[0] * (f[(i)] - f[(i) - (s)]) + cc[1] * (f[(i) + (s)] - f[(i) - 2 * (s)]) + \
                             cc[2] * (f[(i) + 2 * (s)] - f[(i) - 3 * (s)]) + cc[3] * (f[(i) + 3 * (s)] - f[(i) - 4 * (s)]))
#define ORC_DP(f, i, s, cc) (cc[0] * (f[(i) + (s)] - f[(i)]) + cc[1] * (f[(i) + 2 * (s)] - f[(i) - (s)]) + \
                             cc[2] * (f[(i) + 3 * (s)] - f[(i) - 2 * (s)]) + cc[3] * (f[(i) + 4 * (s)] - f[(i) - 3 * (s)]))

typedef struct {
    REAL *rhox, *rhoz, *l2m, *lam, *muxz;
} FN(orc_medium_t);

static void FN(orc_step_fwd)(const FN(orc_grid_t) *g, const FN(orc_medium_t) *m, REAL **p0, REAL **p1)
{
    const int nz = g->nz, nx = g->nx;
    const REAL *zc = g->zc, *xc = g->xc;
    REAL *ovx = p0[0], *ovz = p0[1], *osxx = p0[2], *oszz = p0[3], *osxz = p0[4];
    const REAL *cvx = p1[0], *cvz = p1[1], *csxx = p1[2], *cszz = p1[3], *csxz = p1[4];
    #pragma omp parallel for schedule(static)
    for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++) {
        for (int iz = ORC_FAT; iz < nz - ORC_FAT; iz++) {
            long i = (long)ix * nz + iz;
            ovx[i] = ovx[i] + m->rhox[i] * (ORC_DM(csxx, i, nz, xc) + ORC_DP(csxz, i, 1, zc));
            ovz[i] = ovz[i] + m->rhoz[i] * (ORC_DM(cszz, i, 1, zc) + ORC_DP(csxz, i, nz, xc));
            REAL dvxdx = ORC_DP(cvx, i, nz, xc), dvzdz = ORC_DP(cvz, i, 1, zc);
            osxx[i] = osxx[i] + m->l2m[i] * dvxdx + m->lam[i] * dvzdz;
            oszz[i] = oszz[i] + m->lam[i] * dvxdx + m->l2m[i] * dvzdz;
            osxz[i] = osxz[i] + m->muxz[i] * (ORC_DM(cvx, i, 1, zc) + ORC_DM(cvz, i, nz, xc));
        }
    }
}

/* Adjoint step: scaled copies are formed over the whole grid first (the
 * reference forms them per shared-memory tile, K:395-470). */
static void FN(orc_step_adj)(const FN(orc_grid_t) *g, const FN(orc_medium_t) *m, REAL **p0, REAL **p1,
                             REAL **scr)
{
    const int nz = g->nz, nx = g->nx;
    const long n = (long)nz * nx;
    const REAL *zc = g->zc, *xc = g->xc;
    REAL *vxr = scr[0], *vzr = scr[1], *xxl2 = scr[2], *xxl = scr[3], *zzl2 = scr[4], *zzl = scr[5], *xzm = scr[6];
    const REAL *cvx = p1[0], *cvz = p1[1], *csxx = p1[2], *cszz = p1[3], *csxz = p1[4];
    #pragma omp parallel for schedule(static)
    for (long ix = 0; ix < nx; ix++) {
        for (long i = ix * nz; i < (ix + 1) * nz; i++) {
            vxr[i] = m->rhox[i] * cvx[i];
            vzr[i] = m->rhoz[i] * cvz[i];
            xxl2[i] = m->l2m[i] * csxx[i];
            xxl[i] = m->lam[i] * csxx[i];
            zzl2[i] = m->l2m[i] * cszz[i];
            zzl[i] = m->lam[i] * cszz[i];
            xzm[i] = m->muxz[i] * csxz[i];
        }
    }
    (void)n;
    REAL *ovx = p0[0], *ovz = p0[1], *osxx = p0[2], *oszz = p0[3], *osxz = p0[4];
    #pragma omp parallel for schedule(static)
    for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++) {
        for (int iz = ORC_FAT; iz < nz - ORC_FAT; iz++) {
            long i = (long)ix * nz + iz;
            ovx[i] = ovx[i] - ORC_DM(xxl2, i, nz, xc) - ORC_DM(zzl, i, nz, xc) - ORC_DP(xzm, i, 1, zc);
            ovz[i] = ovz[i] - ORC_DM(xxl, i, 1, zc) - ORC_DM(zzl2, i, 1, zc) - ORC_DP(xzm, i, nz, xc);
            osxx[i] = osxx[i] - ORC_DP(vxr, i, nz, xc);
            oszz[i] = oszz[i] - ORC_DP(vzr, i, 1, zc);
            osxz[i] = osxz[i] - ORC_DM(vxr, i, 1, zc) - ORC_DM(vzr, i, nz, xc);
        }
    }
}

/* dampCosineEdge, K:1192-1221: both time levels, pad band only */
static void FN(orc_damp)(const FN(orc_grid_t) *g, REAL **p0, REAL **p1)
{
    const int nz = g->nz, nx = g->nx;
    #pragma omp parallel for schedule(static)
    for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++) {
        for (int iz = ORC_FAT; iz < nz - ORC_FAT; iz++) {
            int a = iz - ORC_FAT, b = ix - ORC_FAT, c = nz - iz - 1 - ORC_FAT, d = nx - ix - 1 - ORC_FAT;
            int dist = a; if (b < dist) dist = b; if (c < dist) dist = c; if (d < dist) dist = d;
            if (dist < g->minPad) {
                REAL dmp = g->damp[dist];
                long i = (long)ix * nz + iz;
                for (int f = 0; f < 5; f++) { p0[f][i] *= dmp; p1[f][i] *= dmp; }
            }
        }
    }
}

/* ---------------------------------------------------------------- */
/* Free surface at z = 2*FAT (surfaceCondition = 1)                  */
/* ---------------------------------------------------------------- */
#define ORC_SURF (2 * ORC_FAT)

/* ker_step_fwd_surface_top, K:543-587: on the current level, in place */
static void FN(orc_fs_top)(const FN(orc_grid_t) *g, REAL **c)
{
    const int nz = g->nz, nx = g->nx;
    for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++) {
        REAL *vx = c[0] + (long)ix * nz, *vz = c[1] + (long)ix * nz, *szz = c[3] + (long)ix * nz,
             *sxz = c[4] + (long)ix * nz;
        const int s = ORC_SURF;
        szz[s] = 0;
        for (int k = 1; k <= 4; k++) szz[s - k] = -szz[s + k];
        for (int k = 0; k < 4; k++) sxz[s - k] = -sxz[s + 1 + k];
        for (int k = 1; k <= 4; k++) vx[s - k] = 0;
        for (int k = 0; k <= 4; k++) vz[s - k] = 0;
    }
}

/* ker_step_fwd_surface_body, K:589-776: the standard update below the
 * surface, vx and the reduced sigmaxx coefficient (l2m - lam^2/l2m) on it,
 * nothing above it */
static void FN(orc_step_fwd_fs)(const FN(orc_grid_t) *g, const FN(orc_medium_t) *m, REAL **p0, REAL **p1)
{
    const int nz = g->nz, nx = g->nx;
    const REAL *zc = g->zc, *xc = g->xc;
    REAL *ovx = p0[0], *ovz = p0[1], *osxx = p0[2], *oszz = p0[3], *osxz = p0[4];
    const REAL *cvx = p1[0], *cvz = p1[1], *csxx = p1[2], *cszz = p1[3], *csxz = p1[4];
    #pragma omp parallel for schedule(static)
    for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++) {
        for (int iz = ORC_SURF; iz < nz - ORC_FAT; iz++) {
            long i = (long)ix * nz + iz;
            ovx[i] = ovx[i] + m->rhox[i] * (ORC_DM(csxx, i, nz, xc) + ORC_DP(csxz, i, 1, zc));
            REAL dvxdx = ORC_DP(cvx, i, nz, xc);
            if (iz == ORC_SURF) {
                osxx[i] = osxx[i] + (m->l2m[i] - (m->lam[i] * m->lam[i] / m->l2m[i])) * dvxdx;
                continue;
            }
            ovz[i] = ovz[i] + m->rhoz[i] * (ORC_DM(cszz, i, 1, zc) + ORC_DP(csxz, i, nz, xc));
            REAL dvzdz = ORC_DP(cvz, i, 1, zc);
            osxx[i] = osxx[i] + m->l2m[i] * dvxdx + m->lam[i] * dvzdz;
            oszz[i] = oszz[i] + m->lam[i] * dvxdx + m->l2m[i] * dvzdz;
            osxz[i] = osxz[i] + m->muxz[i] * (ORC_DM(cvx, i, 1, zc) + ORC_DM(cvz, i, nz, xc));
        }
    }
}

/* Adjoint of the free-surface step in the loop form of orc_step_adj:
 * p0 <- M^T (p0 + U^T p1), with U the masked update above (its products
 * vanish where U does not update) and M the top pass (M^T returns the mirrored
 * stress rows to their sources below the surface and zeroes the rows M
 * overwrites). */
static void FN(orc_step_adj_fs)(const FN(orc_grid_t) *g, const FN(orc_medium_t) *m, REAL **p0, REAL **p1,
                                REAL **scr)
{
    const int nz = g->nz, nx = g->nx;
    const REAL *zc = g->zc, *xc = g->xc;
    REAL *vxr = scr[0], *vzr = scr[1], *xxl2 = scr[2], *xxl = scr[3], *zzl2 = scr[4], *zzl = scr[5], *xzm = scr[6];
    const REAL *cvx = p1[0], *cvz = p1[1], *csxx = p1[2], *cszz = p1[3], *csxz = p1[4];
    #pragma omp parallel for schedule(static)
    for (long ix = 0; ix < nx; ix++) {
        for (long iz = 0; iz < nz; iz++) {
            const long i = ix * nz + iz;
            const int below = iz > ORC_SURF, on = iz == ORC_SURF;
            vxr[i] = (below || on) ? m->rhox[i] * cvx[i] : 0;
            vzr[i] = below ? m->rhoz[i] * cvz[i] : 0;
            xxl2[i] = below ? m->l2m[i] * csxx[i]
                            : on ? (m->l2m[i] - (m->lam[i] * m->lam[i] / m->l2m[i])) * csxx[i] : 0;
            xxl[i] = below ? m->lam[i] * csxx[i] : 0;
            zzl2[i] = below ? m->l2m[i] * cszz[i] : 0;
            zzl[i] = below ? m->lam[i] * cszz[i] : 0;
            xzm[i] = below ? m->muxz[i] * csxz[i] : 0;
        }
    }
    REAL *ovx = p0[0], *ovz = p0[1], *osxx = p0[2], *oszz = p0[3], *osxz = p0[4];
    #pragma omp parallel for schedule(static)
    for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++) {
        for (int iz = ORC_FAT; iz < nz - ORC_FAT; iz++) {
            long i = (long)ix * nz + iz;
            ovx[i] = ovx[i] - ORC_DM(xxl2, i, nz, xc) - ORC_DM(zzl, i, nz, xc) - ORC_DP(xzm, i, 1, zc);
            ovz[i] = ovz[i] - ORC_DM(xxl, i, 1, zc) - ORC_DM(zzl2, i, 1, zc) - ORC_DP(xzm, i, nz, xc);
            osxx[i] = osxx[i] - ORC_DP(vxr, i, nz, xc);
            oszz[i] = oszz[i] - ORC_DP(vzr, i, 1, zc);
            osxz[i] = osxz[i] - ORC_DM(vxr, i, 1, zc) - ORC_DM(vzr, i, nz, xc);
        }
        /* M^T on the column */
        REAL *vx = ovx + (long)ix * nz, *vz = ovz + (long)ix * nz, *szz = oszz + (long)ix * nz,
             *sxz = osxz + (long)ix * nz;
        const int sf = ORC_SURF;
        for (int k = 1; k <= 4; k++) { szz[sf + k] = szz[sf + k] - szz[sf - k]; szz[sf - k] = 0; }
        szz[sf] = 0;
        for (int k = 0; k < 4; k++) { sxz[sf + 1 + k] = sxz[sf + 1 + k] - sxz[sf - k]; sxz[sf - k] = 0; }
        for (int k = 1; k <= 4; k++) vx[sf - k] = 0;
        for (int k = 0; k <= 4; k++) vz[sf - k] = 0;
    }
}

/* dampCosineEdge_freesurface, K:1223-1252: no taper at the top */
static void FN(orc_damp_fs)(const FN(orc_grid_t) *g, REAL **p0, REAL **p1)
{
    const int nz = g->nz, nx = g->nx;
    #pragma omp parallel for schedule(static)
    for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++) {
        for (int iz = ORC_FAT; iz < nz - ORC_FAT; iz++) {
            int b = ix - ORC_FAT, c = nz - iz - 1 - ORC_FAT, d = nx - ix - 1 - ORC_FAT;
            int dist = b; if (c < dist) dist = c; if (d < dist) dist = d;
            if (dist < g->minPad) {
                REAL dmp = g->damp[dist];
                long i = (long)ix * nz + iz;
                for (int f = 0; f < 5; f++) { p0[f][i] *= dmp; p1[f][i] *= dmp; }
            }
        }
    }
}

static void FN(orc_swap)(REAL **p0, REAL **p1)
{
    for (int f = 0; f < 5; f++) { REAL *t = p0[f]; p0[f] = p1[f]; p1[f] = t; }
}

/* field order everywhere: 0 vx, 1 vz, 2 sigmaxx, 3 sigmazz, 4 sigmaxz.
 * position lists: 0 center (sxx, szz), 1 x-shifted (vx), 2 z-shifted (vz),
 * 3 xz-shifted (sxz).  Signals are [nPoints][nt], time fastest. */
static const int FN(orc_field_grid)[5] = {1, 2, 0, 0, 3};

/* ker_inject_interp_source_*, K:172-189 (coarse signal, linear time interp) */
static void FN(orc_inject_coarse)(const FN(orc_grid_t) *g, REAL **p, REAL *const *sig, const int *const *pos,
                                  const int *npos, int its, int fi)
{
    for (int f = 0; f < 5; f++) {
        int gr = FN(orc_field_grid)[f];
        for (int k = 0; k < npos[gr]; k++) {
            const REAL *s = sig[f] + (long)g->nts * k;
            p[f][pos[gr][k]] += s[its] * g->filt[fi] + s[its + 1] * g->filt[g->h + fi];
        }
    }
}

/* ker_record_interp_data_* / ker_record_interp_source_*, K:7-60, 100-116 */
static void FN(orc_extract_coarse)(const FN(orc_grid_t) *g, REAL **p, REAL *const *out, const int *const *pos,
                                   const int *npos, int its, int fi)
{
    for (int f = 0; f < 5; f++) {
        int gr = FN(orc_field_grid)[f];
        for (int k = 0; k < npos[gr]; k++) {
            REAL *o = out[f] + (long)g->nts * k;
            REAL v = p[f][pos[gr][k]];
            o[its] += v * g->filt[fi];
            o[its + 1] += v * g->filt[g->h + fi];
        }
    }
}

/* ker_inject_source_*, K:121-168 (fine-time Born source) */
static void FN(orc_inject_fine)(const FN(orc_grid_t) *g, REAL **p, REAL *const *sig, const int *const *pos,
                                const int *npos, int itw)
{
    for (int f = 0; f < 5; f++) {
        int gr = FN(orc_field_grid)[f];
        for (int k = 0; k < npos[gr]; k++) p[f][pos[gr][k]] += sig[f][(long)k * g->ntw + itw];
    }
}

/* ------------------------------------------------------------------ */
/* Nonlinear propagation on the regular grid                           */
/* propShotsElasticFwdGpu / propShotsElasticAdjGpu,                    */
/* F/prop/src/nonlinearPropElasticGpuFunctions.cu:561-648, 932-1027    */
/* model: 5 source arrays [nSrcReg(grid)][nts]; data: 5 [nRecReg][nts] */
/* fwd overwrites data, adj overwrites model                           */
/* ------------------------------------------------------------------ */
/* interpWavefield (K:1258-1291): coarse-time samples of the new level of all
 * five fields, W [nts][5][nx][nz]; every interior cell (the reference kernel
 * omits the FAT offset in z at K:1262 and so never writes the last four
 * interior rows; this restatement writes them). */
static void FN(orc_save_wavefield)(const FN(orc_grid_t) *g, REAL **p, REAL *W, int its, int fi)
{
    const long n = (long)g->nz * g->nx;
#pragma omp parallel for
    for (int ix = ORC_FAT; ix < g->nx - ORC_FAT; ix++)
        for (int f = 0; f < 5; f++)
            for (int iz = ORC_FAT; iz < g->nz - ORC_FAT; iz++) {
                const long i = (long)ix * g->nz + iz;
                W[((long)its * 5 + f) * n + i] += p[f][i] * g->filt[fi];
                W[((long)(its + 1) * 5 + f) * n + i] += p[f][i] * g->filt[g->h + fi];
            }
}

/* wavefield: NULL, or [nts][5][nx][nz] overwritten with the saved wavefield
 * (propShotsElastic{Fwd,Adj}GpuWavefield, F/prop/src/nonlinearPropElasticGpuFunctions.cu:649-760, 1029-1110) */
int FN(orc_nl_prop_fs)(int adj, int nz, int nx, float dz, float dx, int nts, float dts, int sub_int,
                       int minPad, float alphaCos, REAL *const *medium5, REAL *const *model, REAL *const *data,
                       const int *const *srcPos, const int *nSrc, const int *const *recPos, const int *nRec,
                       REAL *wavefield, int surface)
{
    FN(orc_grid_t) g;
    if (FN(orc_grid_init)(&g, nz, nx, dz, dx, nts, dts, sub_int, minPad, alphaCos)) return -1;
    FN(orc_medium_t) m = {medium5[0], medium5[1], medium5[2], medium5[3], medium5[4]};
    long n = (long)nz * nx;
    REAL *buf = (REAL *)calloc(17 * n, sizeof(REAL));
    if (!buf) return -2;
    REAL *p0[5], *p1[5], *scr[7];
    for (int f = 0; f < 5; f++) { p0[f] = buf + f * n; p1[f] = buf + (5 + f) * n; }
    for (int f = 0; f < 7; f++) scr[f] = buf + (10 + f) * n;
    if (wavefield) memset(wavefield, 0, sizeof(REAL) * 5 * (size_t)nts * n);
    if (!adj) {
        for (int f = 0; f < 5; f++) memset(data[f], 0, sizeof(REAL) * nts * nRec[FN(orc_field_grid)[f]]);
        for (int its = 0; its < nts - 1; its++)
            for (int it2 = 1; it2 < g.S + 1; it2++) {
                if (surface) {
                    FN(orc_fs_top)(&g, p1);
                    FN(orc_step_fwd_fs)(&g, &m, p0, p1);
                } else {
                    FN(orc_step_fwd)(&g, &m, p0, p1);
                }
                FN(orc_inject_coarse)(&g, p0, model, srcPos, nSrc, its, it2 - 1);
                if (surface) FN(orc_damp_fs)(&g, p0, p1);
                else FN(orc_damp)(&g, p0, p1);
                if (wavefield) FN(orc_save_wavefield)(&g, p0, wavefield, its, it2);
                FN(orc_extract_coarse)(&g, p0, data, recPos, nRec, its, it2);
                FN(orc_swap)(p0, p1);
            }
    } else {
        for (int f = 0; f < 5; f++) memset(model[f], 0, sizeof(REAL) * nts * nSrc[FN(orc_field_grid)[f]]);
        for (int its = nts - 2; its > -1; its--)
            for (int it2 = g.S - 1; it2 > -1; it2--) {
                if (surface) FN(orc_step_adj_fs)(&g, &m, p0, p1, scr);
                else FN(orc_step_adj)(&g, &m, p0, p1, scr);
                FN(orc_inject_coarse)(&g, p0, data, recPos, nRec, its, it2 + 1);
                if (surface) FN(orc_damp_fs)(&g, p0, p1);
                else FN(orc_damp)(&g, p0, p1);
                if (wavefield) FN(orc_save_wavefield)(&g, p0, wavefield, its, it2);
                FN(orc_extract_coarse)(&g, p0, model, srcPos, nSrc, its, it2);
                FN(orc_swap)(p0, p1);
            }
    }
    free(buf);
    return 0;
}

int FN(orc_nl_prop)(int adj, int nz, int nx, float dz, float dx, int nts, float dts, int sub_int,
                    int minPad, float alphaCos, REAL *const *medium5, REAL *const *model, REAL *const *data,
                    const int *const *srcPos, const int *nSrc, const int *const *recPos, const int *nRec)
{
    return FN(orc_nl_prop_fs)(adj, nz, nx, dz, dx, nts, dts, sub_int, minPad, alphaCos, medium5, model, data,
                              srcPos, nSrc, recPos, nRec, NULL, 0);
}

int FN(orc_nl_prop_wf)(int adj, int nz, int nx, float dz, float dx, int nts, float dts, int sub_int,
                       int minPad, float alphaCos, REAL *const *medium5, REAL *const *model, REAL *const *data,
                       const int *const *srcPos, const int *nSrc, const int *const *recPos, const int *nRec,
                       REAL *wavefield)
{
    return FN(orc_nl_prop_fs)(adj, nz, nx, dz, dx, nts, dts, sub_int, minPad, alphaCos, medium5, model, data,
                              srcPos, nSrc, recPos, nRec, wavefield, 0);
}

/* ------------------------------------------------------------------ */
/* Born secondary source / imaging condition, K:1381-1459, 1538-1613   */
/* ------------------------------------------------------------------ */
static void FN(orc_imaging_fwd)(const FN(orc_grid_t) *g, const REAL *Wvx, const REAL *Wvz, REAL *const *dm,
                                REAL **ss, int its)
{
    const int nz = g->nz, nx = g->nx;
    const long n = (long)nz * nx;
    const REAL *zc = g->zc, *xc = g->xc;
    const REAL *vxc = Wvx + its * n, *vzc = Wvz + its * n;
    #pragma omp parallel for schedule(static)
    for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++) {
        for (int iz = ORC_FAT; iz < nz - ORC_FAT; iz++) {
            long i = (long)ix * nz + iz;
            REAL dvx_dx = ORC_DP(vxc, i, nz, xc);
            REAL dvz_dz = ORC_DP(vzc, i, 1, zc);
            if (its == 0) {
                ss[0][i] = dm[0][i] * (-Wvx[n + i]) * g->dts_inv;
                ss[1][i] = dm[1][i] * (-Wvz[n + i]) * g->dts_inv;
            } else if (its == g->nts - 1) {
                ss[0][i] = dm[0][i] * (Wvx[(its - 1) * n + i]) * g->dts_inv;
                ss[1][i] = dm[1][i] * (Wvz[(its - 1) * n + i]) * g->dts_inv;
            } else {
                ss[0][i] = dm[0][i] * (Wvx[(its - 1) * n + i] - Wvx[(its + 1) * n + i]) * g->dts_inv;
                ss[1][i] = dm[1][i] * (Wvz[(its - 1) * n + i] - Wvz[(its + 1) * n + i]) * g->dts_inv;
            }
            ss[2][i] = (REAL)(dm[2][i] * (dvx_dx + dvz_dz) + 2.0 * dm[3][i] * dvx_dx);
            ss[3][i] = (REAL)(dm[2][i] * (dvx_dx + dvz_dz) + 2.0 * dm[3][i] * dvz_dz);
            ss[4][i] = dm[4][i] * (ORC_DM(vxc, i, 1, zc) + ORC_DM(vzc, i, nz, xc));
        }
    }
}

static void FN(orc_imaging_adj)(const FN(orc_grid_t) *g, const REAL *Wvx, const REAL *Wvz, REAL *const *dm,
                                REAL *const *ss, int its)
{
    const int nz = g->nz, nx = g->nx;
    const long n = (long)nz * nx;
    const REAL *zc = g->zc, *xc = g->xc;
    const REAL *vxc = Wvx + its * n, *vzc = Wvz + its * n;
    #pragma omp parallel for schedule(static)
    for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++) {
        for (int iz = ORC_FAT; iz < nz - ORC_FAT; iz++) {
            long i = (long)ix * nz + iz;
            REAL dvx_dx = ORC_DP(vxc, i, nz, xc);
            REAL dvz_dz = ORC_DP(vzc, i, 1, zc);
            if (its == 0) {
                dm[0][i] += ss[0][i] * (-Wvx[n + i]) * g->dts_inv;
                dm[1][i] += ss[1][i] * (-Wvz[n + i]) * g->dts_inv;
            } else if (its == g->nts - 1) {
                dm[0][i] += ss[0][i] * (Wvx[(its - 1) * n + i]) * g->dts_inv;
                dm[1][i] += ss[1][i] * (Wvz[(its - 1) * n + i]) * g->dts_inv;
            } else {
                dm[0][i] += ss[0][i] * (Wvx[(its - 1) * n + i] - Wvx[(its + 1) * n + i]) * g->dts_inv;
                dm[1][i] += ss[1][i] * (Wvz[(its - 1) * n + i] - Wvz[(its + 1) * n + i]) * g->dts_inv;
            }
            dm[2][i] += (ss[2][i] + ss[3][i]) * (dvx_dx + dvz_dz);
            dm[3][i] = (REAL)(dm[3][i] + 2.0 * (dvx_dx * ss[2][i] + dvz_dz * ss[3][i]));
            dm[4][i] += ss[4][i] * (ORC_DM(vxc, i, 1, zc) + ORC_DM(vzc, i, nz, xc));
        }
    }
}

/* Source wavefield with coarse Vx/Vz history (BornElasticGpuFunctions.cu:746-768,
 * interpWavefieldSingleComp K:1337-1346).  W is [nts][nz][nx-major] per comp. */
static void FN(orc_born_source)(const FN(orc_grid_t) *g, const FN(orc_medium_t) *m, REAL **p0, REAL **p1,
                                REAL *const *srcDtw, const int *const *srcPos, const int *nSrc, REAL *Wvx, REAL *Wvz)
{
    const int nz = g->nz, nx = g->nx;
    const long n = (long)nz * nx;
    for (int its = 0; its < g->nts - 1; its++)
        for (int it2 = 1; it2 < g->S + 1; it2++) {
            int itw = its * g->S + it2;
            FN(orc_step_fwd)(g, m, p0, p1);
            FN(orc_inject_fine)(g, p0, srcDtw, srcPos, nSrc, itw - 1);
            FN(orc_damp)(g, p0, p1);
            REAL f0 = g->filt[it2], f1 = g->filt[g->h + it2];
            #pragma omp parallel for schedule(static)
            for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++)
                for (int iz = ORC_FAT; iz < nz - ORC_FAT; iz++) {
                    long i = (long)ix * nz + iz;
                    Wvx[its * n + i] += p0[0][i] * f0;
                    Wvx[(its + 1) * n + i] += p0[0][i] * f1;
                    Wvz[its * n + i] += p0[1][i] * f0;
                    Wvz[(its + 1) * n + i] += p0[1][i] * f1;
                }
            FN(orc_swap)(p0, p1);
        }
}

/* BornShotsFwdGpu / BornShotsAdjGpu (non-stream path),
 * F/prop/src/BornElasticGpuFunctions.cu:719-849, 1100-1191.
 * srcDtw: 5 fine-time source arrays [nSrcReg][ntw]; dm: 5 staggered+scaled
 * perturbations [nx][nz]; data: 5 [nRecReg][nts].
 * fwd overwrites data; adj ACCUMULATES into dm (the reference copies dm in). */
int FN(orc_born_prop)(int adj, int nz, int nx, float dz, float dx, int nts, float dts, int sub_int,
                      int minPad, float alphaCos, REAL *const *medium5, REAL *const *srcDtw, REAL *const *dm,
                      REAL *const *data, const int *const *srcPos, const int *nSrc, const int *const *recPos,
                      const int *nRec)
{
    FN(orc_grid_t) g;
    if (FN(orc_grid_init)(&g, nz, nx, dz, dx, nts, dts, sub_int, minPad, alphaCos)) return -1;
    FN(orc_medium_t) m = {medium5[0], medium5[1], medium5[2], medium5[3], medium5[4]};
    const long n = (long)nz * nx;
    REAL *buf = (REAL *)calloc(27 * n, sizeof(REAL));
    REAL *W = (REAL *)calloc(2 * (long)nts * n, sizeof(REAL));
    if (!buf || !W) { free(buf); free(W); return -2; }
    REAL *Wvx = W, *Wvz = W + (long)nts * n;
    REAL *p0[5], *p1[5], *scr[7], *ssL[5], *ssR[5];
    for (int f = 0; f < 5; f++) { p0[f] = buf + f * n; p1[f] = buf + (5 + f) * n; }
    for (int f = 0; f < 7; f++) scr[f] = buf + (10 + f) * n;
    for (int f = 0; f < 5; f++) { ssL[f] = buf + (17 + f) * n; ssR[f] = buf + (22 + f) * n; }

    FN(orc_born_source)(&g, &m, p0, p1, srcDtw, srcPos, nSrc, Wvx, Wvz);
    memset(buf, 0, sizeof(REAL) * 27 * n);
    for (int f = 0; f < 5; f++) { p0[f] = buf + f * n; p1[f] = buf + (5 + f) * n; }

    if (!adj) {
        for (int f = 0; f < 5; f++) memset(data[f], 0, sizeof(REAL) * nts * nRec[FN(orc_field_grid)[f]]);
        FN(orc_imaging_fwd)(&g, Wvx, Wvz, dm, ssL, 0);
        for (int its = 0; its < nts - 1; its++) {
            FN(orc_imaging_fwd)(&g, Wvx, Wvz, dm, ssR, its + 1);
            for (int it2 = 1; it2 < g.S + 1; it2++) {
                FN(orc_step_fwd)(&g, &m, p0, p1);
                REAL f0 = g.filt[it2 - 1], f1 = g.filt[g.h + it2 - 1];
                #pragma omp parallel for schedule(static)
                for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++)
                    for (int iz = ORC_FAT; iz < nz - ORC_FAT; iz++) {
                        long i = (long)ix * nz + iz;
                        for (int f = 0; f < 5; f++) p0[f][i] += ssL[f][i] * f0 + ssR[f][i] * f1;
                    }
                FN(orc_damp)(&g, p0, p1);
                FN(orc_extract_coarse)(&g, p0, data, recPos, nRec, its, it2);
                FN(orc_swap)(p0, p1);
            }
            for (int f = 0; f < 5; f++) { REAL *t = ssL[f]; ssL[f] = ssR[f]; ssR[f] = t; memset(ssR[f], 0, sizeof(REAL) * n); }
        }
    } else {
        for (int its = nts - 2; its > -1; its--) {
            for (int it2 = g.S - 1; it2 > -1; it2--) {
                FN(orc_step_adj)(&g, &m, p0, p1, scr);
                FN(orc_inject_coarse)(&g, p0, data, recPos, nRec, its, it2 + 1);
                FN(orc_damp)(&g, p0, p1);
                REAL f0 = g.filt[it2], f1 = g.filt[g.h + it2];
                #pragma omp parallel for schedule(static)
                for (int ix = ORC_FAT; ix < nx - ORC_FAT; ix++)
                    for (int iz = ORC_FAT; iz < nz - ORC_FAT; iz++) {
                        long i = (long)ix * nz + iz;
                        for (int f = 0; f < 5; f++) { ssL[f][i] += p0[f][i] * f0; ssR[f][i] += p0[f][i] * f1; }
                    }
                FN(orc_swap)(p0, p1);
            }
            FN(orc_imaging_adj)(&g, Wvx, Wvz, dm, ssR, its + 1);
            for (int f = 0; f < 5; f++) { REAL *t = ssL[f]; ssL[f] = ssR[f]; ssR[f] = t; memset(ssL[f], 0, sizeof(REAL) * n); }
        }
        FN(orc_imaging_adj)(&g, Wvx, Wvz, dm, ssR, 0);
    }
    free(buf); free(W);
    return 0;
}

#undef ORC_DM
#undef ORC_DP
