// Host side of the engine: finite-difference parameters and QC, medium
// preparation, staggering, spatial and temporal interpolation of the
// acquisition, the multi-shot operators, and the extern "C" boundary.
//
// Restates (paths relative to the reference project, F = elastic_iso_lib/elastic_iso_float/prop):
//   fdParamElastic            F/src/fdParamElastic.cpp:12-332
//   staggerX / staggerZ       F/src/stagger.cpp:18-114
//   spaceInterpGpu            F/src/spaceInterpGpu.cpp:11-362
//   interpTimeLinTbb          F/src/interpTimeLinTbb.cpp:9-102
//   nonlinearPropElasticGpu   F/src/nonlinearPropElasticGpu.cpp:43-473 (per-shot host prep)
//   seismicElasticOperator2D  F/include/seismicElasticOperator2D.cpp:27-117 (Born source prep)
//   nonlinearPropElasticShotsGpu::forward/adjoint  F/src/nonlinearPropElasticShotsGpu.cpp:80-422
//   BornElasticShotsGpu::forward/adjoint           F/src/BornElasticShotsGpu.cpp:85-378
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <sstream>
#include <exception>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "eio_internal.h"

#define EIO_API extern "C" __attribute__((visibility("default")))

namespace eio {

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

// ------------------------------------------------------------------ fdParam
void stagger_x(int adj, int add, int nz, int nx, float* model, float* data) {
    const long long n = (long long)nz * nx;
    if (!adj) {
        if (!add) std::fill(data, data + n, 0.f);
#pragma omp parallel for schedule(static)
        for (int ix = 0; ix < nx - 1; ix++)
            for (int iz = 0; iz < nz; iz++) {
                const long long i = (long long)ix * nz + iz;
                data[i] = (float)(data[i] + 0.5 * (model[i] + model[i + nz]));
            }
        for (int iz = 0; iz < nz; iz++) data[(long long)(nx - 1) * nz + iz] += model[(long long)(nx - 1) * nz + iz];
    } else {
        if (!add) std::fill(model, model + n, 0.f);
#pragma omp parallel for schedule(static)
        for (int ix = 1; ix < nx - 1; ix++)
            for (int iz = 0; iz < nz; iz++) {
                const long long i = (long long)ix * nz + iz;
                model[i] = (float)(model[i] + 0.5 * (data[i] + data[i - nz]));
            }
        for (int iz = 0; iz < nz; iz++) {
            model[iz] = (float)(model[iz] + 0.5 * data[iz]);
            const long long l = (long long)(nx - 1) * nz + iz;
            model[l] = (float)(model[l] + (data[l] + 0.5 * data[l - nz]));
        }
    }
}

void stagger_z(int adj, int add, int nz, int nx, float* model, float* data) {
    const long long n = (long long)nz * nx;
    if (!adj) {
        if (!add) std::fill(data, data + n, 0.f);
#pragma omp parallel for schedule(static)
        for (int ix = 0; ix < nx; ix++) {
            float* d = data + (long long)ix * nz;
            const float* m = model + (long long)ix * nz;
            for (int iz = 0; iz < nz - 1; iz++) d[iz] = (float)(d[iz] + 0.5 * (m[iz] + m[iz + 1]));
            d[nz - 1] += m[nz - 1];
        }
    } else {
        if (!add) std::fill(model, model + n, 0.f);
#pragma omp parallel for schedule(static)
        for (int ix = 0; ix < nx; ix++) {
            float* m = model + (long long)ix * nz;
            const float* d = data + (long long)ix * nz;
            for (int iz = 1; iz < nz - 1; iz++) m[iz] = (float)(m[iz] + 0.5 * (d[iz] + d[iz - 1]));
            m[0] = (float)(m[0] + 0.5 * d[0]);
            m[nz - 1] = (float)(m[nz - 1] + (d[nz - 1] + 0.5 * d[nz - 2]));
        }
    }
}

static std::string fmt(double v) {
    std::ostringstream s;
    s << v;
    return s.str();
}

void build_fdparam(const eio_fd_params& pin, const float* ep, FdParam& o) {
    eio_fd_params p = pin;
    if (p.nts < 2) throw Error(EIO_ERR_ARG, "nts must be >= 2");
    if (p.nz <= 0 || p.nx <= 0) throw Error(EIO_ERR_ARG, "nz and nx must be positive");
    if (p.surfaceCondition != 0 && p.surfaceCondition != 1)
        throw Error(EIO_ERR_ARG, "surfaceCondition must be 0 or 1");
    o.S = 2 * p.sub;
    if (o.S > SUB_MAX || o.S >= SUB_MAX)
        throw Error(EIO_ERR_QC, "**** ERROR: 2*_sub is greater than the allowed SUB_MAX value. " +
                                    std::to_string(o.S) + " > " + std::to_string(SUB_MAX) + " ****");
    if (p.sub < 1) throw Error(EIO_ERR_ARG, "sub must be >= 1");
    o.ntw = (p.nts - 1) * o.S + 1;
    o.dtw = p.dts / float(o.S);
    if (p.mod_par == 2) { p.dz *= 1000.f; p.dx *= 1000.f; p.oz *= 1000.f; p.ox *= 1000.f; }
    // fdParamElastic.cpp:43-44: with the free surface the top pad is no taper
    const int zPad = p.surfaceCondition ? p.zPadPlus : std::min(p.zPadMinus, p.zPadPlus);
    const int xPad = std::min(p.xPadMinus, p.xPadPlus);
    o.minPad = std::min(zPad, xPad);
    if (o.minPad >= PAD_MAX) throw Error(EIO_ERR_QC, "**** ERROR: Padding value is too high ****");
    if (o.minPad < 0) throw Error(EIO_ERR_ARG, "negative padding");
    if (p.blockSize != 16)
        throw Error(EIO_ERR_QC, "**** ERROR: Block size for time stepper is not consistent with parfile ****");
    if (p.fat != 4) throw Error(EIO_ERR_UNSUPPORTED, "fat must be 4 (8th-order stencil)");
    o.p = p;
    const int nz = p.nz, nx = p.nx, fat = p.fat;
    const long long n = (long long)nz * nx;
    // every cell of the medium enters the stencil: a NaN or Inf would spread through the wavefields (and
    // pass the velocity QC below, whose comparisons are false for NaN)
    {
        long long bad = LLONG_MAX;
#pragma omp parallel for reduction(min : bad) schedule(static)
        for (long long i = 0; i < 3 * n; i++)
            if (!std::isfinite(ep[i]) && i < bad) bad = i;
        if (bad != LLONG_MAX) {
            static const char* names[3] = {"rho", "lambda", "mu"};
            const long long k = bad % n;
            throw Error(EIO_ERR_ARG, std::string("non-finite elastic parameter ") + names[bad / n] + " at ix=" +
                                         std::to_string(k / nz) + ", iz=" + std::to_string(k % nz));
        }
    }
    // velocity range, fdParamElastic.cpp:80-97 (note the reference's 2*fat upper bound)
    float vmin = 10000.f, vmax = -1.f;
    for (int ix = fat; ix < nx - 2 * fat; ix++)
        for (int iz = fat; iz < nz - 2 * fat; iz++) {
            const long long i = (long long)ix * nz + iz;
            const float rho = ep[i], lam = ep[n + i], mu = ep[2 * n + i];
            const float vp = std::sqrt((lam + 2 * mu) / rho), vs = std::sqrt(mu / rho);
            if (vp < vmin) vmin = vp;
            if (vp > vmax) vmax = vp;
            if (vs < vmin && vs != 0) vmin = vs;
            if (vs > vmax) vmax = vs;
        }
    o.minVpVs = vmin;
    o.maxVpVs = vmax;
    // checkFdStability / checkFdDispersion / checkModelSize, fdParamElastic.cpp:256-297
    const float courant = vmax * o.dtw * 2.0f / std::min(p.dz, p.dx);
    if (courant > 0.45f)
        throw Error(EIO_ERR_QC, "**** ERROR: Courant is too big: " + fmt(courant) + " ****\nMax velocity value: " +
                                    fmt(vmax) + " [m/s]\nDtw: " + fmt(o.dtw) + " [s]\nMin (dz, dx): " +
                                    fmt(std::min(p.dz, p.dx)) + " [m]");
    const float disp = vmin / (p.fMax * std::max(p.dz, p.dx));
    if (disp < 3.0f)
        throw Error(EIO_ERR_QC, "**** ERROR: Dispersion is too small: " + fmt(disp) + " > 3 ****\nMin velocity value = " +
                                    fmt(vmin) + " [m/s]\nMax (dz, dx) = " + fmt(std::max(p.dz, p.dx)) +
                                    " [m]\nMax frequency = " + fmt(p.fMax) + " [Hz]");
    if ((nz - 2 * fat) % p.blockSize != 0)
        throw Error(EIO_ERR_QC, "**** ERROR: nz-2*_fat not a multiple of block size ****");
    if ((nx - 2 * fat) % p.blockSize != 0)
        throw Error(EIO_ERR_QC, "**** ERROR: nx-2*_fat not a multiple of block size ****");

    // scaled staggered medium, fdParamElastic.cpp:116-148
    for (int f = 0; f < 5; f++) o.par[f].assign(n, 0.f);
    std::vector<float> rho(ep, ep + n), mu(ep + 2 * n, ep + 3 * n), tmp(n);
    stagger_x(1, 0, nz, nx, o.par[0].data(), rho.data());
    stagger_z(1, 0, nz, nx, o.par[1].data(), rho.data());
    stagger_x(1, 0, nz, nx, tmp.data(), mu.data());
    stagger_z(1, 0, nz, nx, o.par[4].data(), tmp.data());
    const float dtw = o.dtw;
    for (long long i = 0; i < n; i++) {
        const float lam = ep[n + i], m = ep[2 * n + i];
        o.par[0][i] = (float)(2.0 * dtw / o.par[0][i]);
        o.par[1][i] = (float)(2.0 * dtw / o.par[1][i]);
        o.par[2][i] = (float)(2.0 * dtw * (lam + 2 * m));
        o.par[3][i] = (float)(2.0 * dtw * lam);
        o.par[4][i] = (float)(2.0 * dtw * o.par[4][i]);
    }
    // free surface: sigmaxx on the surface row z = 2*fat is driven by
    // lamb2MuDtw - lambDtw^2 / lamb2MuDtw (K:716-717, same float operations)
    o.fsc.assign(nx, 0.f);
    if (p.surfaceCondition)
        for (int ix = 0; ix < nx; ix++) {
            const long long i = (long long)ix * nz + 2 * fat;
            o.fsc[ix] = o.par[2][i] - (o.par[3][i] * o.par[3][i] / o.par[2][i]);
        }
    // FD coefficients, time filter and taper, nonlinearPropElasticGpuFunctions.cu:155-202
    static const double C[4] = {1.196289062541883, -0.079752604188901, 0.009570312506634, -6.975446437140719e-04};
    for (int k = 0; k < 4; k++) { o.zc[k] = (float)(C[k] / p.dz); o.xc[k] = (float)(C[k] / p.dx); }
    const int h = o.S + 1;
    o.filt.assign(2 * h, 0.f);
    const float sc = std::sqrt(float(o.ntw) / float(p.nts));
    for (int i = 0; i < h; i++) {
        const float a = (float)(1.0 - 1.0 * i / o.S);
        const float b = (float)(1.0 - a);
        o.filt[i] = (float)(a * (1.0 / sc));
        o.filt[i + h] = (float)(b * (1.0 / sc));
    }
    o.damp.assign(std::max(o.minPad, 1), 1.f);
    for (int i = 0; i < o.minPad; i++) {
        float arg = (float)(M_PI / (1.0 * o.minPad) * 1.0 * (o.minPad - i));
        arg = (float)(p.alphaCos + (1.0 - p.alphaCos) * std::cos(arg));
        o.damp[i] = arg;
    }
    o.dts_inv = (float)(1.0 / (2.0 * p.dts));
}

// ------------------------------------------------------------------ time interp
void time_interp(int adj, int add, int nts, float dts, float ots, int S, int nDev, float* coarse, float* fine) {
    const int ntw = (nts - 1) * S + 1;
    const float dtw = dts / S, otw = ots;
    float scale = float(ntw) / float(nts);
    scale = (float)(1.0 / std::sqrt(scale));
    if (!adj) {
        if (!add) std::fill(fine, fine + (long long)nDev * ntw, 0.f);
        for (int d = 0; d < nDev; d++) {
            const float* m = coarse + (long long)d * nts;
            float* f = fine + (long long)d * ntw;
            for (int itw = 0; itw < ntw - 1; itw++) {
                const float tw = otw + itw * dtw;
                float w = (tw - ots) / dts;
                const int i0 = (int)w;
                w = w - i0;
                f[itw] = (float)(f[itw] + (m[i0] * (1.0 - w) + m[i0 + 1] * w) * scale);
            }
            f[ntw - 1] += scale * m[nts - 1];
        }
    } else {
        if (!add) std::fill(coarse, coarse + (long long)nDev * nts, 0.f);
        for (int d = 0; d < nDev; d++) {
            float* m = coarse + (long long)d * nts;
            const float* f = fine + (long long)d * ntw;
            for (int itw = 0; itw < ntw - 1; itw++) {
                const float tw = otw + itw * dtw;
                float w = (tw - ots) / dts;
                const int i0 = (int)w;
                w = w - i0;
                m[i0] = (float)(m[i0] + scale * f[itw] * (1.0 - w));
                m[i0 + 1] += scale * f[itw] * w;
            }
            m[nts - 1] += scale * f[ntw - 1];
        }
    }
}

// ------------------------------------------------------------------ spatial interp
static double sinc_pi(double x) {
    // published Boost.Math sinc_pi algorithm: Taylor expansion near zero
    const double eps = 2.220446049250313e-16, t2 = std::sqrt(eps), tn = std::sqrt(t2);
    const double ax = std::fabs(x);
    if (ax >= tn) return std::sin(x) / x;
    double r = 1.0;
    if (ax >= eps) {
        const double x2 = x * x;
        r -= x2 / 6.0;
        if (ax >= t2) r += (x2 * x2) / 120.0;
    }
    return r;
}
static double normal_pdf(double mean, double sd, double x) {
    const double z = (x - mean) / sd;
    return std::exp(-0.5 * z * z) / (sd * std::sqrt(2.0 * M_PI));
}

void build_sinterp(const float* zc, const float* xc, int nDev, int nz, float oz, float dz, int nx, float ox,
                   float dx, int nt, const std::string& method, int nFilt, int dipole, float zDip, float xDip,
                   SInterp& s) {
    int m;
    if (method == "linear") { m = 0; nFilt = 1; }
    else if (method == "sinc") m = 1;
    else if (method == "gauss") m = 2;
    else throw Error(EIO_ERR_ARG, "**** ERROR: Space interp method not defined ****");
    if (nFilt < 1) throw Error(EIO_ERR_ARG, "nFilt must be >= 1");
    if (m != 0 && dipole == 1)
        throw Error(EIO_ERR_ARG, m == 1 ? "**** ERROR: Spatial sinc interpolation and dipole acquisition not implemented ****"
                                         : "**** ERROR: Gaussian spatial interpolation and dipole acquisition not implemented ****");
    if (nDev < 0 || nt < 1) throw Error(EIO_ERR_ARG, "invalid device count or nt");
    const int n2 = 2 * nFilt;
    const int nft = (m == 0) ? (dipole == 1 ? 8 : 4) : n2 * n2;
    // checkOutOfBounds, spaceInterpGpu.cpp:364-388
    const float zMax = oz + (nz - 1) * dz, xMax = ox + (nx - 1) * dx;
    const float zBuf = dz * nFilt, xBuf = dx * nFilt;
    for (int i = 0; i < nDev; i++) {
        if (zc[i] >= zMax - zBuf || zc[i] <= oz + zBuf)
            throw Error(EIO_ERR_BOUNDS, "**** ERROR: One of the device is out of bounds in the z direction ****");
        if (xc[i] >= xMax - xBuf || xc[i] <= ox + xBuf)
            throw Error(EIO_ERR_BOUNDS, "**** ERROR: One of the device is out of bounds in the x direction ****");
    }
    s.nIrreg = nDev; s.nft = nft; s.nt = nt; s.nz = nz; s.nx = nx;
    s.gpi.assign((size_t)nDev * nft, 0);
    s.w.assign((size_t)nDev * nft, 0.f);
    const float zDS = zDip * dz, xDS = xDip * dx;
    for (int d = 0; d < nDev; d++) {
        int* g = s.gpi.data() + (size_t)d * nft;
        float* w = s.w.data() + (size_t)d * nft;
        if (m == 0) {
            float wz = (zc[d] - oz) / dz, wx = (xc[d] - ox) / dx;
            const int zr = (int)wz; wz = wz - zr; wz = (float)(1.0 - wz);
            const int xr = (int)wx; wx = wx - xr; wx = (float)(1.0 - wx);
            g[0] = xr * nz + zr;      w[0] = wz * wx;
            g[1] = g[0] + 1;          w[1] = (float)((1.0 - wz) * wx);
            g[2] = g[0] + nz;         w[2] = (float)(wz * (1.0 - wx));
            g[3] = g[0] + nz + 1;     w[3] = (float)((1.0 - wz) * (1.0 - wx));
            if (dipole == 1) {
                float a = (zc[d] + zDS - oz) / dz, b = (xc[d] + xDS - ox) / dx;
                const int za = (int)a; a = a - za; a = (float)(1.0 - a);
                const int xb = (int)b; b = b - xb; b = (float)(1.0 - b);
                g[4] = xb * nz + za;      w[4] = (float)((-1.0) * a * b);
                g[5] = g[4] + 1;          w[5] = (float)((-1.0) * (1.0 - a) * b);
                g[6] = g[4] + nz;         w[6] = (float)((-1.0) * a * (1.0 - b));
                g[7] = g[4] + nz + 1;     w[7] = (float)((-1.0) * (1.0 - a) * (1.0 - b));
            }
        } else {
            const float zi = zc[d], xi = xc[d];
            const int zr = (int)((zi - oz) / dz), xr = (int)((xi - ox) / dx);
            float sum = 0.f;
            for (int ix = 0; ix < n2; ix++)
                for (int iz = 0; iz < n2; iz++) {
                    const float xcur = (xr + ix - nFilt + 1) * dx + ox;
                    const float zcur = (zr + iz - nFilt + 1) * dz + oz;
                    const float xin = (xi - xcur) / dx, zin = (zi - zcur) / dz;
                    const float v = (m == 1) ? (float)(sinc_pi(M_PI * zin) * sinc_pi(M_PI * xin))
                                             : (float)(normal_pdf(xi, 2 * dx, xcur) * normal_pdf(zi, 2 * dz, zcur));
                    w[n2 * ix + iz] = v;
                    g[n2 * ix + iz] = nz * (xr + ix - nFilt + 1) + (zr + iz - nFilt + 1);
                    sum += v;
                }
            for (int i = 0; i < nft; i++) w[i] = w[i] / sum;
        }
    }
    // convertIrregToReg: unique grid points in first-seen order, spaceInterpGpu.cpp:288-311
    std::unordered_map<int, int> idx;
    s.slot.assign(s.gpi.size(), 0);
    s.uniq.clear();
    for (size_t i = 0; i < s.gpi.size(); i++) {
        auto it = idx.find(s.gpi[i]);
        if (it == idx.end()) {
            idx.emplace(s.gpi[i], (int)s.uniq.size());
            s.slot[i] = (int)s.uniq.size();
            s.uniq.push_back(s.gpi[i]);
        } else {
            s.slot[i] = it->second;
        }
    }
    s.nReg = (int)s.uniq.size();
}

void sinterp_forward(const SInterp& s, bool add, const float* reg, float* irreg) {
    const int nt = s.nt;
    if (!add) std::fill(irreg, irreg + (size_t)s.nIrreg * nt, 0.f);
    for (int d = 0; d < s.nIrreg; d++)
        for (int f = 0; f < s.nft; f++) {
            const size_t i1 = (size_t)d * s.nft + f;
            const float w = s.w[i1];
            const float* m = reg + (size_t)s.slot[i1] * nt;
            float* o = irreg + (size_t)d * nt;
            for (int t = 0; t < nt; t++) o[t] += w * m[t];
        }
}

void sinterp_adjoint(const SInterp& s, bool add, float* reg, const float* irreg) {
    const int nt = s.nt;
    if (!add) std::fill(reg, reg + (size_t)s.nReg * nt, 0.f);
    for (int d = 0; d < s.nIrreg; d++)
        for (int f = 0; f < s.nft; f++) {
            const size_t i1 = (size_t)d * s.nft + f;
            const float w = s.w[i1];
            float* m = reg + (size_t)s.slot[i1] * nt;
            const float* o = irreg + (size_t)d * nt;
            for (int t = 0; t < nt; t++) m[t] += w * o[t];
        }
}

}  // namespace eio

// ====================================================================== C ABI
using namespace eio;

struct eio_sinterp {
    SInterp s;
};

struct eio_ctx {
    FdParam fd;
    Engine* eng = nullptr;
    int device = 0;
    // per-shot windows of the multi-shot operators (eio_ctx_set_shot_windows); empty: whole grid
    std::vector<int> win_ix0, win_nx;
    // shot lanes: further engines (own streams and buffers) on the same device that
    // run shots of a multi-shot call concurrently with eng (eio_ctx_set_lanes)
    std::vector<Engine*> extra;
    int lanes = 2;
    int batch = STEP_BATCH;   // nonlinear operators: shots per lockstep launch (1 = lanes)
    int born_batch = 1;       // Born operators: shots per lockstep group (1 = lanes, measured faster)
    std::vector<std::vector<float>> lane_tmp;   // per-lane host staging of one shot's data (kept across calls)
    int hist_where = 0;       // source-history location policy of every lane (eio_ctx_set_history_location)
    int check_finite = 0;     // scan host inputs and outputs of each call for NaN / Inf (eio_ctx_set_check_finite)
};

// lane k's staging buffer of at least n floats (contents undefined)
static float* lane_staging(eio_ctx* c, int k, size_t n) {
    if ((int)c->lane_tmp.size() <= k) c->lane_tmp.resize(k + 1);
    if (c->lane_tmp[k].size() < n) c->lane_tmp[k].resize(n);
    return c->lane_tmp[k].data();
}

static Engine* lane_engine(eio_ctx* c, int k) { return k == 0 ? c->eng : c->extra[k - 1]; }

// Lanes for a call over nShots shots, each lane needing about lane_bytes of
// device memory for the call: at most c->lanes and nShots, fewer when the free
// memory would not hold what the lanes still have to allocate (a new lane all
// of it; an existing one its Born history, which is allocated at first use).
// New lanes take the first lane's kernel choice (tuned first), checkpoint
// precision and graph setting.
static int ensure_lanes(eio_ctx* c, int nShots, size_t lane_bytes, int want = 0) {
    int n = std::max(1, std::min(want > 0 ? want : c->lanes, nShots));
    const int have = 1 + (int)c->extra.size();
    if (n > 1) {
        size_t fr = 0, tot = 0;
        if (cudaSetDevice(c->device) == cudaSuccess && cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
            auto need = [&](int lanes) {
                size_t b = 0;
                for (int k = 0; k < lanes; k++) {
                    const size_t held = k < have ? engine_history_bytes(lane_engine(c, k)) : 0;
                    const size_t want = k < have ? (lane_bytes > held ? lane_bytes - held : 0) : lane_bytes;
                    b += want + want / 5;
                }
                return b + ((size_t)256 << 20);
            };
            while (n > 1 && need(n) > fr) n--;
        } else {
            n = std::min(n, have);
        }
    }
    if (n > 1 && !engine_is_tuned(c->eng)) engine_autotune(c->eng);
    while ((int)c->extra.size() < n - 1) {
        Engine* e = engine_create(c->device, c->fd);
        try {
            int kind, tz, cw, cpr;
            engine_get_kernel(c->eng, &kind, &tz, &cw, &cpr);
            engine_set_kernel(e, kind, tz, cw, cpr);
            engine_set_checkpoint(e, engine_get_checkpoint(c->eng));
            engine_set_graphs(e, engine_get_graphs(c->eng));
            engine_set_wait_limit(e, engine_get_wait_limit(c->eng));
            engine_set_persistent(e, engine_get_persistent(c->eng));
            engine_set_history_where(e, c->hist_where);
            engine_share_medium(e, c->eng);   // one copy of the medium for every lane (L2)
        } catch (...) {
            engine_destroy(e);
            throw;
        }
        c->extra.push_back(e);
    }
    return n;
}

// Shots 0..nShots-1 over n lanes: lane k takes shots k, k + n, ... in order, on
// its own host thread; the first error is rethrown after every lane stopped.
template <class F>
static void run_lanes(eio_ctx* c, int n, int nShots, F&& f) {
    if (n <= 1) {
        for (int s = 0; s < nShots; s++) f(0, c->eng, s);
        return;
    }
    std::vector<std::exception_ptr> err(n);
    std::vector<std::thread> th;
    th.reserve(n);
    for (int k = 0; k < n; k++)
        th.emplace_back([&, k] {
            try {
                for (int s = k; s < nShots; s += n) f(k, lane_engine(c, k), s);
            } catch (...) {
                err[k] = std::current_exception();
            }
        });
    for (auto& t : th) t.join();
    for (auto& x : err)
        if (x) std::rethrow_exception(x);
}

// Born shots in lockstep groups (engine_born_shots_batch / engine_born_batch_dev):
// each shot of a group runs on a lane of its own (its buffers and its own
// history), so the group is as wide as the shot batch setting, the lane count
// and the free memory allow; 0 when the shots run on the lanes instead (a
// single shot or lane, a 16-bit history, sub > 1, or a shot batch of 1).
static size_t lane_bytes(const eio_ctx* c, bool born);
static int born_batch_width(eio_ctx* c, int nShots) {
    const int want = std::min(std::min(c->born_batch, c->lanes), (int)STEP_BATCH);
    if (want < 2 || nShots < 2 || !engine_batchable(c->eng)) return 0;
    const int nb = ensure_lanes(c, nShots, lane_bytes(c, true), want);
    return nb >= 2 ? nb : 0;
}

// consecutive groups of at most nb shots with sizes as even as possible: (first shot, count)
static std::vector<std::pair<int, int>> shot_groups(int nShots, int nb) {
    const int ng = (nShots + nb - 1) / nb;
    std::vector<std::pair<int, int>> out;
    for (int k = 0, s = 0; k < ng; k++) {
        const int n = nShots / ng + (k < nShots % ng ? 1 : 0);
        out.emplace_back(s, n);
        s += n;
    }
    return out;
}

// device bytes a lane needs for a shot: wavefield levels, secondary sources and, for Born, the history
// (with shot windows set, of the widest window: a lane's buffers grow to the largest shot it runs)
static size_t lane_bytes(const eio_ctx* c, bool born) {
    int nx = c->fd.p.nx;
    if (!c->win_nx.empty()) nx = *std::max_element(c->win_nx.begin(), c->win_nx.end());
    const size_t n = (size_t)c->fd.p.nz * nx;
    size_t b = sizeof(float) * n * 40;
    if (born) b += (size_t)2 * c->fd.p.nts * n * (engine_get_checkpoint(c->eng) ? 2 : 4);
    return b;
}

template <class F>
static int guarded(F&& f) {
    try {
        f();
        return EIO_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return EIO_ERR_NOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return EIO_ERR_ARG;
    }
}

static const int kFG[5] = {1, 2, 0, 0, 3};   // field -> grid (x, z, center, center, xz)

EIO_API void eio_fd_params_default(eio_fd_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->fMax = 1000.f;
    p->blockSize = 16;
    p->fat = 4;
    p->alphaCos = 0.99f;
    p->surfaceCondition = 0;
    p->mod_par = 1;
    p->errorTolerance = 1e-6f;
}

EIO_API const char* eio_last_error(void) { return g_last_error.c_str(); }
EIO_API int eio_version(void) { return 1; }

EIO_API int eio_sinterp_create(const float* zCoord, const float* xCoord, int nDevice, int nz, float oz, float dz,
                               int nx, float ox, float dx, int nt, const char* method, int nFilt, int dipole,
                               float zDipoleShift, float xDipoleShift, eio_sinterp** out) {
    return guarded([&] {
        if (!out || !method || (nDevice > 0 && (!zCoord || !xCoord))) throw Error(EIO_ERR_ARG, "null argument");
        auto s = std::make_unique<eio_sinterp>();
        build_sinterp(zCoord, xCoord, nDevice, nz, oz, dz, nx, ox, dx, nt, method, nFilt, dipole, zDipoleShift,
                      xDipoleShift, s->s);
        *out = s.release();
    });
}
EIO_API void eio_sinterp_destroy(eio_sinterp* s) { delete s; }
EIO_API int eio_sinterp_sizes(const eio_sinterp* s, int* nIrreg, int* nReg, int* nFiltTotal) {
    return guarded([&] {
        if (!s) throw Error(EIO_ERR_ARG, "null interpolator");
        if (nIrreg) *nIrreg = s->s.nIrreg;
        if (nReg) *nReg = s->s.nReg;
        if (nFiltTotal) *nFiltTotal = s->s.nft;
    });
}
EIO_API int eio_sinterp_positions(const eio_sinterp* s, int* regPos) {
    return guarded([&] {
        if (!s || !regPos) throw Error(EIO_ERR_ARG, "null argument");
        std::copy(s->s.uniq.begin(), s->s.uniq.end(), regPos);
    });
}
EIO_API int eio_sinterp_weights(const eio_sinterp* s, int* gpi, float* w) {
    return guarded([&] {
        if (!s) throw Error(EIO_ERR_ARG, "null interpolator");
        if (gpi) std::copy(s->s.gpi.begin(), s->s.gpi.end(), gpi);
        if (w) std::copy(s->s.w.begin(), s->s.w.end(), w);
    });
}
EIO_API int eio_sinterp_forward(const eio_sinterp* s, int add, const float* reg, float* irreg) {
    return guarded([&] {
        if (!s || !reg || !irreg) throw Error(EIO_ERR_ARG, "null argument");
        sinterp_forward(s->s, add != 0, reg, irreg);
    });
}
EIO_API int eio_sinterp_adjoint(const eio_sinterp* s, int add, float* reg, const float* irreg) {
    return guarded([&] {
        if (!s || !reg || !irreg) throw Error(EIO_ERR_ARG, "null argument");
        sinterp_adjoint(s->s, add != 0, reg, irreg);
    });
}

EIO_API int eio_medium_prepare(const eio_fd_params* p, const float* ep, float* rx, float* rz, float* l2m, float* lam,
                               float* mu) {
    return guarded([&] {
        if (!p || !ep) throw Error(EIO_ERR_ARG, "null argument");
        FdParam fd;
        build_fdparam(*p, ep, fd);
        float* o[5] = {rx, rz, l2m, lam, mu};
        for (int f = 0; f < 5; f++)
            if (o[f]) std::copy(fd.par[f].begin(), fd.par[f].end(), o[f]);
    });
}

EIO_API int eio_stagger(int axis, int adj, int add, int nz, int nx, float* model, float* data) {
    return guarded([&] {
        if (!model || !data || nz < 2 || nx < 2) throw Error(EIO_ERR_ARG, "invalid stagger arguments");
        if (axis == 0) stagger_x(adj, add, nz, nx, model, data);
        else stagger_z(adj, add, nz, nx, model, data);
    });
}

EIO_API int eio_time_interp(int adj, int add, int nts, float dts, float ots, int S, int nDev, float* coarse,
                            float* fine) {
    return guarded([&] {
        if (!coarse || !fine || nts < 2 || S < 1) throw Error(EIO_ERR_ARG, "invalid time-interp arguments");
        time_interp(adj, add, nts, dts, ots, S, nDev, coarse, fine);
    });
}

EIO_API int eio_ctx_create(const eio_fd_params* p, const float* ep, int device, eio_ctx** out) {
    return guarded([&] {
        if (!p || !ep || !out) throw Error(EIO_ERR_ARG, "null argument");
        auto c = std::make_unique<eio_ctx>();
        build_fdparam(*p, ep, c->fd);
        c->device = device;
        c->eng = engine_create(device, c->fd);
        *out = c.release();
    });
}
EIO_API int eio_ctx_set_background(eio_ctx* c, const float* ep) {
    return guarded([&] {
        if (!c || !ep) throw Error(EIO_ERR_ARG, "null argument");
        FdParam fd;
        build_fdparam(c->fd.p, ep, fd);   // QC may throw; the context keeps its old medium then
        engine_set_medium(c->eng, fd);
        for (Engine* e : c->extra) engine_set_medium(e, fd);
        c->fd = std::move(fd);
    });
}
EIO_API void eio_ctx_destroy(eio_ctx* c) {
    if (!c) return;
    for (Engine* e : c->extra) engine_destroy(e);
    engine_destroy(c->eng);
    delete c;
}
EIO_API int eio_ctx_set_history_location(eio_ctx* c, int where) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        engine_set_history_where(c->eng, where);
        for (Engine* e : c->extra) engine_set_history_where(e, where);
        c->hist_where = where;
    });
}
EIO_API int eio_ctx_get_history_location(const eio_ctx* c, int* where) {
    return guarded([&] {
        if (!c || !where) throw Error(EIO_ERR_ARG, "null argument");
        *where = engine_history_where(c->eng);
    });
}
EIO_API int eio_ctx_set_check_finite(eio_ctx* c, int on) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        c->check_finite = on ? 1 : 0;
    });
}
EIO_API int eio_set_device_memory_cap(long long bytes) {
    return guarded([&] { set_device_memory_cap(bytes); });
}
EIO_API int eio_get_device_memory_used(long long* bytes) {
    return guarded([&] {
        if (!bytes) throw Error(EIO_ERR_ARG, "null result");
        *bytes = device_memory_used();
    });
}
EIO_API int eio_ctx_set_checkpoint_precision(eio_ctx* c, int mode) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        engine_set_checkpoint(c->eng, mode);
        for (Engine* e : c->extra) engine_set_checkpoint(e, mode);
    });
}
EIO_API int eio_ctx_get_medium(const eio_ctx* c, float* rx, float* rz, float* l2m, float* lam, float* mu) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        float* o[5] = {rx, rz, l2m, lam, mu};
        for (int f = 0; f < 5; f++)
            if (o[f]) std::copy(c->fd.par[f].begin(), c->fd.par[f].end(), o[f]);
    });
}
EIO_API int eio_ctx_counts(const eio_ctx* c, long long* fineSteps, long long* cells) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        if (fineSteps) *fineSteps = (long long)(c->fd.p.nts - 1) * c->fd.S;
        if (cells) *cells = (long long)(c->fd.p.nz - 8) * (c->fd.p.nx - 8);
    });
}
EIO_API void* eio_ctx_stream(eio_ctx* c) { return c ? engine_stream(c->eng) : nullptr; }
EIO_API int eio_ctx_set_kernel(eio_ctx* c, int kind, int tz, int cw, int cpr) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        engine_set_kernel(c->eng, kind, tz, cw, cpr);
        for (Engine* e : c->extra) engine_set_kernel(e, kind, tz, cw, cpr);
    });
}
EIO_API int eio_ctx_set_wait_limit(eio_ctx* c, long long polls) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        engine_set_wait_limit(c->eng, polls);
        for (Engine* e : c->extra) engine_set_wait_limit(e, polls);
    });
}
EIO_API int eio_ctx_set_persistent(eio_ctx* c, int mask) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        engine_set_persistent(c->eng, mask);
        for (Engine* e : c->extra) engine_set_persistent(e, mask);
    });
}
EIO_API int eio_ctx_get_persistent(const eio_ctx* c, int* mask) {
    return guarded([&] {
        if (!c || !mask) throw Error(EIO_ERR_ARG, "null context or output");
        *mask = engine_get_persistent(c->eng);
    });
}
EIO_API int eio_ctx_get_wait_limit(const eio_ctx* c, long long* polls) {
    return guarded([&] {
        if (!c || !polls) throw Error(EIO_ERR_ARG, "null context or output");
        *polls = engine_get_wait_limit(c->eng);
    });
}
EIO_API int eio_ctx_autotune(eio_ctx* c, int* kind, int* tz, int* cw, int* cpr) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        engine_autotune(c->eng);
        int k, t, w, r;
        engine_get_kernel(c->eng, &k, &t, &w, &r);
        for (Engine* e : c->extra) engine_set_kernel(e, k, t, w, r);
        engine_get_kernel(c->eng, kind, tz, cw, cpr);
    });
}
EIO_API int eio_ctx_get_kernel(const eio_ctx* c, int* kind, int* tz, int* cw, int* cpr) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        engine_get_kernel(c->eng, kind, tz, cw, cpr);
    });
}
EIO_API int eio_ctx_stats(eio_ctx* c, int enable, int reset, long long* launches, long long* stepLaunches,
                          double* stepMs) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        // summed over the lanes
        long long la = 0, sl = 0;
        double ms = 0.0;
        for (int k = 0; k <= (int)c->extra.size(); k++) {
            long long a = 0, b = 0;
            double m = 0.0;
            engine_stats(lane_engine(c, k), enable, reset, &a, &b, &m, nullptr, nullptr);
            la += a; sl += b; ms += m;
        }
        if (launches) *launches = la;
        if (stepLaunches) *stepLaunches = sl;
        if (stepMs) *stepMs = ms;
    });
}
EIO_API int eio_ctx_step_cells(const eio_ctx* c, long long* cells) {
    return guarded([&] {
        if (!c || !cells) throw Error(EIO_ERR_ARG, "null context or output");
        long long n = engine_step_cells(c->eng);
        for (Engine* e : c->extra) n += engine_step_cells(e);
        *cells = n;
    });
}
EIO_API int eio_reduce64(int device, int op, int dtype, const void* x, const void* y, long long n, int onDevice,
                         double* result) {
    return guarded([&] {
        if (!result) throw Error(EIO_ERR_ARG, "null result");
        *result = reduce64(device, op, dtype, x, y, n, onDevice != 0);
    });
}
EIO_API int eio_ctx_set_born_batch(eio_ctx* c, int shots) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        if (shots < 1 || shots > STEP_BATCH) throw Error(EIO_ERR_ARG, "Born shot batch must be 1 .. 8");
        c->born_batch = shots;
    });
}
EIO_API int eio_ctx_set_shot_batch(eio_ctx* c, int shots) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        if (shots < 1 || shots > STEP_BATCH) throw Error(EIO_ERR_ARG, "shot batch must be 1 .. 8");
        c->batch = shots;
    });
}
EIO_API int eio_ctx_set_lanes(eio_ctx* c, int lanes) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        if (lanes < 1 || lanes > 8) throw Error(EIO_ERR_ARG, "lanes must be 1 .. 8");
        c->lanes = lanes;
        while ((int)c->extra.size() > lanes - 1) {   // release the lanes beyond the new count
            engine_destroy(c->extra.back());
            c->extra.pop_back();
        }
    });
}
EIO_API int eio_ctx_get_lanes(const eio_ctx* c, int* lanes, int* active) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        if (lanes) *lanes = c->lanes;
        if (active) *active = 1 + (int)c->extra.size();
    });
}
static ShotGeom make_geom(const int* const srcPos[4], const int nSrc[4], const int* const recPos[4],
                          const int nRec[4]);
EIO_API int eio_born_shots_dev(eio_ctx* c, int adj, int nShots, float* const* srcDtw, float* const dm[5],
                               float* const* data, const int* const* srcPos, const int* nSrc,
                               const int* const* recPos, const int* nRec) {
    return guarded([&] {
        if (!c || !srcDtw || !dm || !data || !srcPos || !nSrc || !recPos || !nRec || nShots < 1)
            throw Error(EIO_ERR_ARG, "null argument");
        const int nb = born_batch_width(c, nShots);
        const int nl = nb ? nb : ensure_lanes(c, nShots, lane_bytes(c, true));
        std::vector<float*> lane_dm((size_t)5 * nl);
        for (int k = 0; k < nl; k++) {
            if (adj && k > 0) {   // the other lanes image into their own buffers, added below
                engine_dm_zero(lane_engine(c, k));
                engine_dm_ptrs(lane_engine(c, k), lane_dm.data() + 5 * k);
            } else {
                for (int f = 0; f < 5; f++) lane_dm[5 * k + f] = dm[f];
            }
        }
        if (nb) {   // groups of shots in lockstep: shot i of a group on lane i
            std::vector<Engine*> es(nb);
            for (int k = 0; k < nb; k++) es[k] = lane_engine(c, k);
            for (const auto& grp : shot_groups(nShots, nb)) {
                const int s0 = grp.first, n = grp.second;
                std::vector<ShotGeom> g(n);
                std::vector<float*> dmv((size_t)5 * n);
                for (int i = 0; i < n; i++) {
                    const size_t s = (size_t)(s0 + i);
                    g[i] = make_geom(srcPos + 4 * s, nSrc + 4 * s, recPos + 4 * s, nRec + 4 * s);
                    for (int f = 0; f < 5; f++) dmv[5 * i + f] = adj ? lane_dm[5 * i + f] : dm[f];
                }
                engine_born_batch_dev(es.data(), n, adj, srcDtw + 5 * (size_t)s0, dmv.data(), data + 5 * (size_t)s0,
                                      g.data());
            }
            if (adj)
                for (int k = 1; k < nl; k++) engine_dm_add(lane_engine(c, k), dm);
            return;
        }
        run_lanes(c, nl, nShots, [&](int k, Engine* eng, int s) {
            engine_born(eng, adj, srcDtw + 5 * (size_t)s, lane_dm.data() + 5 * k, data + 5 * (size_t)s,
                        make_geom(srcPos + 4 * (size_t)s, nSrc + 4 * (size_t)s, recPos + 4 * (size_t)s,
                                  nRec + 4 * (size_t)s));
        });
        if (adj)
            for (int k = 1; k < nl; k++) engine_dm_add(lane_engine(c, k), dm);
    });
}
EIO_API int eio_ctx_set_shot_windows(eio_ctx* c, int nShots, const int* ix0, const int* nxw) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        if (nShots < 0 || (nShots > 0 && (!ix0 || !nxw))) throw Error(EIO_ERR_ARG, "null window list");
        const int nx = c->fd.p.nx, fat = c->fd.p.fat;
        for (int i = 0; i < nShots; i++)
            if (ix0[i] < 0 || nxw[i] < 2 * fat + 16 || (nxw[i] - 2 * fat) % 16 || ix0[i] + nxw[i] > nx)
                throw Error(EIO_ERR_ARG, "shot window " + std::to_string(i) + " [" + std::to_string(ix0[i]) + ", " +
                                             std::to_string(ix0[i] + nxw[i]) +
                                             ") must lie in the grid and hold 2*fat + a multiple of 16 columns");
        c->win_ix0.assign(ix0, ix0 + nShots);
        c->win_nx.assign(nxw, nxw + nShots);
    });
}
EIO_API int eio_ctx_set_graphs(eio_ctx* c, int enable) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        engine_set_graphs(c->eng, enable);
        for (Engine* e : c->extra) engine_set_graphs(e, enable);
    });
}
EIO_API int eio_ctx_pair_stats(eio_ctx* c, long long* pairLaunches, double* pairMs) {
    return guarded([&] {
        if (!c) throw Error(EIO_ERR_ARG, "null context");
        long long pl = 0;
        double pm = 0.0;
        for (int k = 0; k <= (int)c->extra.size(); k++) {
            long long a = 0;
            double m = 0.0;
            engine_stats(lane_engine(c, k), -1, 0, nullptr, nullptr, nullptr, &a, &m);
            pl += a; pm += m;
        }
        if (pairLaunches) *pairLaunches = pl;
        if (pairMs) *pairMs = pm;
    });
}

static ShotGeom make_geom(const int* const srcPos[4], const int nSrc[4], const int* const recPos[4],
                          const int nRec[4]) {
    ShotGeom g;
    for (int k = 0; k < 4; k++) {
        g.srcPos[k] = srcPos[k]; g.nSrc[k] = nSrc[k];
        g.recPos[k] = recPos[k]; g.nRec[k] = nRec[k];
        if (nSrc[k] < 0 || nRec[k] < 0) throw Error(EIO_ERR_ARG, "negative point count");
    }
    return g;
}

EIO_API int eio_nl_fwd_reg(eio_ctx* c, float* const model[5], float* const data[5], const int* const srcPos[4],
                           const int nSrc[4], const int* const recPos[4], const int nRec[4]) {
    return guarded([&] { engine_nl_host(c->eng, 0, model, data, make_geom(srcPos, nSrc, recPos, nRec)); });
}
EIO_API int eio_nl_adj_reg(eio_ctx* c, float* const model[5], float* const data[5], const int* const srcPos[4],
                           const int nSrc[4], const int* const recPos[4], const int nRec[4]) {
    return guarded([&] { engine_nl_host(c->eng, 1, model, data, make_geom(srcPos, nSrc, recPos, nRec)); });
}
EIO_API int eio_born_fwd_reg(eio_ctx* c, float* const srcDtw[5], float* const dm[5], float* const data[5],
                             const int* const srcPos[4], const int nSrc[4], const int* const recPos[4],
                             const int nRec[4]) {
    return guarded([&] { engine_born_host(c->eng, 0, srcDtw, dm, data, make_geom(srcPos, nSrc, recPos, nRec)); });
}
EIO_API int eio_born_adj_reg(eio_ctx* c, float* const srcDtw[5], float* const dm[5], float* const data[5],
                             const int* const srcPos[4], const int nSrc[4], const int* const recPos[4],
                             const int nRec[4]) {
    return guarded([&] { engine_born_host(c->eng, 1, srcDtw, dm, data, make_geom(srcPos, nSrc, recPos, nRec)); });
}
EIO_API int eio_nl_fwd_reg_dev(eio_ctx* c, float* const model[5], float* const data[5], const int* const srcPos[4],
                               const int nSrc[4], const int* const recPos[4], const int nRec[4]) {
    return guarded([&] { engine_nl(c->eng, 0, model, data, make_geom(srcPos, nSrc, recPos, nRec)); });
}
EIO_API int eio_nl_adj_reg_dev(eio_ctx* c, float* const model[5], float* const data[5], const int* const srcPos[4],
                               const int nSrc[4], const int* const recPos[4], const int nRec[4]) {
    return guarded([&] { engine_nl(c->eng, 1, model, data, make_geom(srcPos, nSrc, recPos, nRec)); });
}
EIO_API int eio_born_fwd_reg_dev(eio_ctx* c, float* const srcDtw[5], float* const dm[5], float* const data[5],
                                 const int* const srcPos[4], const int nSrc[4], const int* const recPos[4],
                                 const int nRec[4]) {
    return guarded([&] { engine_born(c->eng, 0, srcDtw, dm, data, make_geom(srcPos, nSrc, recPos, nRec)); });
}
EIO_API int eio_born_adj_reg_dev(eio_ctx* c, float* const srcDtw[5], float* const dm[5], float* const data[5],
                                 const int* const srcPos[4], const int nSrc[4], const int* const recPos[4],
                                 const int nRec[4]) {
    return guarded([&] { engine_born(c->eng, 1, srcDtw, dm, data, make_geom(srcPos, nSrc, recPos, nRec)); });
}

// ------------------------------------------------------------ multi-shot operators
namespace {

struct ShotGrids {
    const SInterp* s[4];
    const SInterp* r[4];
};

ShotGrids shot_grids(eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom, int iExp) {
    ShotGrids g;
    const int ir = (nRecGeom == 1) ? 0 : iExp;
    for (int k = 0; k < 4; k++) {
        if (!src[4 * iExp + k] || !rec[4 * ir + k]) throw Error(EIO_ERR_ARG, "null interpolator in geometry list");
        g.s[k] = &src[4 * iExp + k]->s;
        g.r[k] = &rec[4 * ir + k]->s;
    }
    return g;
}

// per-shot source signals on the regular grid, scaled like
// nonlinearPropElasticGpu.cpp:119-144 (scale by 2*dtw or the staggered
// buoyancy at the injection point, then by 1/(dx*dz))
void scale_sources(const FdParam& fd, const ShotGrids& g, std::vector<float>* reg, int nt) {
    const float tdtw = 2.0f * fd.dtw;   // exact: power-of-two scaling of a float
    const float area = (float)(1.0 / (fd.p.dx * fd.p.dz));
    for (int f = 0; f < 5; f++) {
        const SInterp& s = *g.s[kFG[f]];
        for (int k = 0; k < s.nReg; k++) {
            float* v = reg[f].data() + (size_t)k * nt;
            const float sc = (f == 0) ? fd.par[0][s.uniq[k]] : (f == 1) ? fd.par[1][s.uniq[k]] : tdtw;
            for (int t = 0; t < nt; t++) v[t] = v[t] * sc;
        }
    }
    for (int f = 0; f < 5; f++)
        for (auto& v : reg[f]) v = v * area;
}

// adjoint order, nonlinearPropElasticGpu.cpp:425-452: area first, then 2*dtw / buoyancy
void scale_sources_adj(const FdParam& fd, const ShotGrids& g, std::vector<float>* reg, int nt) {
    const float tdtw = 2.0f * fd.dtw;
    const float area = (float)(1.0 / (fd.p.dx * fd.p.dz));
    for (int f = 0; f < 5; f++)
        for (auto& v : reg[f]) v = v * area;
    for (int f = 0; f < 5; f++) {
        const SInterp& s = *g.s[kFG[f]];
        for (int k = 0; k < s.nReg; k++) {
            float* v = reg[f].data() + (size_t)k * nt;
            const float sc = (f == 0) ? fd.par[0][s.uniq[k]] : (f == 1) ? fd.par[1][s.uniq[k]] : tdtw;
            for (int t = 0; t < nt; t++) v[t] = v[t] * sc;
        }
    }
}

ShotGeom reg_geom(const ShotGrids& g) {
    ShotGeom sg;
    for (int k = 0; k < 4; k++) {
        sg.srcPos[k] = g.s[k]->uniq.data(); sg.nSrc[k] = g.s[k]->nReg;
        sg.recPos[k] = g.r[k]->uniq.data(); sg.nRec[k] = g.r[k]->nReg;
    }
    return sg;
}

// Shot `shot` of a multi-shot call on its window (eio_ctx_set_shot_windows):
// the engine crops to columns [ix0, ix0 + nxw) and the regular positions shift
// by ix0 * nz.  Every device must lie in the window's updated interior.  The
// whole grid comes back when the guard goes.
struct ShotWindow {
    eio_ctx* c;
    Engine* eng;
    std::vector<int> pos[8];
    ShotGeom sg;
    ShotWindow(eio_ctx* ctx, Engine* lane, const ShotGrids& g, int shot, int nShots) : c(ctx), eng(lane) {
        sg = reg_geom(g);
        if (c->win_nx.empty()) return;
        if ((int)c->win_nx.size() != nShots)
            throw Error(EIO_ERR_ARG, "shot windows were set for " + std::to_string(c->win_nx.size()) + " shots, the call has " +
                                         std::to_string(nShots));
        const int ix0 = c->win_ix0[shot], nxw = c->win_nx[shot], nz = c->fd.p.nz, fat = c->fd.p.fat;
        const long long off = (long long)ix0 * nz;
        for (int k = 0; k < 8; k++) {
            const int* p = k < 4 ? sg.srcPos[k] : sg.recPos[k - 4];
            const int n = k < 4 ? sg.nSrc[k] : sg.nRec[k - 4];
            pos[k].resize(n);
            for (int i = 0; i < n; i++) {
                const int ix = p[i] / nz;
                if (ix < ix0 + fat || ix >= ix0 + nxw - fat)
                    throw Error(EIO_ERR_BOUNDS, "a device of shot " + std::to_string(shot) + " (column " +
                                                    std::to_string(ix) + ") lies outside the updated interior of its window");
                pos[k][i] = (int)(p[i] - off);
            }
            if (k < 4) sg.srcPos[k] = pos[k].data();
            else sg.recPos[k - 4] = pos[k].data();
        }
        engine_set_window(eng, ix0, nxw);
    }
    ~ShotWindow() {
        if (!c->win_nx.empty()) {
            try { engine_set_window(eng, 0, 0); } catch (...) {}
        }
    }
    ShotWindow(const ShotWindow&) = delete;
    ShotWindow& operator=(const ShotWindow&) = delete;
};

void check_nt(const ShotGrids& g, int nts) {
    for (int k = 0; k < 4; k++)
        if (g.s[k]->nt != nts || g.r[k]->nt != nts)
            throw Error(EIO_ERR_ARG, "**** ERROR: nts not consistent with parfile ****");
    for (int k = 1; k < 4; k++)
        if (g.s[k]->nIrreg != g.s[0]->nIrreg || g.r[k]->nIrreg != g.r[0]->nIrreg)
            throw Error(EIO_ERR_ARG, "the four staggered grids of a shot must hold the same devices");
}

// nonlinearPropElasticGpu::forward with add = false: irregular source -> data slice;
// wfld (host [nts][5][nx][nz]) receives the saved wavefield when not null
void nl_shot_forward(eio_ctx* c, Engine* eng, const ShotGrids& g, const ShotGeom& sg, const float* model,
                     float* data, float* wfld = nullptr) {
    const int nts = c->fd.p.nts;
    const int nsi = g.s[0]->nIrreg;
    std::vector<float> reg[5];
    float* mp[5];
    for (int f = 0; f < 5; f++) {
        const SInterp& s = *g.s[kFG[f]];
        reg[f].assign((size_t)s.nReg * nts, 0.f);
        sinterp_adjoint(s, false, reg[f].data(), model + (size_t)f * nsi * nts);
    }
    scale_sources(c->fd, g, reg, nts);
    for (int f = 0; f < 5; f++) mp[f] = reg[f].data();
    // receivers are interpolated to the devices on the GPU (same sums as sinterp_forward)
    engine_nl_shot(eng, 0, mp, sg, g.r, data, wfld);
}

// The adjoint wavefield is scaled like the adjoint sources
// (nonlinearPropElasticGpu.cpp:432-446): vx by rhoxDtw, vz by rhozDtw, the
// stresses by 2*dtw (in double, as the reference), all by 1/(dx*dz).
static void scale_adjoint_wavefield(const FdParam& fd, float* w) {
    const float area = (float)(1.0 / (fd.p.dx * fd.p.dz));
    const size_t n = (size_t)fd.p.nz * fd.p.nx;
    const double tdtw = 2.0 * (double)fd.dtw * (double)area;
#pragma omp parallel for schedule(static)
    for (int it = 0; it < fd.p.nts; it++) {
        float* slice = w + (size_t)it * 5 * n;
        for (size_t i = 0; i < n; i++) {
            slice[i] *= fd.par[0][i] * area;
            slice[n + i] *= fd.par[1][i] * area;
        }
        for (size_t i = 2 * n; i < 5 * n; i++) slice[i] = (float)((double)slice[i] * tdtw);
    }
}

// nonlinearPropElasticGpu::adjoint with add = true into model; wfld as for nl_shot_forward
void nl_shot_adjoint(eio_ctx* c, Engine* eng, const ShotGrids& g, const ShotGeom& sg, float* model,
                     const float* data, float* wfld = nullptr) {
    const int nts = c->fd.p.nts;
    const int nsi = g.s[0]->nIrreg;
    std::vector<float> reg[5];
    float* mp[5];
    for (int f = 0; f < 5; f++) {
        reg[f].assign((size_t)g.s[kFG[f]]->nReg * nts, 0.f);
        mp[f] = reg[f].data();
    }
    // the data are spread onto the regular grid on the GPU (same sums as sinterp_adjoint)
    engine_nl_shot(eng, 1, mp, sg, g.r, const_cast<float*>(data), wfld);
    if (wfld) scale_adjoint_wavefield(c->fd, wfld);
    scale_sources_adj(c->fd, g, reg, nts);
    for (int f = 0; f < 5; f++) sinterp_forward(*g.s[kFG[f]], true, reg[f].data(), model + (size_t)f * nsi * nts);
}

// Born setSources: irregular signal -> scaled regular fine-time source (seismicElasticOperator2D.cpp:27-117)
void born_sources(eio_ctx* c, const ShotGrids& g, const float* sig, std::vector<float>* fine) {
    const int nts = c->fd.p.nts, ntw = c->fd.ntw;
    const int nsi = g.s[0]->nIrreg;
    std::vector<float> reg[5];
    for (int f = 0; f < 5; f++) {
        const SInterp& s = *g.s[kFG[f]];
        reg[f].assign((size_t)s.nReg * nts, 0.f);
        sinterp_adjoint(s, false, reg[f].data(), sig + (size_t)f * nsi * nts);
    }
    scale_sources(c->fd, g, reg, nts);
    for (int f = 0; f < 5; f++) {
        const int nr = g.s[kFG[f]]->nReg;
        fine[f].assign((size_t)nr * ntw, 0.f);
        time_interp(0, 0, nts, c->fd.p.dts, c->fd.p.ots, c->fd.S, nr, reg[f].data(), fine[f].data());
    }
}

// (drho, dlambda, dmu) -> 5 staggered, scaled components (BornElasticShotsGpu.cpp:107-150)
void born_model_slice(const FdParam& fd, const float* model, std::vector<float>* sl) {
    const int nz = fd.p.nz, nx = fd.p.nx;
    const size_t n = (size_t)nz * nx;
    std::vector<float> tmp(model, model + n), tmp1(n);
    for (int f = 0; f < 5; f++) sl[f].assign(n, 0.f);
    stagger_x(1, 0, nz, nx, sl[0].data(), tmp.data());
    stagger_z(1, 0, nz, nx, sl[1].data(), tmp.data());
    std::copy(model + n, model + 2 * n, sl[2].begin());
    std::copy(model + 2 * n, model + 3 * n, sl[3].begin());
    std::copy(model + 2 * n, model + 3 * n, tmp.begin());
    stagger_x(1, 0, nz, nx, tmp1.data(), tmp.data());
    stagger_z(1, 0, nz, nx, sl[4].data(), tmp1.data());
    const double tdtw = 2.0 * fd.dtw;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; i++) {
        sl[0][i] *= fd.par[0][i];
        sl[1][i] *= fd.par[1][i];
        sl[2][i] = (float)(sl[2][i] * tdtw);
        sl[3][i] = (float)(sl[3][i] * tdtw);
        sl[4][i] = (float)(sl[4][i] * tdtw);
    }
}

}  // namespace

EIO_API int eio_born_prepare_sources(eio_ctx* c, const float* signal, eio_sinterp* const src[4], float* const out[5]) {
    return guarded([&] {
        if (!c || !signal || !src || !out) throw Error(EIO_ERR_ARG, "null argument");
        ShotGrids g;
        for (int k = 0; k < 4; k++) {
            if (!src[k]) throw Error(EIO_ERR_ARG, "null interpolator");
            g.s[k] = &src[k]->s;
            g.r[k] = &src[k]->s;
        }
        check_nt(g, c->fd.p.nts);
        std::vector<float> fine[5];
        born_sources(c, g, signal, fine);
        for (int f = 0; f < 5; f++) std::copy(fine[f].begin(), fine[f].end(), out[f]);
    });
}

EIO_API int eio_nl_prepare_sources(eio_ctx* c, const float* model, eio_sinterp* const src[4], float* const out[5]) {
    return guarded([&] {
        if (!c || !model || !src || !out) throw Error(EIO_ERR_ARG, "null argument");
        ShotGrids g;
        for (int k = 0; k < 4; k++) {
            if (!src[k]) throw Error(EIO_ERR_ARG, "null interpolator");
            g.s[k] = &src[k]->s;
            g.r[k] = &src[k]->s;
        }
        const int nts = c->fd.p.nts;
        check_nt(g, nts);
        const int nsi = g.s[0]->nIrreg;
        std::vector<float> reg[5];
        for (int f = 0; f < 5; f++) {
            const SInterp& s = *g.s[kFG[f]];
            reg[f].assign((size_t)s.nReg * nts, 0.f);
            sinterp_adjoint(s, false, reg[f].data(), model + (size_t)f * nsi * nts);
        }
        scale_sources(c->fd, g, reg, nts);
        for (int f = 0; f < 5; f++) std::copy(reg[f].begin(), reg[f].end(), out[f]);
    });
}

EIO_API int eio_born_prepare_model(eio_ctx* c, const float* model, float* const out[5]) {
    return guarded([&] {
        if (!c || !model || !out) throw Error(EIO_ERR_ARG, "null argument");
        std::vector<float> sl[5];
        born_model_slice(c->fd, model, sl);
        for (int f = 0; f < 5; f++) std::copy(sl[f].begin(), sl[f].end(), out[f]);
    });
}

// One group of up to c->batch shots for engine_nl_shots_batch: the engines
// (lanes 0..cnt-1) set to the shots' windows, their geometries, receiver
// interpolators and one regular source buffer per shot and field.
struct ShotGroup {
    int s0, cnt;
    std::vector<ShotGrids> gs;
    std::vector<std::unique_ptr<ShotWindow>> wins;
    std::vector<ShotGeom> geo;
    std::vector<std::vector<float>> reg;     // [cnt * 5]
    std::vector<float*> mp;                  // [cnt * 5] -> reg
    std::vector<float*> dp;                  // [cnt] irregular traces of each shot
    std::vector<const SInterp*> rp;          // [cnt * 4]
    std::vector<Engine*> eng;
    ShotGroup(eio_ctx* c, int first, int n, int nExp, eio_sinterp* const* src, eio_sinterp* const* rec,
              int nRecGeom)
        : s0(first), cnt(n), geo(n), reg((size_t)5 * n), mp((size_t)5 * n), dp(n), rp((size_t)4 * n), eng(n) {
        const int nts = c->fd.p.nts;
        for (int i = 0; i < cnt; i++) {
            eng[i] = lane_engine(c, i);
            gs.push_back(shot_grids(src, rec, nRecGeom, s0 + i));
        }
        for (int i = 0; i < cnt; i++) {
            const ShotGrids& g = gs[i];
            wins.emplace_back(new ShotWindow(c, eng[i], g, s0 + i, nExp));
            geo[i] = wins.back()->sg;
            for (int f = 0; f < 5; f++) {
                reg[(size_t)5 * i + f].assign((size_t)g.s[kFG[f]]->nReg * nts, 0.f);
                mp[(size_t)5 * i + f] = reg[(size_t)5 * i + f].data();
            }
            for (int k = 0; k < 4; k++) rp[(size_t)4 * i + k] = g.r[k];
        }
    }
    void run(int adj) { engine_nl_shots_batch(eng.data(), cnt, adj, mp.data(), geo.data(), rp.data(), dp.data()); }
};

// Nonlinear forward of every shot in groups of c->batch engines advanced in
// lockstep (engine_nl_shots_batch): one launch per fine step for the group.
static void nl_forward_batched(eio_ctx* c, int add, int nExp, int nModelExp, const float* model, float* data,
                               eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom, size_t dslice,
                               size_t mslice) {
    const int nts = c->fd.p.nts;
    const int nb = ensure_lanes(c, nExp, lane_bytes(c, false), std::min(c->batch, (int)STEP_BATCH));
    for (int s0 = 0; s0 < nExp; s0 += nb) {
        ShotGroup grp(c, s0, std::min(nb, nExp - s0), nExp, src, rec, nRecGeom);
        for (int i = 0; i < grp.cnt; i++) {
            const int e = s0 + i;
            const ShotGrids& g = grp.gs[i];
            const float* ms = model + (nModelExp == 1 ? 0 : (size_t)e * mslice);
            const int nsi = g.s[0]->nIrreg;
            for (int f = 0; f < 5; f++)
                sinterp_adjoint(*g.s[kFG[f]], false, grp.mp[(size_t)5 * i + f], ms + (size_t)f * nsi * nts);
            scale_sources(c->fd, g, &grp.reg[(size_t)5 * i], nts);
            grp.dp[i] = add ? lane_staging(c, i, dslice) : data + (size_t)e * dslice;
        }
        grp.run(0);
        if (add)
            for (int i = 0; i < grp.cnt; i++) {
                float* d = data + (size_t)(s0 + i) * dslice;
                const float* t = grp.dp[i];
#pragma omp parallel for schedule(static)
                for (long long j = 0; j < (long long)dslice; j++) d[j] += t[j];
            }
    }
}

static int nl_forward_impl(eio_ctx* c, int add, int nExp, int nModelExp, const float* model, float* data,
                           eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom, int wShot, float* wfld) {
    return guarded([&] {
        if (!c || !model || !data || !src || !rec || nExp < 1) throw Error(EIO_ERR_ARG, "null argument");
        if (nModelExp != 1 && nModelExp != nExp) throw Error(EIO_ERR_ARG, "model shot axis must be 1 or nExp");
        if (nRecGeom != 1 && nRecGeom != nExp) throw Error(EIO_ERR_ARG, "receiver geometry count must be 1 or nExp");
        const int nts = c->fd.p.nts;
        ShotGrids g0 = shot_grids(src, rec, nRecGeom, 0);
        const size_t dslice = (size_t)5 * g0.r[0]->nIrreg * nts;
        const size_t mslice = (size_t)5 * g0.s[0]->nIrreg * nts;
        for (int e = 0; e < nExp; e++) {
            ShotGrids g = shot_grids(src, rec, nRecGeom, e);
            check_nt(g, nts);
            if ((size_t)5 * g.s[0]->nIrreg * nts != mslice || (size_t)5 * g.r[0]->nIrreg * nts != dslice)
                throw Error(EIO_ERR_ARG, "device counts differ between shots");
        }
        if (c->batch > 1 && nExp > 1 && !(wShot >= 0 && wShot < nExp && wfld) && !c->fd.p.surfaceCondition) {
            nl_forward_batched(c, add, nExp, nModelExp, model, data, src, rec, nRecGeom, dslice, mslice);
            return;
        }
        const int nl = ensure_lanes(c, nExp, lane_bytes(c, false));
        std::vector<float*> tmp(nl);
        for (int k = 0; k < nl; k++) tmp[k] = add ? lane_staging(c, k, dslice) : nullptr;
        run_lanes(c, nl, nExp, [&](int k, Engine* eng, int e) {
            ShotGrids g = shot_grids(src, rec, nRecGeom, e);
            ShotWindow win(c, eng, g, e, nExp);
            float* d = data + (size_t)e * dslice;
            // add = false: straight into the shot's slice; add = true: staged, then added
            nl_shot_forward(c, eng, g, win.sg, model + (nModelExp == 1 ? 0 : (size_t)e * mslice), add ? tmp[k] : d,
                            e == wShot ? wfld : nullptr);
            if (add) {
                const float* t = tmp[k];
#pragma omp parallel for schedule(static)
                for (long long i = 0; i < (long long)dslice; i++) d[i] += t[i];
            }
        });
    });
}

// Nonlinear adjoint of every shot in groups of c->batch engines advanced in
// lockstep (engine_nl_shots_batch); each shot's source traces are scaled and
// interpolated as in nl_shot_adjoint and added to its model slice, shots in
// order (one stack over every shot for a constant source signal).
static void nl_adjoint_batched(eio_ctx* c, int nExp, int nModelExp, float* model, const float* data,
                               eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom, size_t dslice,
                               size_t mslice) {
    const int nts = c->fd.p.nts;
    const int nb = ensure_lanes(c, nExp, lane_bytes(c, false), std::min(c->batch, (int)STEP_BATCH));
    for (int s0 = 0; s0 < nExp; s0 += nb) {
        ShotGroup grp(c, s0, std::min(nb, nExp - s0), nExp, src, rec, nRecGeom);
        for (int i = 0; i < grp.cnt; i++) grp.dp[i] = const_cast<float*>(data) + (size_t)(s0 + i) * dslice;
        grp.run(1);
        for (int i = 0; i < grp.cnt; i++) {
            const int e = s0 + i;
            const ShotGrids& g = grp.gs[i];
            const int nsi = g.s[0]->nIrreg;
            scale_sources_adj(c->fd, g, &grp.reg[(size_t)5 * i], nts);
            float* m = model + (nModelExp == 1 ? 0 : (size_t)e * mslice);
            for (int f = 0; f < 5; f++)
                sinterp_forward(*g.s[kFG[f]], true, grp.mp[(size_t)5 * i + f], m + (size_t)f * nsi * nts);
        }
    }
}

static int nl_adjoint_impl(eio_ctx* c, int add, int nExp, int nModelExp, float* model, const float* data,
                           eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom, int wShot, float* wfld) {
    return guarded([&] {
        if (!c || !model || !data || !src || !rec || nExp < 1) throw Error(EIO_ERR_ARG, "null argument");
        if (nModelExp != 1 && nModelExp != nExp) throw Error(EIO_ERR_ARG, "model shot axis must be 1 or nExp");
        if (nRecGeom != 1 && nRecGeom != nExp) throw Error(EIO_ERR_ARG, "receiver geometry count must be 1 or nExp");
        const int nts = c->fd.p.nts;
        ShotGrids g0 = shot_grids(src, rec, nRecGeom, 0);
        const size_t dslice = (size_t)5 * g0.r[0]->nIrreg * nts;
        const size_t mslice = (size_t)5 * g0.s[0]->nIrreg * nts;
        if (!add) std::fill(model, model + mslice * nModelExp, 0.f);
        for (int e = 0; e < nExp; e++) {
            ShotGrids g = shot_grids(src, rec, nRecGeom, e);
            check_nt(g, nts);
            if ((size_t)5 * g.s[0]->nIrreg * nts != mslice || (size_t)5 * g.r[0]->nIrreg * nts != dslice)
                throw Error(EIO_ERR_ARG, "device counts differ between shots");
        }
        if (c->batch > 1 && nExp > 1 && !(wShot >= 0 && wShot < nExp && wfld) && !c->fd.p.surfaceCondition) {
            nl_adjoint_batched(c, nExp, nModelExp, model, data, src, rec, nRecGeom, dslice, mslice);
            return;
        }
        const int nl = ensure_lanes(c, nExp, lane_bytes(c, false));
        // constant source signal: every shot stacks into one model (nonlinearPropElasticShotsGpu.cpp:384-417),
        // here one partial stack per lane, added in lane order
        std::vector<std::vector<float>> slice(nl, std::vector<float>(mslice, 0.f));
        run_lanes(c, nl, nExp, [&](int k, Engine* eng, int e) {
            ShotGrids g = shot_grids(src, rec, nRecGeom, e);
            ShotWindow win(c, eng, g, e, nExp);
            if (nModelExp == 1) {
                nl_shot_adjoint(c, eng, g, win.sg, slice[k].data(), data + (size_t)e * dslice,
                                e == wShot ? wfld : nullptr);
            } else {
                std::fill(slice[k].begin(), slice[k].end(), 0.f);
                nl_shot_adjoint(c, eng, g, win.sg, slice[k].data(), data + (size_t)e * dslice,
                                e == wShot ? wfld : nullptr);
                float* m = model + (size_t)e * mslice;
                const float* sk = slice[k].data();
#pragma omp parallel for schedule(static)
                for (long long i = 0; i < (long long)mslice; i++) m[i] += sk[i];
            }
        });
        if (nModelExp == 1)
            for (int k = 0; k < nl; k++) {
                const float* sk = slice[k].data();
#pragma omp parallel for schedule(static)
                for (long long i = 0; i < (long long)mslice; i++) model[i] += sk[i];
            }
    });
}

// ---- optional NaN / Inf scans of a call's host inputs and outputs (eio_ctx_set_check_finite)
struct FSpan {
    const float* p;
    size_t n;
    const char* what;
};
static void require_finite(const FSpan& s, int code, const char* side) {
    if (!s.p) return;
    long long bad = LLONG_MAX;
#pragma omp parallel for reduction(min : bad) schedule(static)
    for (long long i = 0; i < (long long)s.n; i++)
        if (!std::isfinite(s.p[i]) && i < bad) bad = i;
    if (bad != LLONG_MAX)
        throw Error(code, std::string("non-finite value in the ") + side + " " + s.what + " at element " +
                              std::to_string(bad) + (code == EIO_ERR_NONFINITE ? " (unstable propagation?)" : ""));
}
// inputs rejected with EIO_ERR_ARG before the call; outputs with EIO_ERR_NONFINITE after it
template <class In, class Call, class Out>
static int finite_call(eio_ctx* c, In inputs, Call call, Out outputs) {
    if (c && c->check_finite) {
        const int rc = guarded([&] {
            for (const FSpan& f : inputs()) require_finite(f, EIO_ERR_ARG, "input");
        });
        if (rc != EIO_OK) return rc;
    }
    int rc = call();
    if (rc == EIO_OK && c && c->check_finite)
        rc = guarded([&] {
            for (const FSpan& f : outputs()) require_finite(f, EIO_ERR_NONFINITE, "output");
        });
    return rc;
}
// elements of a multi-shot call's data (nExp shots of 5 x receivers x nts) and source-model arrays
static size_t data_elems(eio_ctx* c, eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom, int nExp) {
    ShotGrids g = shot_grids(src, rec, nRecGeom, 0);
    return (size_t)nExp * 5 * g.r[0]->nIrreg * c->fd.p.nts;
}
static size_t src_elems(eio_ctx* c, eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom, int nModelExp) {
    ShotGrids g = shot_grids(src, rec, nRecGeom, 0);
    return (size_t)nModelExp * 5 * g.s[0]->nIrreg * c->fd.p.nts;
}

EIO_API int eio_nl_forward(eio_ctx* c, int add, int nExp, int nModelExp, const float* model, float* data,
                           eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom) {
    return finite_call(
        c, [&] { return std::vector<FSpan>{{model, src_elems(c, src, rec, nRecGeom, nModelExp), "source traces"}}; },
        [&] { return nl_forward_impl(c, add, nExp, nModelExp, model, data, src, rec, nRecGeom, -1, nullptr); },
        [&] { return std::vector<FSpan>{{data, data_elems(c, src, rec, nRecGeom, nExp), "data"}}; });
}

EIO_API int eio_nl_adjoint(eio_ctx* c, int add, int nExp, int nModelExp, float* model, const float* data,
                           eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom) {
    return finite_call(
        c, [&] { return std::vector<FSpan>{{data, data_elems(c, src, rec, nRecGeom, nExp), "data"}}; },
        [&] { return nl_adjoint_impl(c, add, nExp, nModelExp, model, data, src, rec, nRecGeom, -1, nullptr); },
        [&] { return std::vector<FSpan>{{model, src_elems(c, src, rec, nRecGeom, nModelExp), "source traces"}}; });
}

static void check_wavefield_shot(int nExp, int wShot, const float* wfld) {
    if (wShot >= nExp) throw Error(EIO_ERR_ARG, "wavefield shot number beyond the number of shots");
    if (wShot >= 0 && !wfld) throw Error(EIO_ERR_ARG, "null wavefield buffer");
}

EIO_API int eio_nl_forward_wavefield(eio_ctx* c, int add, int nExp, int nModelExp, const float* model, float* data,
                                     eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom, int wShot,
                                     float* wfld) {
    const int st = guarded([&] { check_wavefield_shot(nExp, wShot, wfld); });
    if (st) return st;
    return nl_forward_impl(c, add, nExp, nModelExp, model, data, src, rec, nRecGeom, wShot, wfld);
}

EIO_API int eio_nl_adjoint_wavefield(eio_ctx* c, int add, int nExp, int nModelExp, float* model, const float* data,
                                     eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom, int wShot,
                                     float* wfld) {
    const int st = guarded([&] { check_wavefield_shot(nExp, wShot, wfld); });
    if (st) return st;
    return nl_adjoint_impl(c, add, nExp, nModelExp, model, data, src, rec, nRecGeom, wShot, wfld);
}

// One group of Born shots in lockstep through the operator path: shot s0 + i
// runs on lane i (its window, fine-time sources from the host preparation,
// receivers interpolated on the GPU).  Forward: every shot reads the first
// lane's perturbation at its window; adjoint: shot i images into lane i's
// own buffers (summed by image_to_model).  dataIrreg: per shot host traces.
static void born_group(eio_ctx* c, int adj, int s0, int n, int nExp, eio_sinterp* const* src,
                       eio_sinterp* const* rec, int nRecGeom, const float* const* sigs, int nSignals,
                       float* const* dataIrreg) {
    std::vector<Engine*> es(n);
    std::vector<std::vector<float>> fine((size_t)5 * n);
    std::vector<float*> sp((size_t)5 * n), dmv((size_t)5 * n);
    std::vector<std::unique_ptr<ShotWindow>> wins;
    std::vector<ShotGeom> g(n);
    std::vector<const SInterp*> recs((size_t)4 * n);
    float* base0[5];
    engine_dm_ptrs(lane_engine(c, 0), base0);
    for (int i = 0; i < n; i++) {
        const int e = s0 + i;
        es[i] = lane_engine(c, i);
        ShotGrids gg = shot_grids(src, rec, nRecGeom, e);
        std::vector<float> f5[5];
        born_sources(c, gg, sigs[nSignals == 1 ? 0 : e], f5);
        for (int f = 0; f < 5; f++) {
            fine[5 * i + f] = std::move(f5[f]);
            sp[5 * i + f] = fine[5 * i + f].data();
        }
        wins.emplace_back(new ShotWindow(c, es[i], gg, e, nExp));
        g[i] = wins.back()->sg;
        for (int k = 0; k < 4; k++) recs[4 * i + k] = gg.r[k];
        if (adj) {
            engine_dm_window(es[i], dmv.data() + 5 * i);
        } else {
            const long long off = c->win_nx.empty() ? 0 : (long long)c->win_ix0[e] * c->fd.p.nz;
            for (int f = 0; f < 5; f++) dmv[5 * i + f] = base0[f] + off;
        }
    }
    engine_born_shots_batch(es.data(), n, adj, sp.data(), dmv.data(), g.data(), recs.data(), dataIrreg);
}

static int eio_born_forward_impl(eio_ctx* c, int add, int nExp, const float* model, float* data,
                             const float* const* sigs, int nSignals, eio_sinterp* const* src, eio_sinterp* const* rec,
                             int nRecGeom) {
    return guarded([&] {
        if (!c || !model || !data || !src || !rec || !sigs || nExp < 1) throw Error(EIO_ERR_ARG, "null argument");
        if (nSignals != 1 && nSignals != nExp) throw Error(EIO_ERR_ARG, "source signal count must be 1 or nExp");
        if (nRecGeom != 1 && nRecGeom != nExp) throw Error(EIO_ERR_ARG, "receiver geometry count must be 1 or nExp");
        const int nts = c->fd.p.nts;
        ShotGrids g0 = shot_grids(src, rec, nRecGeom, 0);
        const size_t dslice = (size_t)5 * g0.r[0]->nIrreg * nts;
        std::vector<float> sl[5];   // add = false: each shot's slice is written whole below
        born_model_slice(c->fd, model, sl);
        float* dm[5];
        for (int f = 0; f < 5; f++) dm[f] = sl[f].data();
        for (int e = 0; e < nExp; e++) {
            ShotGrids g = shot_grids(src, rec, nRecGeom, e);
            check_nt(g, nts);
            if ((size_t)5 * g.r[0]->nIrreg * nts != dslice) throw Error(EIO_ERR_ARG, "receiver counts differ");
        }
        const int nb = born_batch_width(c, nExp);
        const int nl = nb ? nb : ensure_lanes(c, nExp, lane_bytes(c, true));
        for (int k = 0; k < nl; k++) engine_dm_upload(lane_engine(c, k), dm);   // stays on the device for every shot
        std::vector<float*> tmp(nl);
        for (int k = 0; k < nl; k++) tmp[k] = add ? lane_staging(c, k, dslice) : nullptr;
        if (nb) {
            for (const auto& grp : shot_groups(nExp, nb)) {
                std::vector<float*> out(grp.second);
                for (int i = 0; i < grp.second; i++) out[i] = add ? tmp[i] : data + (size_t)(grp.first + i) * dslice;
                born_group(c, 0, grp.first, grp.second, nExp, src, rec, nRecGeom, sigs, nSignals, out.data());
                if (add)
                    for (int i = 0; i < grp.second; i++) {
                        float* d = data + (size_t)(grp.first + i) * dslice;
                        const float* t = tmp[i];
#pragma omp parallel for schedule(static)
                        for (long long q = 0; q < (long long)dslice; q++) d[q] += t[q];
                    }
            }
            return;
        }
        run_lanes(c, nl, nExp, [&](int k, Engine* eng, int e) {
            ShotGrids g = shot_grids(src, rec, nRecGeom, e);
            std::vector<float> fine[5];
            born_sources(c, g, sigs[nSignals == 1 ? 0 : e], fine);
            float* sp[5];
            for (int f = 0; f < 5; f++) sp[f] = fine[f].data();
            ShotWindow win(c, eng, g, e, nExp);
            float* d = data + (size_t)e * dslice;
            engine_born_shot(eng, 0, sp, win.sg, g.r, add ? tmp[k] : d);
            if (add) {
                const float* t = tmp[k];
#pragma omp parallel for schedule(static)
                for (long long i = 0; i < (long long)dslice; i++) d[i] += t[i];
            }
        });
    });
}

// The lanes' images (added in lane order on the first lane's device) downloaded
// into sl (dm: its pointers), scaled and un-staggered into model (added):
// BornElasticShotsGpu.cpp:325-371
static void image_to_model(eio_ctx* c, int nl, float* const dm[5], std::vector<float>* sl, float* model) {
    const FdParam& fd = c->fd;
    const int nz = fd.p.nz, nx = fd.p.nx;
    const size_t n = (size_t)nz * nx;
    {
        if (nl > 1) {
            float* d0[5];
            engine_dm_ptrs(c->eng, d0);
            for (int k = 1; k < nl; k++) engine_dm_add(lane_engine(c, k), d0);
        }
        engine_dm_download(c->eng, dm);
        const double tdtw = 2.0 * fd.dtw;
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)n; i++) {
            sl[0][i] *= fd.par[0][i];
            sl[1][i] *= fd.par[1][i];
            sl[2][i] = (float)(sl[2][i] * tdtw);
            sl[3][i] = (float)(sl[3][i] * tdtw);
            sl[4][i] = (float)(sl[4][i] * tdtw);
        }
        std::vector<float> t1(model, model + n);
        stagger_x(0, 1, nz, nx, sl[0].data(), t1.data());
        stagger_z(0, 1, nz, nx, sl[1].data(), t1.data());
        std::copy(t1.begin(), t1.end(), model);
        std::vector<float> t2(n);
        stagger_z(0, 0, nz, nx, sl[4].data(), t2.data());
        std::vector<float> t3(n);
        stagger_x(0, 0, nz, nx, t2.data(), t3.data());
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)n; i++) {
            model[n + i] += sl[2][i];
            model[2 * n + i] += sl[3][i] + t3[i];
        }
    }
}

static int eio_born_adjoint_impl(eio_ctx* c, int add, int nExp, float* model, const float* data,
                             const float* const* sigs, int nSignals, eio_sinterp* const* src, eio_sinterp* const* rec,
                             int nRecGeom) {
    return guarded([&] {
        if (!c || !model || !data || !src || !rec || !sigs || nExp < 1) throw Error(EIO_ERR_ARG, "null argument");
        if (nSignals != 1 && nSignals != nExp) throw Error(EIO_ERR_ARG, "source signal count must be 1 or nExp");
        if (nRecGeom != 1 && nRecGeom != nExp) throw Error(EIO_ERR_ARG, "receiver geometry count must be 1 or nExp");
        const FdParam& fd = c->fd;
        const int nts = fd.p.nts, nz = fd.p.nz, nx = fd.p.nx;
        const size_t n = (size_t)nz * nx;
        if (!add) std::fill(model, model + 3 * n, 0.f);
        ShotGrids g0 = shot_grids(src, rec, nRecGeom, 0);
        const size_t dslice = (size_t)5 * g0.r[0]->nIrreg * nts;
        std::vector<float> sl[5];
        float* dm[5];
        for (int f = 0; f < 5; f++) { sl[f].assign(n, 0.f); dm[f] = sl[f].data(); }
        for (int e = 0; e < nExp; e++) {
            ShotGrids g = shot_grids(src, rec, nRecGeom, e);
            check_nt(g, nts);
            if ((size_t)5 * g.r[0]->nIrreg * nts != dslice) throw Error(EIO_ERR_ARG, "receiver counts differ");
        }
        const int nb = born_batch_width(c, nExp);
        const int nl = nb ? nb : ensure_lanes(c, nExp, lane_bytes(c, true));
        for (int k = 0; k < nl; k++) engine_dm_zero(lane_engine(c, k));   // each lane's shots accumulate on its device
        if (nb) {
            for (const auto& grp : shot_groups(nExp, nb)) {
                std::vector<float*> in(grp.second);
                for (int i = 0; i < grp.second; i++)
                    in[i] = const_cast<float*>(data) + (size_t)(grp.first + i) * dslice;
                born_group(c, 1, grp.first, grp.second, nExp, src, rec, nRecGeom, sigs, nSignals, in.data());
            }
            image_to_model(c, nl, dm, sl, model);
            return;
        }
        run_lanes(c, nl, nExp, [&](int, Engine* eng, int e) {
            ShotGrids g = shot_grids(src, rec, nRecGeom, e);
            std::vector<float> fine[5];
            born_sources(c, g, sigs[nSignals == 1 ? 0 : e], fine);
            float* sp[5];
            for (int f = 0; f < 5; f++) sp[f] = fine[f].data();
            ShotWindow win(c, eng, g, e, nExp);
            engine_born_shot(eng, 1, sp, win.sg, g.r, const_cast<float*>(data) + (size_t)e * dslice);
        });
        image_to_model(c, nl, dm, sl, model);
    });
}



// ------------------------------------------------------------ FWI gradient
namespace {

// residual of one shot: r_k = S_k d - d_obs_k for the sampled components
// (codes 0..4 the fields, 5 the pressure 0.5 (sxx + szz)), its misfit
// 0.5 r.r in FP64, and S^T r into the five fields
struct ShotResidual {
    int nComp, nri, nts;
    const int* comps;
    const float* dobs;          // [nComp][nri][nts] of this shot
    std::vector<float> r;       // [nComp][nri][nts]
};

double shot_residual(void* p, const float* d, float* rt) {
    ShotResidual& s = *static_cast<ShotResidual*>(p);
    const size_t m = (size_t)s.nri * s.nts;
    s.r.resize((size_t)s.nComp * m);
    for (int k = 0; k < s.nComp; k++) {
        const int code = s.comps[k];
        float* rk = s.r.data() + (size_t)k * m;
        const float* ok = s.dobs + (size_t)k * m;
        if (code < 5) {
            const float* df = d + (size_t)code * m;
            for (size_t i = 0; i < m; i++) rk[i] = df[i] - ok[i];
        } else {
            const float* d2 = d + 2 * m;
            const float* d3 = d + 3 * m;
            for (size_t i = 0; i < m; i++) rk[i] = 0.5f * (d2[i] + d3[i]) - ok[i];
        }
    }
    std::fill(rt, rt + 5 * m, 0.f);
    for (int k = 0; k < s.nComp; k++) {
        const int code = s.comps[k];
        const float* rk = s.r.data() + (size_t)k * m;
        if (code < 5) {
            float* tf = rt + (size_t)code * m;
            for (size_t i = 0; i < m; i++) tf[i] += rk[i];
        } else {
            float* t2 = rt + 2 * m;
            float* t3 = rt + 3 * m;
            for (size_t i = 0; i < m; i++) { t2[i] += 0.5f * rk[i]; t3[i] += 0.5f * rk[i]; }
        }
    }
    // FP64 sum in index order on the host thread of the lane: a device
    // reduction here would allocate and free on the device, which waits for
    // the other lanes' kernels
    double acc = 0.0;
    for (float v : s.r) acc += (double)v * (double)v;
    return 0.5 * acc;
}

}  // namespace

static int eio_fwi_gradient_impl(eio_ctx* c, int nExp, int nModelExp, const float* model, const float* dobs, int nComp,
                             const int* comps, eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom,
                             float* data, float* grad, double* misfit) {
    return guarded([&] {
        if (!c || !model || !dobs || !src || !rec || !grad || !misfit || nExp < 1) throw Error(EIO_ERR_ARG, "null argument");
        if (nModelExp != 1 && nModelExp != nExp) throw Error(EIO_ERR_ARG, "model shot axis must be 1 or nExp");
        if (nRecGeom != 1 && nRecGeom != nExp) throw Error(EIO_ERR_ARG, "receiver geometry count must be 1 or nExp");
        if (nComp < 1 || nComp > 6 || !comps) throw Error(EIO_ERR_ARG, "1 .. 6 data components");
        for (int k = 0; k < nComp; k++)
            if (comps[k] < 0 || comps[k] > 5) throw Error(EIO_ERR_ARG, "component codes are 0..4 (fields) or 5 (pressure)");
        if (c->fd.p.surfaceCondition) throw Error(EIO_ERR_UNSUPPORTED, "the Born operators ignore the free surface");
        const FdParam& fd = c->fd;
        const int nts = fd.p.nts;
        const size_t n = (size_t)fd.p.nz * fd.p.nx;
        ShotGrids g0 = shot_grids(src, rec, nRecGeom, 0);
        const int nri = g0.r[0]->nIrreg, nsi = g0.s[0]->nIrreg;
        const size_t dslice = (size_t)5 * nri * nts, oslice = (size_t)nComp * nri * nts;
        const size_t mslice = (size_t)5 * nsi * nts;
        for (int e = 0; e < nExp; e++) {
            ShotGrids g = shot_grids(src, rec, nRecGeom, e);
            check_nt(g, nts);
            if ((size_t)5 * g.s[0]->nIrreg * nts != mslice || (size_t)5 * g.r[0]->nIrreg * nts != dslice)
                throw Error(EIO_ERR_ARG, "device counts differ between shots");
        }
        const int nl = ensure_lanes(c, nExp, lane_bytes(c, true));
        for (int k = 0; k < nl; k++) engine_dm_zero(lane_engine(c, k));
        std::vector<std::vector<float>> dtmp(nl), rtmp(nl);
        std::vector<double> phi(nExp, 0.0);
        run_lanes(c, nl, nExp, [&](int k, Engine* eng, int e) {
            ShotGrids g = shot_grids(src, rec, nRecGeom, e);
            const float* ms = model + (nModelExp == 1 ? 0 : (size_t)e * mslice);
            std::vector<float> reg[5];
            float* mp[5];
            for (int f = 0; f < 5; f++) {
                const SInterp& s = *g.s[kFG[f]];
                reg[f].assign((size_t)s.nReg * nts, 0.f);
                sinterp_adjoint(s, false, reg[f].data(), ms + (size_t)f * nsi * nts);
            }
            scale_sources(fd, g, reg, nts);
            for (int f = 0; f < 5; f++) mp[f] = reg[f].data();
            float* d = data ? data + (size_t)e * dslice : nullptr;
            if (!d) {
                dtmp[k].resize(dslice);
                d = dtmp[k].data();
            }
            rtmp[k].resize(dslice);
            ShotResidual sr{nComp, nri, nts, comps, dobs + (size_t)e * oslice, {}};
            ShotWindow win(c, eng, g, e, nExp);
            float* img[5];
            engine_dm_window(eng, img);
            phi[e] = engine_fwi_shot(eng, mp, win.sg, g.r, d, rtmp[k].data(), shot_residual, &sr, img);
        });
        double total = 0.0;
        for (int e = 0; e < nExp; e++) total += phi[e];   // shot order
        *misfit = total;
        std::fill(grad, grad + 3 * n, 0.f);
        std::vector<float> sl[5];
        float* dm[5];
        for (int f = 0; f < 5; f++) { sl[f].assign(n, 0.f); dm[f] = sl[f].data(); }
        image_to_model(c, nl, dm, sl, grad);
    });
}

// ------------------------------------------------------------ learned preconditioner

EIO_API int eio_born_forward(eio_ctx* c, int add, int nExp, const float* model, float* data,
                             const float* const* sigs, int nSignals, eio_sinterp* const* src, eio_sinterp* const* rec,
                             int nRecGeom) {
    return finite_call(
        c, [&] { return std::vector<FSpan>{{model, (size_t)3 * c->fd.p.nz * c->fd.p.nx, "model perturbation"}}; },
        [&] { return eio_born_forward_impl(c, add, nExp, model, data, sigs, nSignals, src, rec, nRecGeom); },
        [&] { return std::vector<FSpan>{{data, data_elems(c, src, rec, nRecGeom, nExp), "data"}}; });
}
EIO_API int eio_born_adjoint(eio_ctx* c, int add, int nExp, float* model, const float* data,
                             const float* const* sigs, int nSignals, eio_sinterp* const* src, eio_sinterp* const* rec,
                             int nRecGeom) {
    return finite_call(
        c, [&] { return std::vector<FSpan>{{data, data_elems(c, src, rec, nRecGeom, nExp), "data"}}; },
        [&] { return eio_born_adjoint_impl(c, add, nExp, model, data, sigs, nSignals, src, rec, nRecGeom); },
        [&] { return std::vector<FSpan>{{model, (size_t)3 * c->fd.p.nz * c->fd.p.nx, "model perturbation"}}; });
}
EIO_API int eio_fwi_gradient(eio_ctx* c, int nExp, int nModelExp, const float* model, const float* dobs, int nComp,
                             const int* comps, eio_sinterp* const* src, eio_sinterp* const* rec, int nRecGeom,
                             float* data, float* grad, double* misfit) {
    return finite_call(
        c, [&] { return std::vector<FSpan>{}; },   // the model is the medium: always checked
        [&] {
            return eio_fwi_gradient_impl(c, nExp, nModelExp, model, dobs, nComp, comps, src, rec, nRecGeom, data, grad,
                                         misfit);
        },
        [&] {
            if (misfit && !std::isfinite(*misfit))
                throw Error(EIO_ERR_NONFINITE, "non-finite misfit (unstable propagation?)");
            return std::vector<FSpan>{{grad, (size_t)3 * c->fd.p.nz * c->fd.p.nx, "gradient"}};
        });
}

EIO_API int eio_cnn_conv3x3(int n, int h, int w, int cin, int cout, const void* x, const void* wt, const void* mask,
                            int relu, void* y, float* y32, void* stream) {
    return guarded([&] { cnn_conv3x3(n, h, w, cin, cout, x, wt, mask, relu, y, y32, stream); });
}
EIO_API int eio_cnn_set_conv_path(int path) {
    return guarded([&] { cnn_set_conv_path(path); });
}
EIO_API int eio_cnn_get_conv_path(int* path) {
    return guarded([&] {
        if (!path) throw Error(EIO_ERR_ARG, "null result");
        *path = cnn_get_conv_path();
    });
}
EIO_API int eio_cnn_set_wait_limit(long long polls) {
    return guarded([&] { cnn_set_wait_limit(polls); });
}
EIO_API int eio_cnn_get_wait_limit(long long* polls) {
    return guarded([&] {
        if (!polls) throw Error(EIO_ERR_ARG, "null output");
        *polls = cnn_get_wait_limit();
    });
}
EIO_API int eio_cnn_status(int reset, int* err) {
    return guarded([&] {
        if (!err) throw Error(EIO_ERR_ARG, "null result");
        *err = cnn_status(reset);
    });
}
EIO_API int eio_cnn_wgrad_scratch(int n, int h, int w, int cin, int cout, long long* floats) {
    return guarded([&] {
        if (!floats) throw Error(EIO_ERR_ARG, "null result");
        *floats = cnn_wgrad_scratch(n, h, w, cin, cout);
    });
}
EIO_API int eio_cnn_conv3x3_wgrad(int n, int h, int w, int cin, int cout, const void* x, const void* dy, float* dw,
                                  float* scratch, long long scratchFloats, void* stream) {
    return guarded([&] { cnn_conv3x3_wgrad(n, h, w, cin, cout, x, dy, dw, scratch, scratchFloats, stream); });
}
EIO_API int eio_cnn_flip(int cin, int cout, const void* w, void* wt, void* stream) {
    return guarded([&] { cnn_flip(cin, cout, w, wt, stream); });
}
EIO_API int eio_cnn_mse(long long npix, int c, int nc, const float* y32, const float* target, void* dz,
                        double* scratch, double* loss, void* stream) {
    return guarded([&] { cnn_mse(npix, c, nc, y32, target, dz, scratch, loss, stream); });
}
EIO_API int eio_cnn_adam(long long n, float* p, float* m, float* v, const float* g, float lr, float b1, float b2,
                         float eps, int step, void* pb, void* stream) {
    return guarded([&] { cnn_adam(n, p, m, v, g, lr, b1, b2, eps, step, pb, stream); });
}

// ---- U-Net preconditioner kernels ------------------------------------------
EIO_API int eio_gemm_bf16(long long M, long long N, long long K, const void* A, long long lda, const void* B,
                          long long ldb, float* C32, void* C16, const void* mask, int relu, int splits, float* scratch,
                          void* stream) {
    return guarded([&] { gemm_bf16(M, N, K, A, lda, B, ldb, C32, C16, mask, relu, splits, scratch, stream); });
}
EIO_API int eio_gemm_set_wait_limit(long long polls) {
    return guarded([&] { gemm_set_wait_limit(polls); });
}
EIO_API int eio_gemm_status(int reset, int* err) {
    return guarded([&] {
        if (!err) throw Error(EIO_ERR_ARG, "null result");
        *err = gemm_status(reset);
    });
}
EIO_API int eio_unet_set_tma(int on) {
    return guarded([&] { unet_set_tma(on); });
}
EIO_API int eio_unet_get_tma(int* on) {
    return guarded([&] {
        if (!on) throw Error(EIO_ERR_ARG, "null result");
        *on = unet_get_tma();
    });
}
EIO_API int eio_unet_conv3x3(int n, int h, int w, int cin, int cout, const void* x, const void* wt, float* y32,
                             void* y16, int relu, void* stream) {
    return guarded([&] { unet_conv3x3(n, h, w, cin, cout, x, wt, y32, y16, relu, stream); });
}
EIO_API int eio_unet_wgrad_scratch(int n, int h, int w, int cin, int cout, long long* floats) {
    return guarded([&] {
        if (!floats) throw Error(EIO_ERR_ARG, "null result");
        *floats = unet_wgrad_scratch(n, h, w, cin, cout);
    });
}
EIO_API int eio_unet_conv3x3_wgrad(int n, int h, int w, int cin, int cout, const void* x, const void* dz, float* dw,
                                   float* scratch, long long scratchFloats, void* stream) {
    return guarded([&] { unet_conv3x3_wgrad(n, h, w, cin, cout, x, dz, dw, scratch, scratchFloats, stream); });
}
EIO_API int eio_unet_flip(int cout, int cin, const void* w, void* wf, void* stream) {
    return guarded([&] { unet_flip(cout, cin, w, wf, stream); });
}
EIO_API int eio_unet_resample(int op, int n, int h, int w, int c, const void* in, void* out, int add, void* stream) {
    return guarded([&] { unet_resample(op, n, h, w, c, in, out, add, stream); });
}
EIO_API int eio_unet_concat(int adj, long long pixels, int ca, int cb, void* a, int addA, void* b, int addB, void* z,
                            void* stream) {
    return guarded([&] { unet_concat(adj, pixels, ca, cb, a, addA, b, addB, z, stream); });
}
EIO_API int eio_unet_relu_adj(long long n, const void* src, const void* mask, void* dst, int add, void* stream) {
    return guarded([&] { unet_relu_adj(n, src, mask, dst, add, stream); });
}
