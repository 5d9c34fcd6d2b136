// Device engine: buffers, sparse point lists and the time loops of the four
// propagations (nonlinear forward/adjoint, Born forward/adjoint).
//
// Time loops restate propShotsElasticFwdGpu / propShotsElasticAdjGpu
// (F/src/nonlinearPropElasticGpuFunctions.cu:561-648, 932-1027) and the
// non-stream paths of BornShotsFwdGpu / BornShotsAdjGpu
// (F/src/BornElasticGpuFunctions.cu:744-849, 1125-1191), with one fused
// k_step launch per fine step instead of 4-12 reference launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "eio_internal.h"
#include "eio_kernels.cuh"

namespace eio {

#define EIO_CUDA(x)                                                                                    \
    do {                                                                                               \
        cudaError_t e_ = (x);                                                                          \
        if (e_ != cudaSuccess)                                                                         \
            throw Error(EIO_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));               \
    } while (0)

// growable device buffer
struct DBuf {
    void* p = nullptr;
    size_t cap = 0;
    void ensure(size_t bytes) {
        if (bytes <= cap) return;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            p = nullptr;
            throw Error(e == cudaErrorMemoryAllocation ? EIO_ERR_NOMEM : EIO_ERR_CUDA,
                        std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
        }
        cap = bytes;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    float* f() const { return static_cast<float*>(p); }
};

static const int kFieldGrid[5] = {1, 2, 0, 0, 3};   // vx->x, vz->z, sxx,szz->center, sxz->xz

struct PointList {
    std::vector<int> tile_start;
    std::vector<PointEntry> ent;
    int ld[5] = {0, 0, 0, 0, 0};
    bool any = false;
};

struct Engine {
    int device = 0;
    cudaStream_t st = nullptr;
    int nz = 0, nx = 0;
    long long n = 0;
    int nts = 0, S = 0, ntw = 0, h = 0;
    float zc[4], xc[4];
    std::vector<float> filt;
    float dts_inv = 0.f;
    int ntz = 0, ntx = 0, ntiles = 0;
    int ckpt = 0;
    DBuf par[5], dampz, dampx, wf[10];
    DBuf inj_ts, inj_ent, ext_ts, ext_ent;
    DBuf sig_in[5], sig_out[5];
    DBuf stage_a[5], stage_b[5], stage_c[5];
    DBuf W, ss[10];
    // launch statistics (bench instrumentation)
    long long launches = 0, step_launches = 0;
    double step_ms = 0.0;
    bool stats = false;
    std::vector<cudaEvent_t> ev;
    size_t ev_used = 0;
};

// Per-launch CUDA-event timing of the fused step kernel (only when enabled).
static void stats_flush(Engine* e) {
    if (!e->stats || e->ev_used == 0) return;
    EIO_CUDA(cudaStreamSynchronize(e->st));
    for (size_t k = 0; k + 1 < e->ev_used; k += 2) {
        float ms = 0.f;
        EIO_CUDA(cudaEventElapsedTime(&ms, e->ev[k], e->ev[k + 1]));
        e->step_ms += ms;
    }
    e->ev_used = 0;
}
static void stats_mark(Engine* e) {
    if (!e->stats) return;
    if (e->ev_used == e->ev.size()) {
        if (e->ev.size() >= 65536) stats_flush(e);
        else {
            const size_t grow = e->ev.empty() ? 4096 : e->ev.size();
            for (size_t i = 0; i < grow; i++) {
                cudaEvent_t x;
                EIO_CUDA(cudaEventCreate(&x));
                e->ev.push_back(x);
            }
        }
    }
    EIO_CUDA(cudaEventRecord(e->ev[e->ev_used++], e->st));
}

static void upload(DBuf& b, const void* h, size_t bytes, cudaStream_t st) {
    b.ensure(std::max<size_t>(bytes, 16));
    if (bytes) EIO_CUDA(cudaMemcpyAsync(b.p, h, bytes, cudaMemcpyHostToDevice, st));
}

void engine_set_medium(Engine* e, const FdParam& fd) {
    EIO_CUDA(cudaSetDevice(e->device));
    const int nz = fd.p.nz, nx = fd.p.nx;
    if (nz != e->nz || nx != e->nx) throw Error(EIO_ERR_ARG, "setBackground: grid size changed");
    for (int f = 0; f < 5; f++) upload(e->par[f], fd.par[f].data(), sizeof(float) * e->n, e->st);
    // per-axis taper tables: the taper of a cell is damp[min(distance to any edge)]
    // and damp[] is non-decreasing, so it equals min(dampz[iz], dampx[ix]).
    std::vector<float> dz(nz, 1.f), dx(nx, 1.f);
    for (int iz = FAT; iz < nz - FAT; iz++) {
        int d = std::min(iz - FAT, nz - iz - 1 - FAT);
        if (d < fd.minPad) dz[iz] = fd.damp[d];
    }
    for (int ix = FAT; ix < nx - FAT; ix++) {
        int d = std::min(ix - FAT, nx - ix - 1 - FAT);
        if (d < fd.minPad) dx[ix] = fd.damp[d];
    }
    for (int i = 1; i < fd.minPad; i++)
        if (fd.damp[i] < fd.damp[i - 1]) throw Error(EIO_ERR_ARG, "cosine taper table is not monotone");
    upload(e->dampz, dz.data(), sizeof(float) * nz, e->st);
    upload(e->dampx, dx.data(), sizeof(float) * nx, e->st);
    e->nts = fd.p.nts;
    e->S = fd.S;
    e->ntw = fd.ntw;
    e->h = fd.S + 1;
    for (int i = 0; i < 4; i++) { e->zc[i] = fd.zc[i]; e->xc[i] = fd.xc[i]; }
    e->filt = fd.filt;
    e->dts_inv = fd.dts_inv;
    EIO_CUDA(cudaStreamSynchronize(e->st));
}

Engine* engine_create(int device, const FdParam& fd) {
    int ndev = 0;
    EIO_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) throw Error(EIO_ERR_ARG, "invalid CUDA device " + std::to_string(device));
    EIO_CUDA(cudaSetDevice(device));
    Engine* e = new Engine();
    try {
        e->device = device;
        e->nz = fd.p.nz;
        e->nx = fd.p.nx;
        e->n = (long long)e->nz * e->nx;
        if ((e->nz - 2 * FAT) % 16 || (e->nx - 2 * FAT) % 16 || e->nz % 4)
            throw Error(EIO_ERR_QC, "nz-2*fat and nx-2*fat must be multiples of 16");
        e->ntz = (e->nz - 2 * FAT + TZ - 1) / TZ;
        e->ntx = (e->nx - 2 * FAT) / TX;
        e->ntiles = e->ntz * e->ntx;
        EIO_CUDA(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
        for (int f = 0; f < 10; f++) e->wf[f].ensure(sizeof(float) * e->n);
        engine_set_medium(e, fd);
    } catch (...) {
        engine_destroy(e);
        throw;
    }
    return e;
}

void engine_destroy(Engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->st) cudaStreamSynchronize(e->st);
    DBuf* all[] = {&e->dampz, &e->dampx, &e->inj_ts, &e->inj_ent, &e->ext_ts, &e->ext_ent, &e->W};
    for (DBuf* b : all) b->release();
    for (int f = 0; f < 5; f++) {
        e->par[f].release(); e->sig_in[f].release(); e->sig_out[f].release();
        e->stage_a[f].release(); e->stage_b[f].release(); e->stage_c[f].release();
    }
    for (int f = 0; f < 10; f++) { e->wf[f].release(); e->ss[f].release(); }
    for (cudaEvent_t x : e->ev) cudaEventDestroy(x);
    if (e->st) cudaStreamDestroy(e->st);
    delete e;
}

void engine_set_checkpoint(Engine* e, int mode) {
    if (mode != 0) throw Error(EIO_ERR_UNSUPPORTED, "only FP32 source-wavefield snapshots are available");
    e->ckpt = mode;
}

void* engine_stream(Engine* e) { return (void*)e->st; }

void engine_stats(Engine* e, int enable, int reset, long long* launches, long long* step_launches, double* step_ms) {
    stats_flush(e);
    if (launches) *launches = e->launches;
    if (step_launches) *step_launches = e->step_launches;
    if (step_ms) *step_ms = e->step_ms;
    if (reset) { e->launches = 0; e->step_launches = 0; e->step_ms = 0.0; }
    if (enable >= 0) e->stats = enable != 0;
}

// Sort the points of the four position lists into per-tile buckets.
static void build_points(const Engine* e, const int* const pos[4], const int npos[4], PointList& pl) {
    std::vector<std::pair<int, PointEntry>> tmp;
    for (int f = 0; f < 5; f++) {
        const int g = kFieldGrid[f];
        pl.ld[f] = npos[g];
        for (int k = 0; k < npos[g]; k++) {
            const int cell = pos[g][k];
            const int ix = cell / e->nz, iz = cell % e->nz;
            if (cell < 0 || ix < FAT || ix >= e->nx - FAT || iz < FAT || iz >= e->nz - FAT)
                throw Error(EIO_ERR_BOUNDS, "acquisition point " + std::to_string(cell) +
                                                " lies outside the updated interior of the grid");
            const int bz = (iz - FAT) / TZ, bx = (ix - FAT) / TX;
            PointEntry pe;
            pe.key = (f << 16) | (((ix - FAT) % TX) << 8) | ((iz - FAT) % TZ);
            pe.col = k;
            tmp.push_back({bx * e->ntz + bz, pe});
        }
    }
    pl.any = !tmp.empty();
    pl.tile_start.assign(e->ntiles + 1, 0);
    for (auto& t : tmp) pl.tile_start[t.first + 1]++;
    for (int i = 0; i < e->ntiles; i++) pl.tile_start[i + 1] += pl.tile_start[i];
    pl.ent.resize(tmp.size());
    std::vector<int> cur(pl.tile_start.begin(), pl.tile_start.end() - 1);
    for (auto& t : tmp) pl.ent[cur[t.first]++] = t.second;
}

static SparseOp upload_points(Engine* e, const PointList& pl, DBuf& ts, DBuf& ent, DBuf* sig) {
    SparseOp op;
    memset(&op, 0, sizeof(op));
    if (!pl.any) return op;
    upload(ts, pl.tile_start.data(), sizeof(int) * pl.tile_start.size(), e->st);
    upload(ent, pl.ent.data(), sizeof(PointEntry) * pl.ent.size(), e->st);
    op.tile_start = static_cast<const int*>(ts.p);
    op.ent = static_cast<const PointEntry*>(ent.p);
    for (int f = 0; f < 5; f++) {
        op.sig[f] = sig[f].f();
        op.ld[f] = pl.ld[f];
    }
    return op;
}

static void transpose(Engine* e, const float* in, float* out, int rows, int cols) {
    if (rows == 0 || cols == 0) return;
    dim3 b(32, 8), g((cols + 31) / 32, (rows + 31) / 32);
    k_transpose<<<g, b, 0, e->st>>>(in, out, rows, cols);
    e->launches++;
}

static StepArgs base_args(Engine* e) {
    StepArgs a;
    memset(&a, 0, sizeof(a));
    for (int f = 0; f < 5; f++) a.par[f] = e->par[f].f();
    a.dampz = e->dampz.f();
    a.dampx = e->dampx.f();
    a.nz = e->nz;
    a.nx = e->nx;
    a.ntz = e->ntz;
    for (int i = 0; i < 4; i++) { a.cz[i] = e->zc[i]; a.cx[i] = e->xc[i]; }
    a.wstride = e->n;
    return a;
}

template <int DIR, int EPI>
static void launch_step(Engine* e, StepArgs& a) {
    stats_mark(e);
    k_step<DIR, EPI><<<e->ntiles, NT, 0, e->st>>>(a);
    stats_mark(e);
    e->launches++;
    e->step_launches++;
}

static void zero_wavefields(Engine* e) {
    for (int f = 0; f < 10; f++) EIO_CUDA(cudaMemsetAsync(e->wf[f].p, 0, sizeof(float) * e->n, e->st));
}

static void check_launch() {
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) throw Error(EIO_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(err));
}

// signal matrices: trace-major device inputs -> time-major device buffers
static void stage_in(Engine* e, float* const tr[5], const int ld[5], int nt, DBuf* dst) {
    for (int f = 0; f < 5; f++) {
        dst[f].ensure(std::max<size_t>(sizeof(float) * (size_t)ld[f] * nt, 16));
        transpose(e, tr[f], dst[f].f(), ld[f], nt);
    }
}
static void zero_out(Engine* e, const int ld[5], int nt, DBuf* dst) {
    for (int f = 0; f < 5; f++) {
        size_t bytes = sizeof(float) * (size_t)ld[f] * nt;
        dst[f].ensure(std::max<size_t>(bytes, 16));
        if (bytes) EIO_CUDA(cudaMemsetAsync(dst[f].p, 0, bytes, e->st));
    }
}
static void stage_out(Engine* e, const int ld[5], int nt, DBuf* src, float* const tr[5]) {
    for (int f = 0; f < 5; f++) transpose(e, src[f].f(), tr[f], nt, ld[f]);
}

void engine_nl(Engine* e, int adj, float* const model[5], float* const data[5], const ShotGeom& g) {
    EIO_CUDA(cudaSetDevice(e->device));
    PointList src, rec;
    build_points(e, g.srcPos, g.nSrc, src);
    build_points(e, g.recPos, g.nRec, rec);
    StepArgs a = base_args(e);
    zero_wavefields(e);
    float* p0[5]; float* p1[5];
    for (int f = 0; f < 5; f++) { p0[f] = e->wf[f].f(); p1[f] = e->wf[5 + f].f(); }
    const float* F = e->filt.data();
    const int h = e->h;
    if (!adj) {
        stage_in(e, model, src.ld, e->nts, e->sig_in);
        zero_out(e, rec.ld, e->nts, e->sig_out);
        a.inj = upload_points(e, src, e->inj_ts, e->inj_ent, e->sig_in);
        a.ext = upload_points(e, rec, e->ext_ts, e->ext_ent, e->sig_out);
        for (int its = 0; its < e->nts - 1; its++)
            for (int it2 = 1; it2 < e->S + 1; it2++) {
                for (int f = 0; f < 5; f++) { a.o[f] = p0[f]; a.c[f] = p1[f]; }
                a.inj.t0 = its; a.inj.w0 = F[it2 - 1]; a.inj.w1 = F[h + it2 - 1];
                a.ext.t0 = its; a.ext.w0 = F[it2]; a.ext.w1 = F[h + it2];
                launch_step<0, EPI_NONE>(e, a);
                std::swap(p0, p1);
            }
        check_launch();
        stage_out(e, rec.ld, e->nts, e->sig_out, data);
    } else {
        stage_in(e, data, rec.ld, e->nts, e->sig_in);
        zero_out(e, src.ld, e->nts, e->sig_out);
        a.inj = upload_points(e, rec, e->inj_ts, e->inj_ent, e->sig_in);
        a.ext = upload_points(e, src, e->ext_ts, e->ext_ent, e->sig_out);
        for (int its = e->nts - 2; its > -1; its--)
            for (int it2 = e->S - 1; it2 > -1; it2--) {
                for (int f = 0; f < 5; f++) { a.o[f] = p0[f]; a.c[f] = p1[f]; }
                a.inj.t0 = its; a.inj.w0 = F[it2 + 1]; a.inj.w1 = F[h + it2 + 1];
                a.ext.t0 = its; a.ext.w0 = F[it2]; a.ext.w1 = F[h + it2];
                launch_step<1, EPI_NONE>(e, a);
                std::swap(p0, p1);
            }
        check_launch();
        stage_out(e, src.ld, e->nts, e->sig_out, model);
    }
    EIO_CUDA(cudaStreamSynchronize(e->st));
    stats_flush(e);
}

static void launch_imaging(Engine* e, int adj, int its, float* const dm[5], float* const ss[5]) {
    ImagingArgs ia;
    memset(&ia, 0, sizeof(ia));
    ia.Wvx = e->W.f();
    ia.Wvz = e->W.f() + (long long)e->nts * e->n;
    ia.wstride = e->n;
    ia.nz = e->nz; ia.nx = e->nx; ia.nts = e->nts; ia.its = its;
    for (int i = 0; i < 4; i++) { ia.cz[i] = e->zc[i]; ia.cx[i] = e->xc[i]; }
    ia.dts_inv = e->dts_inv;
    for (int f = 0; f < 5; f++) { ia.dm[f] = dm[f]; ia.ss[f] = ss[f]; }
    dim3 b(256), g((e->nz - 2 * FAT + 255) / 256, e->nx - 2 * FAT);
    if (adj) k_imaging<1><<<g, b, 0, e->st>>>(ia);
    else k_imaging<0><<<g, b, 0, e->st>>>(ia);
    e->launches++;
}

// Source wavefield + coarse Vx/Vz history (BornElasticGpuFunctions.cu:746-768)
static void born_source(Engine* e, const PointList& src, StepArgs a) {
    const size_t wbytes = sizeof(float) * 2 * (size_t)e->nts * e->n;
    e->W.ensure(wbytes);
    EIO_CUDA(cudaMemsetAsync(e->W.p, 0, wbytes, e->st));
    zero_wavefields(e);
    float* p0[5]; float* p1[5];
    for (int f = 0; f < 5; f++) { p0[f] = e->wf[f].f(); p1[f] = e->wf[5 + f].f(); }
    a.inj = upload_points(e, src, e->inj_ts, e->inj_ent, e->sig_in);
    memset(&a.ext, 0, sizeof(a.ext));
    a.W0 = e->W.f();
    a.W1 = e->W.f() + (long long)e->nts * e->n;
    const float* F = e->filt.data();
    for (int its = 0; its < e->nts - 1; its++)
        for (int it2 = 1; it2 < e->S + 1; it2++) {
            const int itw = its * e->S + it2;
            for (int f = 0; f < 5; f++) { a.o[f] = p0[f]; a.c[f] = p1[f]; }
            a.inj.t0 = itw - 1; a.inj.w0 = 1.f; a.inj.w1 = 0.f;
            a.wt = its; a.ww0 = F[it2]; a.ww1 = F[e->h + it2];
            launch_step<0, EPI_SAVE_W>(e, a);
            std::swap(p0, p1);
        }
    check_launch();
}

void engine_born(Engine* e, int adj, float* const srcDtw[5], float* const dm[5], float* const data[5],
                 const ShotGeom& g) {
    EIO_CUDA(cudaSetDevice(e->device));
    if (e->ckpt != 0) throw Error(EIO_ERR_UNSUPPORTED, "checkpoint mode");
    PointList src, rec;
    build_points(e, g.srcPos, g.nSrc, src);
    build_points(e, g.recPos, g.nRec, rec);
    StepArgs base = base_args(e);
    const float* F = e->filt.data();
    const int h = e->h;
    // phase 1: source wavefield
    stage_in(e, srcDtw, src.ld, e->ntw, e->sig_in);
    born_source(e, src, base);
    // phase 2
    for (int f = 0; f < 10; f++) {
        e->ss[f].ensure(sizeof(float) * e->n);
        EIO_CUDA(cudaMemsetAsync(e->ss[f].p, 0, sizeof(float) * e->n, e->st));
    }
    zero_wavefields(e);
    float* p0[5]; float* p1[5]; float* sL[5]; float* sR[5];
    for (int f = 0; f < 5; f++) {
        p0[f] = e->wf[f].f(); p1[f] = e->wf[5 + f].f();
        sL[f] = e->ss[f].f(); sR[f] = e->ss[5 + f].f();
    }
    StepArgs a = base;
    if (!adj) {
        zero_out(e, rec.ld, e->nts, e->sig_out);
        a.ext = upload_points(e, rec, e->ext_ts, e->ext_ent, e->sig_out);
        launch_imaging(e, 0, 0, dm, sL);
        for (int its = 0; its < e->nts - 1; its++) {
            launch_imaging(e, 0, its + 1, dm, sR);
            for (int it2 = 1; it2 < e->S + 1; it2++) {
                for (int f = 0; f < 5; f++) { a.o[f] = p0[f]; a.c[f] = p1[f]; a.ssL[f] = sL[f]; a.ssR[f] = sR[f]; }
                a.sw0 = F[it2 - 1]; a.sw1 = F[h + it2 - 1];
                a.ext.t0 = its; a.ext.w0 = F[it2]; a.ext.w1 = F[h + it2];
                launch_step<0, EPI_INJ_SS>(e, a);
                std::swap(p0, p1);
            }
            // the imaging kernel rewrites every interior cell of the right slice,
            // so the reference's memset of it (BornElasticGpuFunctions.cu:806-810) is not needed
            std::swap(sL, sR);
        }
        check_launch();
        stage_out(e, rec.ld, e->nts, e->sig_out, data);
    } else {
        stage_in(e, data, rec.ld, e->nts, e->sig_in);
        a.inj = upload_points(e, rec, e->inj_ts, e->inj_ent, e->sig_in);
        for (int its = e->nts - 2; its > -1; its--) {
            for (int it2 = e->S - 1; it2 > -1; it2--) {
                for (int f = 0; f < 5; f++) { a.o[f] = p0[f]; a.c[f] = p1[f]; a.eL[f] = sL[f]; a.eR[f] = sR[f]; }
                a.inj.t0 = its; a.inj.w0 = F[it2 + 1]; a.inj.w1 = F[h + it2 + 1];
                a.sw0 = F[it2]; a.sw1 = F[h + it2];
                launch_step<1, EPI_EXT_SS>(e, a);
                std::swap(p0, p1);
            }
            launch_imaging(e, 1, its + 1, dm, sR);
            std::swap(sL, sR);
            for (int f = 0; f < 5; f++) EIO_CUDA(cudaMemsetAsync(sL[f], 0, sizeof(float) * e->n, e->st));
        }
        launch_imaging(e, 1, 0, dm, sR);
        check_launch();
    }
    EIO_CUDA(cudaStreamSynchronize(e->st));
    stats_flush(e);
}

// ---------------------------------------------------------------- host wrappers
static void h2d(Engine* e, DBuf& b, const float* h, size_t count) {
    b.ensure(std::max<size_t>(sizeof(float) * count, 16));
    if (count) EIO_CUDA(cudaMemcpyAsync(b.p, h, sizeof(float) * count, cudaMemcpyHostToDevice, e->st));
}
static void d2h(Engine* e, float* h, const DBuf& b, size_t count) {
    if (count) EIO_CUDA(cudaMemcpyAsync(h, b.p, sizeof(float) * count, cudaMemcpyDeviceToHost, e->st));
}

void engine_nl_host(Engine* e, int adj, float* const model[5], float* const data[5], const ShotGeom& g) {
    EIO_CUDA(cudaSetDevice(e->device));
    float* dmod[5]; float* ddat[5];
    size_t nm[5], nd[5];
    for (int f = 0; f < 5; f++) {
        nm[f] = (size_t)g.nSrc[kFieldGrid[f]] * e->nts;
        nd[f] = (size_t)g.nRec[kFieldGrid[f]] * e->nts;
        if (!adj) { h2d(e, e->stage_a[f], model[f], nm[f]); e->stage_b[f].ensure(std::max<size_t>(16, 4 * nd[f])); }
        else { h2d(e, e->stage_b[f], data[f], nd[f]); e->stage_a[f].ensure(std::max<size_t>(16, 4 * nm[f])); }
        dmod[f] = e->stage_a[f].f();
        ddat[f] = e->stage_b[f].f();
    }
    engine_nl(e, adj, dmod, ddat, g);
    for (int f = 0; f < 5; f++) {
        if (!adj) d2h(e, data[f], e->stage_b[f], nd[f]);
        else d2h(e, model[f], e->stage_a[f], nm[f]);
    }
    EIO_CUDA(cudaStreamSynchronize(e->st));
}

void engine_born_host(Engine* e, int adj, float* const srcDtw[5], float* const dm[5], float* const data[5],
                      const ShotGeom& g) {
    EIO_CUDA(cudaSetDevice(e->device));
    float* ds[5]; float* dd[5]; float* dr[5];
    size_t ns[5], nr[5];
    for (int f = 0; f < 5; f++) {
        ns[f] = (size_t)g.nSrc[kFieldGrid[f]] * e->ntw;
        nr[f] = (size_t)g.nRec[kFieldGrid[f]] * e->nts;
        h2d(e, e->stage_a[f], srcDtw[f], ns[f]);
        h2d(e, e->stage_c[f], dm[f], e->n);
        if (adj) h2d(e, e->stage_b[f], data[f], nr[f]);
        else e->stage_b[f].ensure(std::max<size_t>(16, 4 * nr[f]));
        ds[f] = e->stage_a[f].f(); dr[f] = e->stage_b[f].f(); dd[f] = e->stage_c[f].f();
    }
    engine_born(e, adj, ds, dd, dr, g);
    for (int f = 0; f < 5; f++) {
        if (!adj) d2h(e, data[f], e->stage_b[f], nr[f]);
        else d2h(e, dm[f], e->stage_c[f], e->n);
    }
    EIO_CUDA(cudaStreamSynchronize(e->st));
}

}  // namespace eio
