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
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "eio_internal.h"
#include "eio_kernels.cuh"
#include "eio_pair.cuh"
#include "eio_sweep.cuh"
#include "eio_tile.cuh"
#include "eio_wave.cuh"

namespace eio {

#define EIO_CUDA(x)                                                                                    \
    do {                                                                                               \
        cudaError_t e_ = (x);                                                                          \
        if (e_ != cudaSuccess)                                                                         \
            throw Error(EIO_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));               \
    } while (0)

// Bytes the library's growable buffers hold on the devices, and an optional
// cap on them (eio_set_device_memory_cap: 0 = none), so that an out-of-memory
// condition can be produced on purpose and its handling tested.
std::atomic<long long> g_dbuf_used{0};
std::atomic<long long> g_dbuf_cap{0};

// growable device buffer; where = 0 (the source history): device memory, or
// mapped pinned host memory reached through its device address when the
// device allocation does not fit; 1: device only; 2: host only
struct DBuf {
    void* p = nullptr;      // device address (the mapped alias for host memory)
    size_t cap = 0;
    bool host = false;
    void* hp = nullptr;     // host address of mapped memory
    void ensure(size_t bytes, int where = 1) {
        if (bytes <= cap && (where == 0 || host == (where == 2))) return;
        release();
        if (where != 2) {
            const long long lim = g_dbuf_cap.load();
            const bool capped = lim > 0 && g_dbuf_used.load() + (long long)bytes > lim;
            cudaError_t e = capped ? cudaErrorMemoryAllocation : cudaMalloc(&p, bytes);
            if (e == cudaSuccess) {
                cap = bytes;
                g_dbuf_used += (long long)bytes;
                return;
            }
            p = nullptr;
            if (!capped) cudaGetLastError();   // a failed allocation leaves no sticky error
            if (e != cudaErrorMemoryAllocation)
                throw Error(EIO_ERR_CUDA, std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
            if (where == 1)
                throw Error(EIO_ERR_NOMEM, std::string("cudaMalloc(") + std::to_string(bytes) + "): " +
                                               (capped ? "above the library's device-memory cap" : cudaGetErrorString(e)));
        }
        cudaError_t e = cudaHostAlloc(&hp, bytes, cudaHostAllocMapped | cudaHostAllocPortable);
        if (e != cudaSuccess) {
            hp = nullptr;
            cudaGetLastError();
            throw Error(EIO_ERR_NOMEM, std::string("neither device nor pinned host memory for ") + std::to_string(bytes) +
                                           " bytes: " + cudaGetErrorString(e));
        }
        void* dp = nullptr;
        e = cudaHostGetDevicePointer(&dp, hp, 0);
        if (e != cudaSuccess) {
            cudaFreeHost(hp);
            hp = nullptr;
            throw Error(EIO_ERR_CUDA, std::string("cudaHostGetDevicePointer: ") + cudaGetErrorString(e));
        }
        p = dp;
        host = true;
        cap = bytes;
    }
    void release() {
        if (host) {
            if (hp) cudaFreeHost(hp);
        } else if (p) {
            cudaFree(p);
            g_dbuf_used -= (long long)cap;
        }
        p = nullptr;
        hp = nullptr;
        host = false;
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
    const int* const* pos = nullptr;   // the position lists the buckets came from
    const int* npos = nullptr;
};

struct Engine {
    int device = 0;
    int nsm = 148;          // SM count of the device
    cudaStream_t st = nullptr;
    // Born imaging runs on a second, lower-priority stream, decoupled from the
    // step kernels by a ring of secondary-source slots and two events per slot
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_ready[4] = {}, ev_free[4] = {}, ev_sync = nullptr;
    int nz = 0, nx = 0;
    long long n = 0;
    int nts = 0, S = 0, ntw = 0, h = 0;
    float zc[4], xc[4];
    std::vector<float> filt;
    float dts_inv = 0.f;
    int ntz = 0, ntx = 0, ntiles = 0;
    int ckpt = 0;           // source-wavefield snapshots: 0 FP32, 1 BF16, 2 FP16 (scaled per snapshot)
    int hist_where = 0;     // source-wavefield history: 0 device, host when it does not fit; 1 device; 2 host
    DBuf Wq, wscale, wstage, wpmax;   // 16-bit history, scales [nts][2], FP32 staging row pair, warp maxima
    // wavefield levels: two sets of 5 slices for the single-step kernels, four
    // for the two-step kernel (it writes both new levels to the free sets)
    DBuf par[5], dampz, dampx, wf[20];
    // the engine whose medium arrays the kernels read (nullptr: its own).  The
    // shot lanes of a context read the first lane's copy, so that lanes running
    // at once share one medium in L2 instead of evicting each other's
    const Engine* med = nullptr;
    // free surface (nonlinear operators only, like the reference): taper
    // without the top edge, sigmaxx coefficient of the surface row per column
    int fs = 0;
    bool fs_active = false;   // set while a free-surface propagation runs (k_step only)
    // shot window: the propagations run on columns [win_ix0, win_ix0 + nx) of the
    // full_nx-column grid (one contiguous block of every [nx][nz] array)
    int full_nx = 0, win_ix0 = 0;
    bool windowed = false;
    std::vector<float> damp;  // taper table of the grid (minPad entries)
    int minPad = 0;
    DBuf dampx_w;
    DBuf dampz_fs, fsc;
    DBuf inj_ts, inj_ent, ext_ts, ext_ent;
    DBuf inj_hts, inj_hent;   // source lists of the widened tiles (two-step kernel)
    DBuf sig_in[5], sig_out[5];
    DBuf stage_a[5], stage_b[5], stage_c[5];
    DBuf W, ss[20];         // secondary-source ring: 4 slots x 5 fields
    DBuf wsave;             // saved wavefield of the *Wavefield operators
    // receiver interpolators of the current shot on the device (one per grid)
    struct DevInterp {
        DBuf slot, w, start, ent;
        int nIrreg = 0, nReg = 0, nft = 0;
    } rint[4];
    DBuf stage_d[5];        // irregular receiver traces [nIrreg][nts] per field
    bool w_clean = false;   // history zeroed and only written by single stores since
    // grid size (nz * nx) the history buffers were last cleared for: their FAT
    // frame is never written, so a new layout (another shot window) clears them
    long long w_n = -1, wq_n = -1, ws_n = -1;
    // step-kernel choice: kind 0 = shared-memory tile kernel (k_step),
    // kind 1 = TMA x-sweep (k_sweep) with strip height tz, chunk width cw and
    // cpr chunks per CTA, kind 2 = persistent TMA-pipelined tile kernel (k_tile),
    // kind 3 = k_step at 4 CTAs per SM, kind 4 = two threads per float4 (k_split),
    // kind 5 = two fine steps per launch (k_pair) with kind 3 for single steps
    int kind = 1, tz = 64, cw = 8, cpr = 8;
    bool tuned = false;
    // tensor maps of the sweep kernel (valid for mtz/mcw)
    int mtz = -1, mcw = -1;
    CUtensorMap mwf_halo[10], mwf_int[10], mpar_halo[5], mpar_int[5];
    // tensor maps of the TMA tile kernel (kind 2), valid for the buffers in tbase
    CUtensorMap twf_halo[10], twf_int[10], tpar_halo[5], tpar_int[5];
    const void* tbase[15] = {};
    int tile_ctas[2] = {0, 0};    // persistent k_tile grid per direction (0 = not yet queried)
    DBuf err;
    // persistent time loop (eio_wave.cuh) of the lockstep shot groups: on by
    // default; the per-step plan, modes, secondary-source samples and unit counters
    // phases of the Born shot groups run as persistent loops (bits: 1 source, 2 scattered, 4 adjoint);
    // 0 by default: measured slower than the per-step launches (eio_ctx_set_persistent)
    int use_wave = 0;
    DBuf wave_plan, wave_mode, wave_ssk, wave_done;
    int wave_ctas[8] = {};   // resident CTAs per k_wave instantiation (0 = not queried)
    // try_wait polls of a TMA pipeline wait in the sweep and tile kernels before
    // it gives up (error flag, drain, EIO_ERR_TIMEOUT); their drains keep DRAIN_LIMIT
    long long wait_limit = WAIT_LIMIT;
    // launch statistics (bench instrumentation)
    long long launches = 0, step_launches = 0, sampled = 0;
    long long step_cells = 0;   // cell updates of the single-step launches (a batch launch: all its shots)
    double step_ms = 0.0;
    long long pair_launches = 0, pair_sampled = 0;   // two-step launches (also counted in step_launches)
    double pair_ms = 0.0;
    bool stats = false;
    std::vector<cudaEvent_t> ev;
    std::vector<unsigned char> ev_pair;   // per event pair: 1 = a two-step launch
    size_t ev_used = 0;
    // CUDA graphs of the time loops, one per distinct launch signature (key)
    struct Graph {
        uint64_t key = 0;
        cudaGraphExec_t exec = nullptr;
        // what one replay adds to the counters
        long long launches = 0, step_launches = 0, sampled = 0, pair_launches = 0, pair_sampled = 0;
        std::vector<cudaEvent_t> ev;          // timing events its event-record nodes write
        std::vector<unsigned char> ev_pair;
        size_t nev = 0;
        bool pending = false;                 // replayed since its events were last read
        unsigned long long used = 0;
    };
    std::vector<Graph*> graphs;
    Graph* cap = nullptr;                     // graph being captured
    bool use_graphs = false;  // measured slower than PDL stream launches on B200: opt-in
    unsigned long long graph_clock = 0;
};

static void graph_free(Engine::Graph* g);

// medium array f (rhoxDtw, rhozDtw, lamb2MuDtw, lambDtw, muxzDtw) the kernels of e read
static float* mpar(const Engine* e, int f) { return (e->med ? e->med : e)->par[f].f(); }

// CUDA-event timing of every STATS_PERIOD-th launch of the fused step kernel
// (only when enabled); sampling keeps the event records out of most gaps.
constexpr long long STATS_PERIOD = 16;
// the two-step kernels need more than 48 KB of dynamic shared memory
static void open_pair_smem() {
    EIO_CUDA(cudaFuncSetAttribute(k_pair<0, EPI_NONE>, cudaFuncAttributeMaxDynamicSharedMemorySize, PAIR_SMEM));
    EIO_CUDA(cudaFuncSetAttribute(k_pair<1, EPI_NONE>, cudaFuncAttributeMaxDynamicSharedMemorySize, PAIR_SMEM));
    EIO_CUDA(cudaFuncSetAttribute(k_pair<0, EPI_TRI>, cudaFuncAttributeMaxDynamicSharedMemorySize, PAIR_SMEM));
    EIO_CUDA(cudaFuncSetAttribute(k_pair<1, EPI_TRI>, cudaFuncAttributeMaxDynamicSharedMemorySize, PAIR_SMEM));
    EIO_CUDA(cudaFuncSetAttribute(k_pair<0, EPI_INJ_SS>, cudaFuncAttributeMaxDynamicSharedMemorySize, PAIR_SMEM));
}

static void stats_flush(Engine* e) {
    bool pending = false;
    for (const Engine::Graph* g : e->graphs) pending = pending || g->pending;
    if (e->ev_used == 0 && !pending) return;
    if (!e->stats) {   // timing was switched off: drop what was recorded
        e->ev_used = 0;
        for (Engine::Graph* g : e->graphs) g->pending = false;
        return;
    }
    EIO_CUDA(cudaStreamSynchronize(e->st));
    auto read = [&](const std::vector<cudaEvent_t>& ev, const std::vector<unsigned char>& is_pair, size_t n) {
        for (size_t k = 0; k + 1 < n; k += 2) {
            float ms = 0.f;
            EIO_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            if (is_pair[k / 2]) e->pair_ms += ms;
            else e->step_ms += ms;
        }
    };
    read(e->ev, e->ev_pair, e->ev_used);
    e->ev_used = 0;
    for (Engine::Graph* g : e->graphs)
        if (g->pending) {
            read(g->ev, g->ev_pair, g->nev);
            g->pending = false;
        }
}
// pair: the launch the mark opens (or closes) is a two-step launch
static void stats_mark(Engine* e, bool pair = false) {
    if (!e->stats) return;
    if (e->cap) {   // capturing: the graph's own events (created before the capture)
        Engine::Graph* g = e->cap;
        if (g->nev < g->ev.size()) {
            g->ev_pair[g->nev / 2] = pair ? 1 : 0;
            // external: an event-record node that records the event at every replay (a plain
            // record inside a capture only orders the captured work)
            EIO_CUDA(cudaEventRecordWithFlags(g->ev[g->nev++], e->st, cudaEventRecordExternal));
        }
        return;
    }
    if (e->ev_used == e->ev.size()) {
        if (e->ev.size() >= 65536) stats_flush(e);
        else {
            const size_t grow = e->ev.empty() ? 4096 : e->ev.size();
            for (size_t i = 0; i < grow; i++) {
                cudaEvent_t x;
                EIO_CUDA(cudaEventCreate(&x));
                e->ev.push_back(x);
            }
            e->ev_pair.resize(e->ev.size() / 2);
        }
    }
    e->ev_pair[e->ev_used / 2] = pair ? 1 : 0;
    EIO_CUDA(cudaEventRecord(e->ev[e->ev_used++], e->st));
}

static void upload(DBuf& b, const void* h, size_t bytes, cudaStream_t st) {
    b.ensure(std::max<size_t>(bytes, 16));
    if (bytes) EIO_CUDA(cudaMemcpyAsync(b.p, h, bytes, cudaMemcpyHostToDevice, st));
}

void engine_set_medium(Engine* e, const FdParam& fd) {
    EIO_CUDA(cudaSetDevice(e->device));
    const int nz = fd.p.nz, nx = fd.p.nx;
    if (nz != e->nz || nx != e->full_nx) throw Error(EIO_ERR_ARG, "setBackground: grid size changed");
    engine_set_window(e, 0, 0);
    e->damp.assign(fd.damp.begin(), fd.damp.begin() + std::min<size_t>(fd.damp.size(), (size_t)std::max(fd.minPad, 0)));
    e->minPad = fd.minPad;
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
    e->fs = fd.p.surfaceCondition;
    if (e->fs) {
        std::vector<float> dzf(nz, 1.f);   // dampCosineEdge_freesurface, K:1223-1252: no top edge
        for (int iz = FAT; iz < nz - FAT; iz++) {
            const int d = nz - iz - 1 - FAT;
            if (d < fd.minPad) dzf[iz] = fd.damp[d];
        }
        upload(e->dampz_fs, dzf.data(), sizeof(float) * nz, e->st);
        upload(e->fsc, fd.fsc.data(), sizeof(float) * nx, e->st);
        EIO_CUDA(cudaStreamSynchronize(e->st));   // the host tables are locals
    }
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
        EIO_CUDA(cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, device));
        e->nz = fd.p.nz;
        e->nx = fd.p.nx;
        e->full_nx = e->nx;
        e->n = (long long)e->nz * e->nx;
        if ((e->nz - 2 * FAT) % 16 || (e->nx - 2 * FAT) % 16 || e->nz % 4)
            throw Error(EIO_ERR_QC, "nz-2*fat and nx-2*fat must be multiples of 16");
        e->ntz = (e->nz - 2 * FAT + TZ - 1) / TZ;
        e->ntx = (e->nx - 2 * FAT) / TX;
        e->ntiles = e->ntz * e->ntx;
        int lo = 0, hi = 0;
        EIO_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        EIO_CUDA(cudaStreamCreateWithPriority(&e->st, cudaStreamNonBlocking, hi));
        EIO_CUDA(cudaStreamCreateWithPriority(&e->st2, cudaStreamNonBlocking, lo));
        for (int k = 0; k < 4; k++) {
            EIO_CUDA(cudaEventCreateWithFlags(&e->ev_ready[k], cudaEventDisableTiming));
            EIO_CUDA(cudaEventCreateWithFlags(&e->ev_free[k], cudaEventDisableTiming));
        }
        EIO_CUDA(cudaEventCreateWithFlags(&e->ev_sync, cudaEventDisableTiming));
        open_pair_smem();
        for (int f = 0; f < 20; f++) {
            e->wf[f].ensure(sizeof(float) * e->n);
            EIO_CUDA(cudaMemsetAsync(e->wf[f].p, 0, sizeof(float) * e->n, e->st));
        }
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
    if (e->st2) cudaStreamSynchronize(e->st2);
    DBuf* all[] = {&e->dampz, &e->dampx, &e->inj_ts, &e->inj_ent, &e->inj_hts, &e->inj_hent, &e->ext_ts, &e->ext_ent,
                   &e->W, &e->err, &e->wsave,
                   &e->Wq, &e->wscale, &e->wstage, &e->wpmax, &e->dampz_fs, &e->fsc, &e->dampx_w};
    for (DBuf* b : all) b->release();
    for (int k = 0; k < 4; k++) {
        e->rint[k].slot.release(); e->rint[k].w.release(); e->rint[k].start.release(); e->rint[k].ent.release();
    }
    for (int f = 0; f < 5; f++) {
        e->stage_d[f].release();
        e->par[f].release(); e->sig_in[f].release(); e->sig_out[f].release();
        e->stage_a[f].release(); e->stage_b[f].release(); e->stage_c[f].release();
    }
    for (int f = 0; f < 20; f++) e->wf[f].release();
    for (int f = 0; f < 20; f++) e->ss[f].release();
    for (cudaEvent_t x : e->ev) cudaEventDestroy(x);
    for (Engine::Graph* g : e->graphs) graph_free(g);
    e->graphs.clear();
    for (int k = 0; k < 4; k++) {
        if (e->ev_ready[k]) cudaEventDestroy(e->ev_ready[k]);
        if (e->ev_free[k]) cudaEventDestroy(e->ev_free[k]);
    }
    if (e->ev_sync) cudaEventDestroy(e->ev_sync);
    if (e->st2) cudaStreamDestroy(e->st2);
    if (e->st) cudaStreamDestroy(e->st);
    delete e;
}

void engine_set_checkpoint(Engine* e, int mode) {
    if (mode < 0 || mode > 2) throw Error(EIO_ERR_ARG, "checkpoint precision must be 0 (FP32), 1 (BF16) or 2 (FP16)");
    e->ckpt = mode;
}

void* engine_stream(Engine* e) { return (void*)e->st; }

// step_launches / step_ms cover every step-kernel launch (single- and two-step),
// pair_launches / pair_ms the two-step ones alone; times are sampled means x counts
void engine_stats(Engine* e, int enable, int reset, long long* launches, long long* step_launches, double* step_ms,
                  long long* pair_launches, double* pair_ms) {
    stats_flush(e);
    const double single = e->sampled ? e->step_ms * (double)e->step_launches / (double)e->sampled : 0.0;
    const double pair = e->pair_sampled ? e->pair_ms * (double)e->pair_launches / (double)e->pair_sampled : 0.0;
    if (launches) *launches = e->launches;
    if (step_launches) *step_launches = e->step_launches + e->pair_launches;
    if (step_ms) *step_ms = single + pair;
    if (pair_launches) *pair_launches = e->pair_launches;
    if (pair_ms) *pair_ms = pair;
    if (reset) {
        e->launches = 0; e->step_launches = 0; e->sampled = 0; e->step_ms = 0.0;
        e->pair_launches = 0; e->pair_sampled = 0; e->pair_ms = 0.0; e->step_cells = 0;
    }
    if (enable >= 0) e->stats = enable != 0;
}
long long engine_step_cells(const Engine* e) { return e->step_cells; }
// the Born operators ignore the free surface (like the reference's Born drivers)
bool engine_batchable(const Engine* e) { return e->S == 2 && e->ckpt == 0; }

// every kind but the sweep (1) uses the 64x16 tiles of k_step and their numbering
static bool tiled(int kind) { return kind != 1; }
// the free surface is built into k_step only; the TMA kernels' tensor maps
// cover the whole grid, so a shot window runs them as kind 3
static int eff_kind(const Engine* e) {
    if (e->fs_active) return 0;
    if (e->windowed && (e->kind == 1 || e->kind == 2)) return 3;
    return e->kind;
}

// tile geometry the sparse point lists are bucketed with
struct TileGeom {
    int tz, tx, ntz;
};
static TileGeom tile_geom(const Engine* e) {
    if (tiled(eff_kind(e))) return {TZ, TX, e->ntz};
    return {e->tz, e->cw, (e->nz - 2 * FAT + e->tz - 1) / e->tz};
}

// CSR of (tile, entry) pairs, entries of a tile in their original order
static void bucket(const std::vector<std::pair<int, PointEntry>>& tmp, int ntiles, PointList& pl) {
    pl.any = !tmp.empty();
    pl.tile_start.assign(ntiles + 1, 0);
    for (auto& t : tmp) pl.tile_start[t.first + 1]++;
    for (int i = 0; i < ntiles; i++) pl.tile_start[i + 1] += pl.tile_start[i];
    pl.ent.resize(tmp.size());
    std::vector<int> cur(pl.tile_start.begin(), pl.tile_start.end() - 1);
    for (auto& t : tmp) pl.ent[cur[t.first]++] = t.second;
}

// Sort the points of the four position lists into per-tile buckets.
static void build_points(const Engine* e, const int* const pos[4], const int npos[4], PointList& pl) {
    pl.pos = pos;
    pl.npos = npos;
    const TileGeom tg = tile_geom(e);
    const int nchunks = (e->nx - 2 * FAT) / tg.tx;
    const int ntiles = tg.ntz * nchunks;
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
            const int bz = (iz - FAT) / tg.tz, bx = (ix - FAT) / tg.tx;
            PointEntry pe;
            pe.key = (f << 16) | (((ix - FAT) % tg.tx) << 8) | ((iz - FAT) % tg.tz);
            pe.col = k;
            // k_step / k_tile number tiles z-fastest, k_sweep strip-major
            tmp.push_back({tiled(eff_kind(e)) ? bx * tg.ntz + bz : bz * nchunks + bx, pe});
        }
    }
    bucket(tmp, ntiles, pl);
}

// Sources of the widened tiles of the two-step kernel (k_pair): a point joins
// the list of every tile whose widened tile (the tile plus the 4-cell stencil
// radius) holds it, keyed from the widened tile's corner.  Bounds are checked
// by build_points.
static void build_halo_points(const Engine* e, const int* const pos[4], const int npos[4], PointList& pl) {
    std::vector<std::pair<int, PointEntry>> tmp;
    for (int f = 0; f < 5; f++) {
        const int g = kFieldGrid[f];
        pl.ld[f] = npos[g];
        for (int k = 0; k < npos[g]; k++) {
            const int cell = pos[g][k];
            const int ix = cell / e->nz, iz = cell % e->nz;
            const int bz0 = (iz - FAT) / TZ, bx0 = (ix - FAT) / TX;
            for (int bz = std::max(bz0 - 1, 0); bz <= std::min(bz0 + 1, e->ntz - 1); bz++)
                for (int bx = std::max(bx0 - 1, 0); bx <= std::min(bx0 + 1, e->ntx - 1); bx++) {
                    const int lz = iz - bz * TZ, lx = ix - bx * TX;   // corner (FAT + bz*TZ - FAT, ...)
                    if (lz < 0 || lz >= SZ || lx < 0 || lx >= SX) continue;
                    PointEntry pe;
                    pe.key = (f << 16) | (lx << 8) | lz;
                    pe.col = k;
                    tmp.push_back({bx * e->ntz + bz, pe});
                }
        }
    }
    bucket(tmp, e->ntiles, pl);
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
    const long long off = (long long)e->win_ix0 * e->nz;   // shot window
    for (int f = 0; f < 5; f++) a.par[f] = mpar(e, f) + off;
    a.dampz = e->fs_active ? e->dampz_fs.f() : e->dampz.f();
    a.dampx = e->windowed ? e->dampx_w.f() : e->dampx.f();
    a.fs = e->fs_active ? 1 : 0;
    a.fsc = e->fsc.f() ? e->fsc.f() + e->win_ix0 : nullptr;
    a.nz = e->nz;
    a.nx = e->nx;
    a.ntz = e->ntz;
    for (int i = 0; i < 4; i++) { a.cz[i] = e->zc[i]; a.cx[i] = e->xc[i]; }
    a.wstride = e->n;
    return a;
}

// ---------------------------------------------------------------- step launch
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        EIO_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess) throw Error(EIO_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 2-D map of one [nx][nz] float field (z innermost) with a box of bz rows x bx columns
static CUtensorMap make_map(const float* base, int nz, int nx, int bz, int bx) {
    CUtensorMap m;
    cuuint64_t dims[2] = {(cuuint64_t)nz, (cuuint64_t)nx};
    cuuint64_t strides[1] = {(cuuint64_t)nz * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)bz, (cuuint32_t)bx};
    cuuint32_t es[2] = {1, 1};
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, es,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(EIO_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

static void ensure_maps(Engine* e) {
    if (e->mtz == e->tz && e->mcw == e->cw) return;
    for (int b = 0; b < 10; b++) {
        e->mwf_halo[b] = make_map(e->wf[b].f(), e->nz, e->nx, e->tz + 2 * FAT, e->cw);
        e->mwf_int[b] = make_map(e->wf[b].f(), e->nz, e->nx, e->tz, e->cw);
    }
    for (int f = 0; f < 5; f++) {
        e->mpar_halo[f] = make_map(mpar(e, f), e->nz, e->nx, e->tz + 2 * FAT, e->cw);
        e->mpar_int[f] = make_map(mpar(e, f), e->nz, e->nx, e->tz, e->cw);
    }
    e->mtz = e->tz;
    e->mcw = e->cw;
}

template <int DIR, int EPI, int TZ, int CW>
static void launch_sweep_t(Engine* e, const SweepArgs& s, int nblocks) {
    using Ly = SweepLayout<TZ, CW, DIR>;
    static bool attr = false;
    if (!attr) {
        EIO_CUDA(cudaFuncSetAttribute(k_sweep<DIR, EPI, TZ, CW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)Ly::BYTES));
        attr = true;
    }
    k_sweep<DIR, EPI, TZ, CW><<<nblocks, Ly::NT, Ly::BYTES, e->st>>>(s);
}

template <int DIR, int EPI>
static void launch_sweep(Engine* e, const StepArgs& a, int cur) {
    ensure_maps(e);
    SweepArgs s;
    memset(&s, 0, sizeof(s));
    const int oc = cur * 5, cc = (1 - cur) * 5;   // buffer of the old / current level
    for (int f = 0; f < 5; f++) {
        s.tc[f] = e->mwf_halo[cc + f];
        s.to[f] = e->mwf_int[oc + f];
        s.tp[f] = DIR == 0 ? e->mpar_int[f] : e->mpar_halo[f];
        s.o[f] = a.o[f];
        s.ssL[f] = a.ssL[f]; s.ssR[f] = a.ssR[f]; s.eL[f] = a.eL[f]; s.eR[f] = a.eR[f];
    }
    s.dampz = a.dampz; s.dampx = a.dampx;
    s.nz = e->nz; s.nx = e->nx;
    s.nstrips = (e->nz - 2 * FAT + e->tz - 1) / e->tz;
    s.nchunks = (e->nx - 2 * FAT) / e->cw;
    s.cpr = std::max(1, std::min(std::min(e->cpr, s.nchunks), SWEEP_MAXK));
    s.nranges = (s.nchunks + s.cpr - 1) / s.cpr;
    for (int i = 0; i < 4; i++) { s.cz[i] = a.cz[i]; s.cx[i] = a.cx[i]; }
    s.inj = a.inj; s.ext = a.ext;
    // the sweep kernel buckets points per (strip, chunk): rebuilt by the caller
    s.W0 = a.W0; s.W1 = a.W1; s.wstride = a.wstride; s.wt = a.wt; s.ww0 = a.ww0; s.ww1 = a.ww1;
    s.sw0 = a.sw0; s.sw1 = a.sw1;
    s.tmode = a.tmode; s.tw_o = a.tw_o; s.tw_c = a.tw_c; s.tw_n = a.tw_n;
    for (int f = 0; f < 5; f++) s.c[f] = a.c[f];
    s.err = static_cast<int*>(e->err.p);
    s.wait_limit = e->wait_limit;
    const int nb = s.nstrips * s.nranges;
    if (e->tz == 64 && e->cw == 8) launch_sweep_t<DIR, EPI, 64, 8>(e, s, nb);
    else if (e->tz == 64 && e->cw == 16) launch_sweep_t<DIR, EPI, 64, 16>(e, s, nb);
    else if (e->tz == 128 && e->cw == 8) launch_sweep_t<DIR, EPI, 128, 8>(e, s, nb);
    else throw Error(EIO_ERR_ARG, "unsupported sweep configuration");
}

static void ensure_tile_maps(Engine* e) {
    bool same = true;
    for (int b = 0; b < 10; b++) same = same && e->tbase[b] == e->wf[b].p;
    for (int f = 0; f < 5; f++) same = same && e->tbase[10 + f] == mpar(e, f);
    if (same) return;
    for (int b = 0; b < 10; b++) {
        e->twf_halo[b] = make_map(e->wf[b].f(), e->nz, e->nx, SZ, SX);
        e->twf_int[b] = make_map(e->wf[b].f(), e->nz, e->nx, TZ, TX);
        e->tbase[b] = e->wf[b].p;
    }
    for (int f = 0; f < 5; f++) {
        e->tpar_halo[f] = make_map(mpar(e, f), e->nz, e->nx, SZ, SX);
        e->tpar_int[f] = make_map(mpar(e, f), e->nz, e->nx, TZ, TX);
        e->tbase[10 + f] = mpar(e, f);
    }
}

template <int DIR, int EPI>
static void launch_tile(Engine* e, const StepArgs& a, int cur) {
    ensure_tile_maps(e);
    static unsigned attr_done = 0;          // one bit per device
    const unsigned bit = 1u << (e->device & 31);
    if (!(attr_done & bit)) {
        EIO_CUDA(cudaFuncSetAttribute(k_tile<DIR, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)TileLayout<DIR>::BYTES));
        EIO_CUDA(cudaFuncSetAttribute(k_tile<DIR, EPI>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        attr_done |= bit;
    }
    if (!e->tile_ctas[DIR]) {
        int per_sm = 0;
        EIO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile<DIR, EPI>, NT,
                                                               TileLayout<DIR>::BYTES));
        if (per_sm < 1) throw Error(EIO_ERR_CUDA, "the TMA tile kernel does not fit on an SM");
        e->tile_ctas[DIR] = per_sm * e->nsm;
    }
    TileArgs t;
    memset(&t, 0, sizeof(t));
    const int oc = cur * 5, cc = (1 - cur) * 5;   // buffer of the old / current level
    for (int f = 0; f < 5; f++) {
        t.tc[f] = e->twf_halo[cc + f];
        t.to[f] = e->twf_int[oc + f];
        t.tp[f] = DIR == 0 ? e->tpar_int[f] : e->tpar_halo[f];
    }
    t.s = a;
    t.ntiles = e->ntiles;
    t.err = static_cast<int*>(e->err.p);
    t.wait_limit = e->wait_limit;
    const int grid = std::min(e->ntiles, e->tile_ctas[DIR]);
    k_tile<DIR, EPI><<<grid, NT, TileLayout<DIR>::BYTES, e->st>>>(t);
}

// step kernels go out with programmatic stream serialization (see pdl_begin)
template <typename K>
static void launch_pdl(K kern, int grid, int block, cudaStream_t st, const StepArgs& a) {
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    EIO_CUDA(cudaLaunchKernelEx(&cfg, kern, a));
}

template <int DIR, int EPI>
static void launch_step(Engine* e, StepArgs& a, int cur) {
    const bool timed = e->stats && (e->step_launches + e->pair_launches) % STATS_PERIOD == 0;
    if (timed) stats_mark(e);
    if constexpr (EPI >= EPI_TRI_IMG) {   // the fused imaging condition is built into k_step only
        // 3 CTAs per SM; 2 for the 16-bit histories, whose decoding would spill at 80 registers
        launch_pdl(k_step<DIR, EPI, EPI == EPI_TRI_IMG ? 3 : 2>, e->ntiles, NT, e->st, a);
    } else {
        const int kind = eff_kind(e);
        bool done = false;
        if constexpr (EPI == EPI_NONE) {   // the nonlinear operators are the only ones with a free surface
            if (e->fs_active) {
                launch_pdl(k_step<DIR, EPI, 3, true>, e->ntiles, NT, e->st, a);
                done = true;
            }
        }
        if (done) {
        } else if (kind == 0) launch_pdl(k_step<DIR, EPI, 3>, e->ntiles, NT, e->st, a);
        else if (kind == 2) launch_tile<DIR, EPI>(e, a, cur);
        else if (kind == 3 || kind == 5) launch_pdl(k_step<DIR, EPI, 4>, e->ntiles, NT, e->st, a);
        else if (kind == 4) launch_pdl(k_split<DIR, EPI>, e->ntiles, NT2, e->st, a);
        else launch_sweep<DIR, EPI>(e, a, cur);
    }
    if (timed) {
        stats_mark(e);
        e->sampled++;
    }
    e->launches++;
    e->step_launches++;
    e->step_cells += (long long)(e->nz - 2 * FAT) * (e->nx - 2 * FAT);
}

// two fine steps in one launch (kind 5); the dynamic shared memory of each
// instantiation is opened when the context is created (open_pair_smem)
template <int DIR, int EPI>
static void launch_pair(Engine* e, const PairArgs& p) {
    static_assert(sizeof(PairArgs) <= 4096, "kernel parameter block");
    const bool timed = e->stats && (e->step_launches + e->pair_launches) % STATS_PERIOD == 0;
    if (timed) stats_mark(e, true);
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(e->ntiles);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = PAIR_SMEM;
    cfg.stream = e->st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    EIO_CUDA(cudaLaunchKernelEx(&cfg, k_pair<DIR, EPI>, p));
    if (timed) {
        stats_mark(e, true);
        e->pair_sampled++;
    }
    e->launches++;
    e->pair_launches++;
}

// Wavefield levels of a propagation: o and c of the next step, and the two
// free sets that a two-step launch writes its new levels to.
struct Levels {
    float* o[5]; float* c[5]; float* f0[5]; float* f1[5];
    explicit Levels(Engine* e) {
        for (int f = 0; f < 5; f++) {
            o[f] = e->wf[f].f(); c[f] = e->wf[5 + f].f(); f0[f] = e->wf[10 + f].f(); f1[f] = e->wf[15 + f].f();
        }
    }
    void set(StepArgs& a) const {
        for (int f = 0; f < 5; f++) { a.o[f] = o[f]; a.c[f] = c[f]; }
    }
    void single() { std::swap(o, c); }                       // the new level replaced o
    void pair() { std::swap(o, f0); std::swap(c, f1); }      // o, c = the two new levels
};

// one two-step launch: a0, a1 carry the per-step parameters of steps t+1 and
// t+2 (a0.inj the time weights of step A); injh = the widened-tile source lists
template <int DIR, int EPI>
static void run_pair(Engine* e, StepArgs a0, StepArgs a1, const SparseOp& injh, Levels& L) {
    PairArgs p;
    for (int f = 0; f < 5; f++) {
        a0.o[f] = L.o[f]; a0.c[f] = L.c[f];
        a1.o[f] = L.f1[f]; a1.c[f] = L.f0[f];
        p.n1[f] = L.f0[f];
    }
    SparseOp hi = injh;
    hi.t0 = a0.inj.t0; hi.w0 = a0.inj.w0; hi.w1 = a0.inj.w1;
    a0.inj = hi;
    p.s[0] = a0;
    p.s[1] = a1;
    launch_pair<DIR, EPI>(e, p);
    L.pair();
}

// ---------------------------------------------------------------- CUDA graphs
// FNV-1a over the values that fix a time loop's launch sequence (kernel
// arguments, buffer addresses, step counts, the kernel choice)
struct LoopKey {
    uint64_t h = 1469598103934665603ull;
    void add(const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ull; }
    }
    template <class T> LoopKey& operator<<(const T& v) { add(&v, sizeof(v)); return *this; }
};

static LoopKey loop_key(const Engine* e, int loop) {
    LoopKey k;
    k << loop << e->kind << e->tz << e->cw << e->cpr << e->fs_active << e->nts << e->S << e->ckpt << e->stats;
    k.add(e->filt.data(), sizeof(float) * e->filt.size());
    for (int f = 0; f < 20; f++) k << e->wf[f].p;
    return k;
}

static void graph_free(Engine::Graph* g) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    for (cudaEvent_t x : g->ev) cudaEventDestroy(x);
    delete g;
}

constexpr size_t MAX_GRAPHS = 8;

// Run one time loop (body issues its launches on e->st, and on e->st2 after
// joining it through an event) as a CUDA graph: captured the first time its key
// is seen, replayed afterwards.  max_steps bounds the step launches (sizes the
// graph's timing events).  Falls back to direct launches if capture fails.
template <class Body>
static void run_graph(Engine* e, uint64_t key, long long max_steps, Body&& body) {
    if (!e->use_graphs) {
        body();
        return;
    }
    Engine::Graph* g = nullptr;
    for (Engine::Graph* x : e->graphs)
        if (x->key == key) g = x;
    if (!g) {
        g = new Engine::Graph();
        g->key = key;
        try {
            if (e->stats) {
                const size_t nev = 2 * (size_t)(max_steps / STATS_PERIOD + 2);
                for (size_t i = 0; i < nev; i++) {
                    cudaEvent_t x;
                    EIO_CUDA(cudaEventCreate(&x));
                    g->ev.push_back(x);
                }
                g->ev_pair.assign(nev / 2, 0);
            }
        } catch (...) {
            graph_free(g);
            throw;
        }
        const long long l0 = e->launches, s0 = e->step_launches, m0 = e->sampled, p0 = e->pair_launches,
                        q0 = e->pair_sampled;
        cudaError_t err = cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) {
            e->cap = g;
            bool failed = false;
            try {
                body();
            } catch (const Error& x) {
                if (x.code != EIO_ERR_CUDA) {
                    e->cap = nullptr;
                    cudaGraph_t gr = nullptr;
                    cudaStreamEndCapture(e->st, &gr);
                    if (gr) cudaGraphDestroy(gr);
                    e->launches = l0; e->step_launches = s0; e->sampled = m0; e->pair_launches = p0;
                    e->pair_sampled = q0;
                    graph_free(g);
                    throw;
                }
                failed = true;   // a call the capture does not take: direct launches below
            }
            if (failed) {
                e->cap = nullptr;
                cudaGraph_t gr = nullptr;
                cudaStreamEndCapture(e->st, &gr);
                if (gr) cudaGraphDestroy(gr);
                cudaGetLastError();
                e->launches = l0; e->step_launches = s0; e->sampled = m0; e->pair_launches = p0; e->pair_sampled = q0;
                graph_free(g);
                e->use_graphs = false;
                body();   // every level set is still zero, so the body may start from any of them
                return;
            }
            e->cap = nullptr;
            cudaGraph_t gr = nullptr;
            err = cudaStreamEndCapture(e->st, &gr);
            if (err == cudaSuccess) err = cudaGraphInstantiate(&g->exec, gr, 0);
            if (gr) cudaGraphDestroy(gr);
        }
        g->launches = e->launches - l0; g->step_launches = e->step_launches - s0; g->sampled = e->sampled - m0;
        g->pair_launches = e->pair_launches - p0; g->pair_sampled = e->pair_sampled - q0;
        e->launches = l0; e->step_launches = s0; e->sampled = m0; e->pair_launches = p0; e->pair_sampled = q0;
        if (err != cudaSuccess) {   // no graphs on this device / driver: launch directly from now on
            cudaGetLastError();
            graph_free(g);
            e->use_graphs = false;
            body();
            return;
        }
        if (e->graphs.size() >= MAX_GRAPHS) {
            size_t old = 0;
            for (size_t i = 1; i < e->graphs.size(); i++)
                if (e->graphs[i]->used < e->graphs[old]->used) old = i;
            stats_flush(e);
            graph_free(e->graphs[old]);
            e->graphs.erase(e->graphs.begin() + old);
        }
        e->graphs.push_back(g);
    }
    if (g->pending) stats_flush(e);   // its events still hold the previous replay
    EIO_CUDA(cudaGraphLaunch(g->exec, e->st));
    g->used = ++e->graph_clock;
    e->launches += g->launches; e->step_launches += g->step_launches; e->sampled += g->sampled;
    e->pair_launches += g->pair_launches; e->pair_sampled += g->pair_sampled;
    g->pending = e->stats && g->nev > 0;
}

// the widened-tile source lists of a propagation (two-step kernel only)
static SparseOp halo_sources(Engine* e, bool use_pair, const int* const pos[4], const int npos[4], DBuf* sig) {
    SparseOp op;
    memset(&op, 0, sizeof(op));
    if (!use_pair) return op;
    PointList pl;
    build_halo_points(e, pos, npos, pl);
    return upload_points(e, pl, e->inj_hts, e->inj_hent, sig);
}

// ---------------------------------------------------------------- autotuner
struct KernelCfg {
    int kind, tz, cw, cpr;
};
static const KernelCfg kCandidates[] = {
    {0, TZ, TX, 0},
    {5, TZ, TX, 0},
    {2, TZ, TX, 0},
    {3, TZ, TX, 0},
    {4, TZ, TX, 0},
    {1, 64, 8, 4}, {1, 64, 8, 8}, {1, 64, 8, 16}, {1, 64, 8, 32},
    {1, 64, 16, 2}, {1, 64, 16, 4}, {1, 64, 16, 8},
    {1, 128, 8, 4}, {1, 128, 8, 8}, {1, 128, 8, 16},
};

static bool cfg_valid(const Engine* e, const KernelCfg& c) {
    if (tiled(c.kind)) return true;
    return (e->nx - 2 * FAT) % c.cw == 0;
}

void engine_set_kernel(Engine* e, int kind, int tz, int cw, int cpr) {
    KernelCfg c{kind, tz, cw, cpr};
    bool known = false;
    for (const KernelCfg& k : kCandidates)
        if (k.kind == c.kind && (tiled(c.kind) || (k.tz == c.tz && k.cw == c.cw))) known = true;
    if (!known || !cfg_valid(e, c) || (kind == 1 && (cpr < 1 || cpr > SWEEP_MAXK))) throw Error(EIO_ERR_ARG, "unsupported kernel configuration");
    e->kind = kind;
    if (kind == 1) { e->tz = tz; e->cw = cw; e->cpr = cpr; }
    e->tuned = true;
}

// Columns [ix0, ix0 + nxw) of the grid as the grid of the next propagations
// (nxw = 0: the whole grid).  The window keeps the grid's taper table: its
// first and last FAT columns are the frozen frame and the taper runs from its
// own edges.  The medium, the Born perturbation and the gradient are the
// grid's arrays offset by ix0 * nz; wavefield levels use the first nz * nxw
// values of their buffers.
void engine_set_window(Engine* e, int ix0, int nxw) {
    if (nxw == 0) { ix0 = 0; nxw = e->full_nx; }
    if (ix0 < 0 || nxw < 2 * FAT + 16 || (nxw - 2 * FAT) % 16 || ix0 + nxw > e->full_nx)
        throw Error(EIO_ERR_ARG, "shot window [" + std::to_string(ix0) + ", " + std::to_string(ix0 + nxw) +
                                     ") must lie in the grid and hold 2*fat + a multiple of 16 columns");
    if (ix0 == e->win_ix0 && nxw == e->nx) return;
    EIO_CUDA(cudaSetDevice(e->device));
    e->win_ix0 = ix0;
    e->nx = nxw;
    e->n = (long long)e->nz * nxw;
    e->ntx = (nxw - 2 * FAT) / TX;
    e->ntiles = e->ntz * e->ntx;
    e->windowed = !(ix0 == 0 && nxw == e->full_nx);
    if (e->windowed) {
        std::vector<float> dx(nxw, 1.f);
        for (int ix = FAT; ix < nxw - FAT; ix++) {
            const int d = std::min(ix - FAT, nxw - ix - 1 - FAT);
            if (d < e->minPad && d < (int)e->damp.size()) dx[ix] = e->damp[d];
        }
        upload(e->dampx_w, dx.data(), sizeof(float) * nxw, e->st);
        EIO_CUDA(cudaStreamSynchronize(e->st));   // dx is a local
    }
}

int engine_window_ix0(const Engine* e) { return e->win_ix0; }

void engine_set_graphs(Engine* e, int enable) {
    stats_flush(e);
    e->use_graphs = enable != 0;
}

void engine_get_kernel(const Engine* e, int* kind, int* tz, int* cw, int* cpr) {
    if (kind) *kind = e->kind;
    if (tz) *tz = tiled(e->kind) ? TZ : e->tz;
    if (cw) *cw = tiled(e->kind) ? TX : e->cw;
    if (cpr) *cpr = tiled(e->kind) ? 0 : e->cpr;
}

static void zero_wavefields(Engine* e);

// Times every candidate on a few forward and adjoint fine steps of this grid
// (no sparse points; the step cost does not depend on the field values) and
// keeps the fastest.
void engine_autotune(Engine* e) {
    EIO_CUDA(cudaSetDevice(e->device));
    const bool stats = e->stats;
    e->stats = false;
    zero_wavefields(e);
    e->err.ensure(16);
    EIO_CUDA(cudaMemsetAsync(e->err.p, 0, sizeof(int), e->st));
    StepArgs a = base_args(e);
    cudaEvent_t t0, t1;
    EIO_CUDA(cudaEventCreate(&t0));
    EIO_CUDA(cudaEventCreate(&t1));
    float best = 1e30f;
    KernelCfg bestc = kCandidates[0];
    for (const KernelCfg& c : kCandidates) {
        if (!cfg_valid(e, c)) continue;
        e->kind = c.kind;
        if (c.kind == 1) { e->tz = c.tz; e->cw = c.cw; e->cpr = c.cpr; }
        float tot = 0.f;   // per fine step
        for (int dir = 0; dir < 2; dir++) {
            int cur = 0;
            const int reps = 12;
            Levels L(e);
            SparseOp none;
            memset(&none, 0, sizeof(none));
            for (int r = 0; r < reps + 3; r++) {
                if (r == 3) EIO_CUDA(cudaEventRecord(t0, e->st));
                if (c.kind == 5) {
                    if (dir == 0) run_pair<0, EPI_NONE>(e, a, a, none, L);
                    else run_pair<1, EPI_NONE>(e, a, a, none, L);
                    continue;
                }
                for (int f = 0; f < 5; f++) { a.o[f] = e->wf[cur * 5 + f].f(); a.c[f] = e->wf[(1 - cur) * 5 + f].f(); }
                if (dir == 0) launch_step<0, EPI_NONE>(e, a, cur);
                else launch_step<1, EPI_NONE>(e, a, cur);
                cur ^= 1;
            }
            EIO_CUDA(cudaEventRecord(t1, e->st));
            EIO_CUDA(cudaEventSynchronize(t1));
            float ms = 0.f;
            EIO_CUDA(cudaEventElapsedTime(&ms, t0, t1));
            tot += ms / (c.kind == 5 ? 2 * reps : reps);
        }
        if (tot < best) { best = tot; bestc = c; }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    e->launches = 0;
    e->step_launches = 0;
    e->pair_launches = 0;
    e->kind = bestc.kind;
    if (bestc.kind == 1) { e->tz = bestc.tz; e->cw = bestc.cw; e->cpr = bestc.cpr; }
    e->tuned = true;
    e->stats = stats;
    int flag = 0;
    EIO_CUDA(cudaMemcpy(&flag, e->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) throw Error(EIO_ERR_TIMEOUT, "a TMA pipeline wait timed out while tuning");
}

static void zero_wavefields(Engine* e) {
    for (int f = 0; f < 20; f++) EIO_CUDA(cudaMemsetAsync(e->wf[f].p, 0, sizeof(float) * e->n, e->st));
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

static void err_reset(Engine* e) {
    e->err.ensure(16);
    EIO_CUDA(cudaMemsetAsync(e->err.p, 0, sizeof(int), e->st));
}
static void err_check(Engine* e) {
    int flag = 0;
    EIO_CUDA(cudaMemcpy(&flag, e->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) throw Error(EIO_ERR_TIMEOUT, "a TMA pipeline wait timed out in the step kernel (output incomplete)");
}

void engine_set_wait_limit(Engine* e, long long polls) { e->wait_limit = polls < 0 ? WAIT_LIMIT : polls; }
void engine_share_medium(Engine* e, const Engine* from) {
    if (from == e) from = nullptr;
    if (from && (from->nz != e->nz || from->full_nx != e->full_nx || from->device != e->device))
        throw Error(EIO_ERR_ARG, "engines of different grids or devices cannot share a medium");
    e->med = from;
    memset(e->tbase, 0, sizeof(e->tbase));   // tensor maps of the TMA tile kernel are rebuilt
    e->mtz = -1;                             // ... and those of the sweep kernel
}
void engine_set_persistent(Engine* e, int mask) {
    if (mask < 0 || mask > 7) throw Error(EIO_ERR_ARG, "persistent-loop mask must be 0 .. 7");
    e->use_wave = mask;
}
int engine_get_persistent(const Engine* e) { return e->use_wave; }
long long engine_get_wait_limit(const Engine* e) { return e->wait_limit; }

// new level (in p) into coarse rows its, its+1 of the saved wavefield
static void save_wavefield(Engine* e, float* W, float* const p[5], int its, float w0, float w1) {
    SaveArgs s;
    for (int f = 0; f < 5; f++) s.p[f] = p[f];
    s.W = W; s.n = e->n; s.nz = e->nz; s.nx = e->nx; s.its = its; s.w0 = w0; s.w1 = w1;
    const int nq = (e->nz - 2 * FAT) / 4;
    dim3 g((nq + 127) / 128, e->nx - 2 * FAT);
    k_save_wavefield<<<g, 128, 0, e->st>>>(s);
    e->launches++;
}

static void fs_top(Engine* e, float* const c[5]) {
    k_fs_top<<<(e->nx - 2 * FAT + 127) / 128, 128, 0, e->st>>>(c[0], c[1], c[3], c[4], e->nz, e->nx);
    e->launches++;
}

// free-surface propagations run with the effective kind 0 while the guard lives
struct FsScope {
    Engine* e;
    explicit FsScope(Engine* en) : e(en) { e->fs_active = e->fs != 0; }
    ~FsScope() { e->fs_active = false; }
};

void engine_nl(Engine* e, int adj, float* const model[5], float* const data[5], const ShotGeom& g, float* wfld) {
    EIO_CUDA(cudaSetDevice(e->device));
    if (wfld && e->windowed) throw Error(EIO_ERR_UNSUPPORTED, "saved wavefields cover the whole grid: no shot windows");
    if (!e->tuned) engine_autotune(e);
    FsScope fs_scope(e);
    err_reset(e);
    PointList src, rec;
    build_points(e, g.srcPos, g.nSrc, src);
    build_points(e, g.recPos, g.nRec, rec);
    StepArgs a = base_args(e);
    zero_wavefields(e);
    Levels L(e);
    int cur = 0;   // buffer set holding the old level (TMA kernels)
    const float* F = e->filt.data();
    const int h = e->h;
    // two fine steps per launch unless a step needs work between the steps
    const bool use_pair = e->kind == 5 && !wfld && !e->fs_active;
    // the fine steps in propagation order: (its, it2)
    std::vector<std::pair<int, int>> steps;
    if (!adj) {
        for (int its = 0; its < e->nts - 1; its++)
            for (int it2 = 1; it2 < e->S + 1; it2++) steps.push_back({its, it2});
    } else {
        for (int its = e->nts - 2; its > -1; its--)
            for (int it2 = e->S - 1; it2 > -1; it2--) steps.push_back({its, it2});
    }
    // time weights of the sparse injection and extraction of one step
    auto weights = [&](StepArgs& x, int its, int it2) {
        const int ki = adj ? it2 + 1 : it2 - 1;
        x.inj.t0 = its; x.inj.w0 = F[ki]; x.inj.w1 = F[h + ki];
        x.ext.t0 = its; x.ext.w0 = F[it2]; x.ext.w1 = F[h + it2];
    };
    SparseOp injh;
    if (!adj) {
        stage_in(e, model, src.ld, e->nts, e->sig_in);
        zero_out(e, rec.ld, e->nts, e->sig_out);
        a.inj = upload_points(e, src, e->inj_ts, e->inj_ent, e->sig_in);
        a.ext = upload_points(e, rec, e->ext_ts, e->ext_ent, e->sig_out);
        injh = halo_sources(e, use_pair, g.srcPos, g.nSrc, e->sig_in);
    } else {
        stage_in(e, data, rec.ld, e->nts, e->sig_in);
        zero_out(e, src.ld, e->nts, e->sig_out);
        a.inj = upload_points(e, rec, e->inj_ts, e->inj_ent, e->sig_in);
        a.ext = upload_points(e, src, e->ext_ts, e->ext_ent, e->sig_out);
        injh = halo_sources(e, use_pair, g.recPos, g.nRec, e->sig_in);
    }
    LoopKey key = loop_key(e, 1);
    key << adj << wfld << use_pair;
    key.add(&a, sizeof(a));
    key.add(&injh, sizeof(injh));
    run_graph(e, key.h, (long long)steps.size(), [&] {
        for (size_t i = 0; i < steps.size();) {
            if (use_pair && i + 1 < steps.size()) {
                StepArgs a0 = a, a1 = a;
                weights(a0, steps[i].first, steps[i].second);
                weights(a1, steps[i + 1].first, steps[i + 1].second);
                if (!adj) run_pair<0, EPI_NONE>(e, a0, a1, injh, L);
                else run_pair<1, EPI_NONE>(e, a0, a1, injh, L);
                i += 2;
                continue;
            }
            const int its = steps[i].first, it2 = steps[i].second;
            L.set(a);
            weights(a, its, it2);
            if (!adj) {
                if (e->fs_active) fs_top(e, L.c);
                launch_step<0, EPI_NONE>(e, a, cur);
            } else {
                launch_step<1, EPI_NONE>(e, a, cur);
            }
            if (wfld) save_wavefield(e, wfld, L.o, its, F[it2], F[h + it2]);
            L.single();
            cur ^= 1;
            i++;
        }
    });
    check_launch();
    if (!adj) stage_out(e, rec.ld, e->nts, e->sig_out, data);
    else stage_out(e, src.ld, e->nts, e->sig_out, model);
    EIO_CUDA(cudaStreamSynchronize(e->st));
    stats_flush(e);
    err_check(e);
}

// the source-wavefield history of the current shot (FP32 or 16-bit codes)
static WHist whist(const Engine* e) {
    WHist h;
    memset(&h, 0, sizeof(h));
    if (e->ckpt) {
        const unsigned short* wq = static_cast<const unsigned short*>(e->Wq.p);
        h.Wvx = wq;
        h.Wvz = wq + (long long)e->nts * e->n;
        h.wscale = e->wscale.f();
    } else {
        h.Wvx = e->W.f();
        h.Wvz = e->W.f() + (long long)e->nts * e->n;
    }
    h.wstride = e->n;
    h.nts = e->nts;
    return h;
}

static void launch_imaging(Engine* e, int adj, int its, float* const dm[5], float* const ss[5],
                           cudaStream_t st) {
    ImagingArgs ia;
    memset(&ia, 0, sizeof(ia));
    ia.h = whist(e);
    ia.nz = e->nz; ia.nx = e->nx; ia.its = its;
    for (int i = 0; i < 4; i++) { ia.cz[i] = e->zc[i]; ia.cx[i] = e->xc[i]; }
    ia.dts_inv = e->dts_inv;
    for (int f = 0; f < 5; f++) { ia.dm[f] = dm[f]; ia.ss[f] = ss[f]; }
    const int ntiles = ((e->nz - 2 * FAT + TZ - 1) / TZ) * ((e->nx - 2 * FAT) / TX);
    switch (e->ckpt * 2 + adj) {
        case 0: k_imaging<0, 0><<<ntiles, NT, 0, st>>>(ia); break;
        case 1: k_imaging<1, 0><<<ntiles, NT, 0, st>>>(ia); break;
        case 2: k_imaging<0, 1><<<ntiles, NT, 0, st>>>(ia); break;
        case 3: k_imaging<1, 1><<<ntiles, NT, 0, st>>>(ia); break;
        case 4: k_imaging<0, 2><<<ntiles, NT, 0, st>>>(ia); break;
        default: k_imaging<1, 2><<<ntiles, NT, 0, st>>>(ia); break;
    }
    e->launches++;
}

// Source wavefield + coarse Vx/Vz history (BornElasticGpuFunctions.cu:746-768).
// The reference accumulates every fine step into rows its and its+1 of the
// history (interpWavefieldSingleComp, K:1337-1346).  With two fine steps per
// coarse sample (sub = 1) row its only ever receives the three fine samples
// that the step (its, it2 = 1) holds as its old, current and new level, so
// that step writes the row once (EPI_TRI, same operation order) and the other
// steps touch no history at all; other sub values keep the running sums.
// 16-bit checkpoints: the coarse sample the EPI_TRI step just wrote to the
// FP32 staging rows becomes row `row` of the 16-bit history
static void quantize_row(Engine* e, int row) {
    const int npart = e->ntiles * 16;
    float* pm = e->wpmax.f();
    QuantArgs q;
    q.stage[0] = e->wstage.f();
    q.stage[1] = e->wstage.f() + e->n;
    unsigned short* wq = static_cast<unsigned short*>(e->Wq.p);
    q.row[0] = wq + (long long)row * e->n;
    q.row[1] = wq + ((long long)e->nts + row) * e->n;
    q.scale = e->wscale.f() + 2 * row;
    q.pmax = pm + (size_t)(row & 1) * 2 * npart;
    q.pmax_next = pm + (size_t)((row + 1) & 1) * 2 * npart;
    q.npart = npart;
    q.nz = e->nz; q.nx = e->nx;
    const int grid = 2 * e->nsm;
    if (e->ckpt == 1) k_quantize<1><<<grid, 256, 0, e->st>>>(q);
    else k_quantize<2><<<grid, 256, 0, e->st>>>(q);
    e->launches++;
}

// Source wavefield with 16-bit snapshots (sub = 1 only): every coarse sample
// goes through the FP32 staging rows, its scale comes from the warp maxima the
// step leaves, and k_quantize stores the codes.  The tile kernels write the
// maxima, so the sweep kernel is not used here.
// Injection (and, for the nonlinear forward, extraction) time weights of the
// source-wavefield propagation at fine step (its, it2): the Born operators
// inject fine-time sources (row itw - 1), the nonlinear forward coarse traces
// with the filter weights and records its receivers (engine_nl_record).
struct SrcWeights {
    const Engine* e;
    bool nl;
    void operator()(StepArgs& x, int its, int it2) const {
        const float* F = e->filt.data();
        const int h = e->h;
        if (nl) {
            x.inj.t0 = its; x.inj.w0 = F[it2 - 1]; x.inj.w1 = F[h + it2 - 1];
            x.ext.t0 = its; x.ext.w0 = F[it2]; x.ext.w1 = F[h + it2];
        } else {
            x.inj.t0 = its * e->S + it2 - 1; x.inj.w0 = 1.f; x.inj.w1 = 0.f;
        }
    }
};

static void born_source_q(Engine* e, const PointList& src, StepArgs a, const SparseOp* ext) {
    if (e->S != 2)
        throw Error(EIO_ERR_UNSUPPORTED, "16-bit source-wavefield snapshots need sub = 1 (two fine steps per sample)");
    const size_t qbytes = sizeof(unsigned short) * 2 * (size_t)e->nts * e->n;
    if (e->Wq.cap < qbytes || e->wq_n != e->n) {
        e->Wq.ensure(qbytes, e->hist_where);
        EIO_CUDA(cudaMemsetAsync(e->Wq.p, 0, qbytes, e->st));   // the FAT frame is never written
        e->wq_n = e->n;
    }
    if (e->wstage.cap < sizeof(float) * 2 * (size_t)e->n || e->ws_n != e->n) {
        e->wstage.ensure(sizeof(float) * 2 * (size_t)e->n);
        EIO_CUDA(cudaMemsetAsync(e->wstage.p, 0, sizeof(float) * 2 * (size_t)e->n, e->st));
        e->ws_n = e->n;
    }
    e->wscale.ensure(sizeof(float) * 2 * (size_t)e->nts);
    const size_t pbytes = sizeof(float) * 2 * 2 * (size_t)e->ntiles * 16;
    e->wpmax.ensure(pbytes);
    EIO_CUDA(cudaMemsetAsync(e->wpmax.p, 0, pbytes, e->st));
    const int kind = e->kind;
    if (kind == 1) e->kind = 0;
    zero_wavefields(e);
    Levels L(e);
    int cur = 0;
    a.inj = upload_points(e, src, e->inj_ts, e->inj_ent, e->sig_in);
    const SparseOp injh = halo_sources(e, kind == 5, src.pos, src.npos, e->sig_in);
    if (ext) a.ext = *ext;
    else memset(&a.ext, 0, sizeof(a.ext));
    const SrcWeights weights{e, ext != nullptr};
    a.W0 = e->wstage.f();
    a.W1 = e->wstage.f() + e->n;
    a.wt = 0;
    const float* F = e->filt.data();
    const int h = e->h;
    const int npart = e->ntiles * 16;
    LoopKey key = loop_key(e, 2);
    key << e->Wq.p << e->wscale.p << e->wstage.p << e->wpmax.p << (ext != nullptr);
    key.add(&a, sizeof(a));
    key.add(&injh, sizeof(injh));
    try {
      run_graph(e, key.h, (long long)(e->nts - 1) * e->S, [&] {
        for (int its = 0; its < e->nts - 1; its++) {
            if (kind == 5 && its < e->nts - 2) {
                // (its, 1) samples row its, (its, 2) only steps; the staging rows
                // are quantized after the pair
                StepArgs a0 = a, a1 = a;
                weights(a0, its, 1);
                a0.tmode = 1; a0.wt = 0; a0.tw_o = F[h + 1]; a0.tw_c = F[h + 2]; a0.tw_n = F[1];
                a0.pmax = e->wpmax.f() + (size_t)(its & 1) * 2 * npart;
                weights(a1, its, 2);
                a1.tmode = 0; a1.pmax = nullptr;
                run_pair<0, EPI_TRI>(e, a0, a1, injh, L);
                quantize_row(e, its);
                continue;
            }
            for (int it2 = 1; it2 < e->S + 1; it2++) {
                L.set(a);
                weights(a, its, it2);
                const bool last = (its == e->nts - 2 && it2 == 2);
                int row = -1;
                if (it2 == 1) {
                    a.tmode = 1; row = its; a.tw_o = F[h + 1]; a.tw_c = F[h + 2]; a.tw_n = F[1];
                } else if (last) {
                    a.tmode = 2; row = its + 1; a.tw_o = 0.f; a.tw_c = F[h + 1]; a.tw_n = F[h + 2];
                }
                if (row >= 0) {
                    a.pmax = e->wpmax.f() + (size_t)(row & 1) * 2 * npart;
                    launch_step<0, EPI_TRI>(e, a, cur);
                    quantize_row(e, row);
                } else {
                    launch_step<0, EPI_NONE>(e, a, cur);
                }
                L.single();
                cur ^= 1;
            }
        }
      });
    } catch (...) {
        e->kind = kind;
        throw;
    }
    e->kind = kind;
    check_launch();
}

// ext: the receiver lists of the nonlinear forward (engine_nl_record), whose
// source traces are coarse; nullptr for the Born operators' fine-time sources
static void born_source(Engine* e, const PointList& src, StepArgs a, const SparseOp* ext = nullptr) {
    if (e->ckpt) {
        born_source_q(e, src, a, ext);
        return;
    }
    const size_t wbytes = sizeof(float) * 2 * (size_t)e->nts * e->n;
    const bool fresh = e->W.cap < wbytes;
    e->W.ensure(wbytes, e->hist_where);
    const bool tri = (e->S == 2);
    // running sums need a zeroed history; single writes only need the never
    // written FAT frame to be zero, which holds from the first clear on
    if (!tri || fresh || !e->w_clean || e->w_n != e->n) EIO_CUDA(cudaMemsetAsync(e->W.p, 0, wbytes, e->st));
    e->w_clean = tri;
    e->w_n = e->n;
    zero_wavefields(e);
    Levels L(e);
    int cur = 0;
    const bool use_pair = tri && e->kind == 5;
    a.inj = upload_points(e, src, e->inj_ts, e->inj_ent, e->sig_in);
    const SparseOp injh = halo_sources(e, use_pair, src.pos, src.npos, e->sig_in);
    if (ext) a.ext = *ext;
    else memset(&a.ext, 0, sizeof(a.ext));
    const SrcWeights weights{e, ext != nullptr};
    a.W0 = e->W.f();
    a.W1 = e->W.f() + (long long)e->nts * e->n;
    const float* F = e->filt.data();
    const int h = e->h;
    LoopKey key = loop_key(e, 3);
    key << tri << use_pair << (ext != nullptr);
    key.add(&a, sizeof(a));
    key.add(&injh, sizeof(injh));
    run_graph(e, key.h, (long long)(e->nts - 1) * e->S, [&] {
    for (int its = 0; its < e->nts - 1; its++) {
        if (use_pair && its < e->nts - 2) {
            // (its, 1) writes row its, (its, 2) only steps
            StepArgs a0 = a, a1 = a;
            weights(a0, its, 1);
            a0.tmode = 1; a0.wt = its; a0.tw_o = F[h + 1]; a0.tw_c = F[h + 2]; a0.tw_n = F[1];
            weights(a1, its, 2);
            a1.tmode = 0;
            run_pair<0, EPI_TRI>(e, a0, a1, injh, L);
            continue;
        }
        for (int it2 = 1; it2 < e->S + 1; it2++) {
            L.set(a);
            weights(a, its, it2);
            if (tri) {
                const bool last = (its == e->nts - 2 && it2 == 2);
                if (it2 == 1) {          // row its = o*f[h+1] + c*f[h+2] + n*f[1]
                    a.tmode = 1; a.wt = its; a.tw_o = F[h + 1]; a.tw_c = F[h + 2]; a.tw_n = F[1];
                    launch_step<0, EPI_TRI>(e, a, cur);
                } else if (last) {       // row nts-1 = c*f[h+1] + n*f[h+2]
                    a.tmode = 2; a.wt = its + 1; a.tw_o = 0.f; a.tw_c = F[h + 1]; a.tw_n = F[h + 2];
                    launch_step<0, EPI_TRI>(e, a, cur);
                } else {
                    launch_step<0, EPI_NONE>(e, a, cur);
                }
            } else {
                a.wt = its; a.ww0 = F[it2]; a.ww1 = F[h + it2];
                launch_step<0, EPI_SAVE_W>(e, a, cur);
            }
            L.single();
            cur ^= 1;
        }
    }
    });
    check_launch();
}

// Nonlinear forward of one shot that also leaves the coarse Vx/Vz history the
// Born operators build in their first phase (the source wavefield of the
// imaging condition), for an adjoint that follows with reuse_history.  The
// nonlinear operators inject the coarse traces with the time filter, the Born
// operators fine-time traces interpolated on the host from the same coarse
// traces: the two source wavefields agree to rounding.  model: regular coarse
// source traces [nReg][nts] per field (device); data: regular receiver traces
// (device), as engine_nl.  No free surface (the Born operators have none).
void engine_nl_record(Engine* e, float* const model[5], float* const data[5], const ShotGeom& g) {
    EIO_CUDA(cudaSetDevice(e->device));
    if (!e->tuned) engine_autotune(e);
    if (e->fs) throw Error(EIO_ERR_UNSUPPORTED, "the Born operators ignore the free surface: no shared history");
    err_reset(e);
    PointList src, rec;
    build_points(e, g.srcPos, g.nSrc, src);
    build_points(e, g.recPos, g.nRec, rec);
    StepArgs base = base_args(e);
    stage_in(e, model, src.ld, e->nts, e->sig_in);
    zero_out(e, rec.ld, e->nts, e->sig_out);
    const SparseOp ext = upload_points(e, rec, e->ext_ts, e->ext_ent, e->sig_out);
    born_source(e, src, base, &ext);
    stage_out(e, rec.ld, e->nts, e->sig_out, data);
    EIO_CUDA(cudaStreamSynchronize(e->st));
    stats_flush(e);
    err_check(e);
}

void engine_born(Engine* e, int adj, float* const srcDtw[5], float* const dm[5], float* const data[5],
                 const ShotGeom& g, bool reuse_history) {
    EIO_CUDA(cudaSetDevice(e->device));
    if (!e->tuned) engine_autotune(e);
    err_reset(e);
    PointList src, rec;
    build_points(e, g.srcPos, g.nSrc, src);
    build_points(e, g.recPos, g.nRec, rec);
    StepArgs base = base_args(e);
    const float* F = e->filt.data();
    const int h = e->h;
    // phase 1: source wavefield (kept from engine_nl_record when reuse_history)
    if (!reuse_history) {
        stage_in(e, srcDtw, src.ld, e->ntw, e->sig_in);
        born_source(e, src, base);
    }
    // phase 2
    constexpr int R = 4;                 // secondary-source ring slots
    float* ring[R][5];
    for (int k = 0; k < R; k++)
        for (int f = 0; f < 5; f++) {
            e->ss[k * 5 + f].ensure(sizeof(float) * e->n);
            ring[k][f] = e->ss[k * 5 + f].f();
        }
    for (int f = 0; f < 10; f++) EIO_CUDA(cudaMemsetAsync(e->ss[f].p, 0, sizeof(float) * e->n, e->st));
    zero_wavefields(e);
    // the imaging stream joins a time loop after everything queued before it
    // (history, model, clears) and the step stream waits for it at the end
    auto fork = [&] {
        EIO_CUDA(cudaEventRecord(e->ev_sync, e->st));
        EIO_CUDA(cudaStreamWaitEvent(e->st2, e->ev_sync, 0));
        for (int k = 0; k < R; k++) {       // no slot is in use at the start
            EIO_CUDA(cudaEventRecord(e->ev_free[k], e->st2));
            EIO_CUDA(cudaEventRecord(e->ev_ready[k], e->st2));
        }
    };
    auto join = [&] {
        EIO_CUDA(cudaEventRecord(e->ev_sync, e->st2));
        EIO_CUDA(cudaStreamWaitEvent(e->st, e->ev_sync, 0));
    };
    float* sL[5]; float* sR[5];
    for (int f = 0; f < 5; f++) { sL[f] = e->ss[f].f(); sR[f] = e->ss[5 + f].f(); }
    Levels L(e);
    int cur = 0;
    const bool use_pair = e->kind == 5;
    StepArgs a = base;
    LoopKey key = loop_key(e, adj ? (e->S == 2 ? 5 : 6) : 4);
    key << use_pair << e->W.p << e->Wq.p << e->wscale.p;
    for (int f = 0; f < 5; f++) key << dm[f];
    for (int f = 0; f < 20; f++) key << e->ss[f].p;
    const long long nsteps = (long long)(e->nts - 1) * e->S;
    if (!adj) {
        zero_out(e, rec.ld, e->nts, e->sig_out);
        a.ext = upload_points(e, rec, e->ext_ts, e->ext_ent, e->sig_out);
        key.add(&a, sizeof(a));
        // secondary sources of coarse sample k go to slot k % R on the imaging
        // stream, up to R-1 samples ahead of the step kernels that inject them;
        // slot k is free once coarse interval k - R (its last reader) is done
        auto image = [&](int k) {
            const int sl = k % R;
            EIO_CUDA(cudaStreamWaitEvent(e->st2, e->ev_free[sl], 0));
            launch_imaging(e, 0, k, dm, ring[sl], e->st2);
            EIO_CUDA(cudaEventRecord(e->ev_ready[sl], e->st2));
        };
        run_graph(e, key.h, nsteps, [&] {
        fork();
        for (int k = 0; k < R - 1 && k < e->nts; k++) image(k);
        for (int its = 0; its < e->nts - 1; its++) {
            if (its + R - 1 < e->nts) image(its + R - 1);
            const int l = its % R, r = (its + 1) % R;
            EIO_CUDA(cudaStreamWaitEvent(e->st, e->ev_ready[l], 0));
            EIO_CUDA(cudaStreamWaitEvent(e->st, e->ev_ready[r], 0));
            for (int f = 0; f < 5; f++) { a.ssL[f] = ring[l][f]; a.ssR[f] = ring[r][f]; }
            auto weights = [&](StepArgs& x, int it2) {
                x.sw0 = F[it2 - 1]; x.sw1 = F[h + it2 - 1];
                x.ext.t0 = its; x.ext.w0 = F[it2]; x.ext.w1 = F[h + it2];
            };
            for (int it2 = 1; it2 < e->S + 1;) {
                if (use_pair && it2 + 1 < e->S + 1) {
                    StepArgs a0 = a, a1 = a;
                    weights(a0, it2);
                    weights(a1, it2 + 1);
                    run_pair<0, EPI_INJ_SS>(e, a0, a1, a.inj, L);   // no sparse sources
                    it2 += 2;
                    continue;
                }
                L.set(a);
                weights(a, it2);
                launch_step<0, EPI_INJ_SS>(e, a, cur);
                L.single();
                cur ^= 1;
                it2++;
            }
            // the imaging kernel rewrites every interior cell of a slot, so the
            // reference's memset of the right slice (BornElasticGpuFunctions.cu:806-810) is not needed
            EIO_CUDA(cudaEventRecord(e->ev_free[l], e->st));
        }
        join();
        });
        check_launch();
        stage_out(e, rec.ld, e->nts, e->sig_out, data);
    } else if (e->S == 2) {
        // Adjoint extraction with two fine steps per coarse sample: the coarse
        // sample T of the reference's running sums ssL/ssR (extractInterpAdjointWavefield,
        // K:1369-1376) is ((p(2T+1) f[1] + p(2T) f[0]) + p(2T-1) f[h+1]) (+ p(2T-2) * f[h] = 0),
        // i.e. the old, current and new level of the step (T-1, it2 = 1): that step
        // writes it once (EPI_TRI) and the imaging condition of T follows on the imaging stream.
        stage_in(e, data, rec.ld, e->nts, e->sig_in);
        a.inj = upload_points(e, rec, e->inj_ts, e->inj_ent, e->sig_in);
        const SparseOp injh = halo_sources(e, use_pair, g.recPos, g.nRec, e->sig_in);
        // sample T goes to slot T % R; its imaging runs on the imaging stream
        // while the adjoint keeps stepping; the slot is rewritten R samples later
        auto imaging = [&](int T) {
            const int sl = T % R;
            EIO_CUDA(cudaEventRecord(e->ev_ready[sl], e->st));
            EIO_CUDA(cudaStreamWaitEvent(e->st2, e->ev_ready[sl], 0));
            launch_imaging(e, 1, T, dm, ring[sl], e->st2);
            EIO_CUDA(cudaEventRecord(e->ev_free[sl], e->st2));
        };
        auto tri = [&](StepArgs& x, int T, int mode, float wo, float wc, float wn) {
            EIO_CUDA(cudaStreamWaitEvent(e->st, e->ev_free[T % R], 0));
            for (int f = 0; f < 5; f++) x.eL[f] = ring[T % R][f];
            x.tmode = mode; x.tw_o = wo; x.tw_c = wc; x.tw_n = wn;
        };
        auto weights = [&](StepArgs& x, int its, int it2) {
            x.inj.t0 = its; x.inj.w0 = F[it2 + 1]; x.inj.w1 = F[h + it2 + 1];
        };
        // single steps image inside the sample step (EPI_TRI_IMG): the adjoint sample
        // never leaves the registers.  That step is a k_step, so the point lists must
        // use its tiles (not the sweep kernel's); the two-step kernel keeps the sample ring
        const bool fuse_img = !use_pair && tiled(eff_kind(e));
        const WHist wh = whist(e);
        auto fused = [&](StepArgs& x, int T, int mode, float wo, float wc, float wn) {
            x.tmode = mode; x.tw_o = wo; x.tw_c = wc; x.tw_n = wn;
            x.wh = wh; x.img_its = T; x.dts_inv = e->dts_inv;
            for (int f = 0; f < 5; f++) x.img[f] = dm[f];
            if (e->ckpt == 0) launch_step<1, EPI_TRI_IMG>(e, x, cur);
            else if (e->ckpt == 1) launch_step<1, EPI_TRI_IMG + 1>(e, x, cur);
            else launch_step<1, EPI_TRI_IMG + 2>(e, x, cur);
        };
        key.add(&a, sizeof(a));
        key.add(&injh, sizeof(injh));
        run_graph(e, key.h, nsteps, [&] {
        fork();
        for (int its = e->nts - 2; its > -1; its--) {
            if (use_pair && its > 0) {
                // (its, 1) writes sample its+1, (its, 0) only steps
                StepArgs a0 = a, a1 = a;
                weights(a0, its, 1);
                tri(a0, its + 1, 1, F[1], F[0], F[h + 1]);
                weights(a1, its, 0);
                a1.tmode = 0;
                run_pair<1, EPI_TRI>(e, a0, a1, injh, L);
                imaging(its + 1);
                continue;
            }
            for (int it2 = e->S - 1; it2 > -1; it2--) {
                L.set(a);
                weights(a, its, it2);
                if (it2 == 1) {
                    if (fuse_img) {
                        fused(a, its + 1, 1, F[1], F[0], F[h + 1]);
                    } else {
                        tri(a, its + 1, 1, F[1], F[0], F[h + 1]);
                        launch_step<1, EPI_TRI>(e, a, cur);
                        imaging(its + 1);
                    }
                } else if (its == 0) {   // sample 0 = p(1) f[1] + p(0) f[0]
                    if (fuse_img) {
                        fused(a, 0, 2, 0.f, F[1], F[0]);
                    } else {
                        tri(a, 0, 2, 0.f, F[1], F[0]);
                        launch_step<1, EPI_TRI>(e, a, cur);
                        imaging(0);
                    }
                } else {
                    launch_step<1, EPI_NONE>(e, a, cur);
                }
                L.single();
                cur ^= 1;
            }
        }
        join();
        });
        check_launch();
    } else {
        stage_in(e, data, rec.ld, e->nts, e->sig_in);
        a.inj = upload_points(e, rec, e->inj_ts, e->inj_ent, e->sig_in);
        key.add(&a, sizeof(a));
        run_graph(e, key.h, nsteps, [&] {
        for (int its = e->nts - 2; its > -1; its--) {
            for (int it2 = e->S - 1; it2 > -1; it2--) {
                L.set(a);
                for (int f = 0; f < 5; f++) { a.eL[f] = sL[f]; a.eR[f] = sR[f]; }
                a.inj.t0 = its; a.inj.w0 = F[it2 + 1]; a.inj.w1 = F[h + it2 + 1];
                a.sw0 = F[it2]; a.sw1 = F[h + it2];
                launch_step<1, EPI_EXT_SS>(e, a, cur);
                L.single();
                cur ^= 1;
            }
            launch_imaging(e, 1, its + 1, dm, sR, e->st);
            std::swap(sL, sR);
            for (int f = 0; f < 5; f++) EIO_CUDA(cudaMemsetAsync(sL[f], 0, sizeof(float) * e->n, e->st));
        }
        launch_imaging(e, 1, 0, dm, sR, e->st);
        });
        check_launch();
    }
    EIO_CUDA(cudaStreamSynchronize(e->st));
    stats_flush(e);
    err_check(e);
}

// ---------------------------------------------------------------- host wrappers
static void h2d(Engine* e, DBuf& b, const float* h, size_t count) {
    b.ensure(std::max<size_t>(sizeof(float) * count, 16));
    if (count) EIO_CUDA(cudaMemcpyAsync(b.p, h, sizeof(float) * count, cudaMemcpyHostToDevice, e->st));
}
static void d2h(Engine* e, float* h, const DBuf& b, size_t count) {
    if (count) EIO_CUDA(cudaMemcpyAsync(h, b.p, sizeof(float) * count, cudaMemcpyDeviceToHost, e->st));
}

void engine_nl_host(Engine* e, int adj, float* const model[5], float* const data[5], const ShotGeom& g, float* wfld) {
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
    float* wdev = nullptr;
    const size_t wcount = (size_t)5 * e->nts * e->n;
    if (wfld) {
        e->wsave.ensure(sizeof(float) * wcount);
        EIO_CUDA(cudaMemsetAsync(e->wsave.p, 0, sizeof(float) * wcount, e->st));
        wdev = e->wsave.f();
    }
    engine_nl(e, adj, dmod, ddat, g, wdev);
    if (wfld) d2h(e, wfld, e->wsave, wcount);
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

// ---------------------------------------------------------------- multi-shot host paths
// The multi-shot operators keep the Born perturbation (forward) or the
// accumulating gradient (adjoint) on the device across shots, and interpolate
// the receiver traces between the regular grid and the devices on the GPU, so
// only the irregular traces cross PCIe.

// dst += src over n floats (n a multiple of 4, 16-byte aligned arrays)
__global__ void __launch_bounds__(256) k_add4(float* __restrict__ dst, const float* __restrict__ src, long long n4)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        float4 a = reinterpret_cast<float4*>(dst)[i];
        const float4 b = reinterpret_cast<const float4*>(src)[i];
        a.x += b.x; a.y += b.y; a.z += b.z; a.w += b.w;
        reinterpret_cast<float4*>(dst)[i] = a;
    }
}

bool engine_is_tuned(const Engine* e) { return e->tuned; }
// device bytes of source-wavefield history this engine already holds
size_t engine_history_bytes(const Engine* e) { return (e->W.host ? 0 : e->W.cap) + (e->Wq.host ? 0 : e->Wq.cap); }
void engine_set_history_where(Engine* e, int where) {
    if (where < 0 || where > 2) throw Error(EIO_ERR_ARG, "history location: 0 (device, host when short), 1 device, 2 host");
    e->hist_where = where;
}
// 0: no history held, 1: device memory, 2: mapped host memory
int engine_history_where(const Engine* e) {
    const DBuf& b = e->ckpt ? e->Wq : e->W;
    return b.cap == 0 ? 0 : (b.host ? 2 : 1);
}
void set_device_memory_cap(long long bytes) { g_dbuf_cap = bytes > 0 ? bytes : 0; }
long long device_memory_used() { return g_dbuf_used.load(); }
int engine_get_checkpoint(const Engine* e) { return e->ckpt; }
int engine_get_graphs(const Engine* e) { return e->use_graphs ? 1 : 0; }
size_t engine_cells(const Engine* e) { return (size_t)e->nz * e->full_nx; }

// the lane's own image (whole grid), zeroed, for a lane other than the first
void engine_dm_ptrs(Engine* e, float* out[5]) {
    const size_t n = (size_t)e->nz * e->full_nx;
    for (int f = 0; f < 5; f++) {
        e->stage_c[f].ensure(sizeof(float) * n);
        out[f] = e->stage_c[f].f();
    }
}

// dst (device, whole grid, 5 components) += this lane's image
void engine_dm_add(Engine* e, float* const dst[5]) {
    EIO_CUDA(cudaSetDevice(e->device));
    const long long n4 = (long long)e->nz * e->full_nx / 4;
    for (int f = 0; f < 5; f++) {
        k_add4<<<4 * e->nsm, 256, 0, e->st>>>(dst[f], e->stage_c[f].f(), n4);
        e->launches++;
    }
    check_launch();
    EIO_CUDA(cudaStreamSynchronize(e->st));
}

// the perturbation / image always covers the whole grid (shot windows are views of it)
void engine_dm_upload(Engine* e, float* const dm[5]) {
    EIO_CUDA(cudaSetDevice(e->device));
    const size_t n = (size_t)e->nz * e->full_nx;
    for (int f = 0; f < 5; f++) h2d(e, e->stage_c[f], dm[f], n);
}
void engine_dm_zero(Engine* e) {
    EIO_CUDA(cudaSetDevice(e->device));
    const size_t n = (size_t)e->nz * e->full_nx;
    for (int f = 0; f < 5; f++) {
        e->stage_c[f].ensure(sizeof(float) * n);
        EIO_CUDA(cudaMemsetAsync(e->stage_c[f].p, 0, sizeof(float) * n, e->st));
    }
}
void engine_dm_download(Engine* e, float* const dm[5]) {
    const size_t n = (size_t)e->nz * e->full_nx;
    for (int f = 0; f < 5; f++) d2h(e, dm[f], e->stage_c[f], n);
    EIO_CUDA(cudaStreamSynchronize(e->st));
}

// receiver interpolators of one shot: weights, slots and the inverse (slot ->
// entries in ascending device, filter order) on the device
static void upload_interps(Engine* e, const SInterp* const rec[4]) {
    for (int k = 0; k < 4; k++) {
        const SInterp& s = *rec[k];
        Engine::DevInterp& d = e->rint[k];
        const size_t ne = (size_t)s.nIrreg * s.nft;
        std::vector<int> start(s.nReg + 1, 0), ent(ne);
        for (size_t i = 0; i < ne; i++) start[s.slot[i] + 1]++;
        for (int r = 0; r < s.nReg; r++) start[r + 1] += start[r];
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (size_t i = 0; i < ne; i++) ent[fill[s.slot[i]]++] = (int)i;
        upload(d.slot, s.slot.data(), sizeof(int) * ne, e->st);
        upload(d.w, s.w.data(), sizeof(float) * ne, e->st);
        upload(d.start, start.data(), sizeof(int) * start.size(), e->st);
        upload(d.ent, ent.data(), sizeof(int) * ne, e->st);
        d.nIrreg = s.nIrreg; d.nReg = s.nReg; d.nft = s.nft;
        // the host copies above are pageable and are read when the copies run
        EIO_CUDA(cudaStreamSynchronize(e->st));
    }
}

static void interp_fwd(Engine* e, int grid, const float* reg, float* irreg) {
    const Engine::DevInterp& d = e->rint[grid];
    const long long n = (long long)d.nIrreg * e->nts;
    if (n == 0) return;
    k_interp_fwd<<<(unsigned)((n + 255) / 256), 256, 0, e->st>>>(reg, irreg, static_cast<const int*>(d.slot.p),
                                                                 d.w.f(), d.nIrreg, d.nft, e->nts);
    e->launches++;
}
static void interp_adj(Engine* e, int grid, const float* irreg, float* reg) {
    const Engine::DevInterp& d = e->rint[grid];
    const long long n = (long long)d.nReg * e->nts;
    if (n == 0) return;
    k_interp_adj<<<(unsigned)((n + 255) / 256), 256, 0, e->st>>>(irreg, reg, static_cast<const int*>(d.start.p),
                                                                 static_cast<const int*>(d.ent.p), d.w.f(), d.nReg,
                                                                 d.nft, e->nts);
    e->launches++;
}

// regular-grid receiver buffers (stage_b) and irregular ones (stage_d) of one shot;
// the adjoint fills stage_b from the irregular host traces
static void stage_receivers(Engine* e, int adj, const ShotGeom& g, const SInterp* const rec[4], const float* dataIrreg,
                            float* dr[5]) {
    upload_interps(e, rec);
    const int nIrreg = rec[0]->nIrreg;
    for (int f = 0; f < 5; f++) {
        const int grid = kFieldGrid[f];
        const size_t nr = (size_t)g.nRec[grid] * e->nts, ni = (size_t)nIrreg * e->nts;
        e->stage_b[f].ensure(std::max<size_t>(16, sizeof(float) * nr));
        e->stage_d[f].ensure(std::max<size_t>(16, sizeof(float) * ni));
        if (adj) {
            h2d(e, e->stage_d[f], dataIrreg + (size_t)f * ni, ni);
            interp_adj(e, grid, e->stage_d[f].f(), e->stage_b[f].f());
        }
        dr[f] = e->stage_b[f].f();
    }
}
static void return_receivers(Engine* e, const SInterp* const rec[4], float* dataIrreg) {
    const size_t ni = (size_t)rec[0]->nIrreg * e->nts;
    for (int f = 0; f < 5; f++) {
        interp_fwd(e, kFieldGrid[f], e->stage_b[f].f(), e->stage_d[f].f());
        d2h(e, dataIrreg + (size_t)f * ni, e->stage_d[f], ni);
    }
}

void engine_born_shot(Engine* e, int adj, float* const srcDtw[5], const ShotGeom& g, const SInterp* const rec[4],
                      float* dataIrreg) {
    EIO_CUDA(cudaSetDevice(e->device));
    float* ds[5]; float* dd[5]; float* dr[5];
    for (int f = 0; f < 5; f++) {
        h2d(e, e->stage_a[f], srcDtw[f], (size_t)g.nSrc[kFieldGrid[f]] * e->ntw);
        ds[f] = e->stage_a[f].f();
        dd[f] = e->stage_c[f].f() + (long long)e->win_ix0 * e->nz;   // the shot window of the image
    }
    stage_receivers(e, adj, g, rec, dataIrreg, dr);
    engine_born(e, adj, ds, dd, dr, g);
    if (!adj) return_receivers(e, rec, dataIrreg);
    EIO_CUDA(cudaStreamSynchronize(e->st));
}

// One shot of an FWI gradient: the nonlinear forward of the regular coarse
// sources modelReg recording the Born history (engine_nl_record), the modelled
// irregular data to dataIrreg (host [5][nIrreg][nts]), then the host callback
// residual(dataIrreg, resid) that fills resid (host, same layout: S^T of the
// sampled residual) and returns its misfit, then the Born adjoint of resid on
// the recorded history into the image dm (device).  Two propagations instead
// of the three of a nonlinear forward followed by a Born adjoint.
double engine_fwi_shot(Engine* e, float* const modelReg[5], const ShotGeom& g, const SInterp* const rec[4],
                       float* dataIrreg, float* resid, double (*residual)(void*, const float*, float*), void* ctx,
                       float* const dm[5]) {
    EIO_CUDA(cudaSetDevice(e->device));
    float* ms[5]; float* dr[5];
    for (int f = 0; f < 5; f++) {
        h2d(e, e->stage_a[f], modelReg[f], (size_t)g.nSrc[kFieldGrid[f]] * e->nts);
        ms[f] = e->stage_a[f].f();
    }
    stage_receivers(e, 0, g, rec, nullptr, dr);
    engine_nl_record(e, ms, dr, g);
    return_receivers(e, rec, dataIrreg);
    EIO_CUDA(cudaStreamSynchronize(e->st));
    const double phi = residual(ctx, dataIrreg, resid);
    stage_receivers(e, 1, g, rec, resid, dr);
    float* none[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    engine_born(e, 1, none, dm, dr, g, true);
    EIO_CUDA(cudaStreamSynchronize(e->st));
    return phi;
}

// ---------------------------------------------------------------- Born shots in lockstep
// The Born operators and the fused FWI gradient for nb shots at once, one
// engine per shot (own wavefields, history, secondary-source ring, point
// lists, window), every fine step one k_step_shots launch for all of them
// (CTA b: tile b / nb of shot b % nb).  All shots read the first engine's
// medium arrays (every engine of a context holds the same medium), so the
// shots' CTAs of one tile read a medium tile from HBM once.  The phases, time
// weights and epilogues are those of born_source and engine_born (FP32
// history, two fine steps per coarse sample), so every shot's traces and
// image equal its one-shot propagation with the tile kernel (k_step, 4 CTAs
// per SM; 3 for the fused adjoint imaging step) bit for bit.  Launches go to
// the first engine's streams (imaging on its second stream); that stream
// waits for every engine's preparation and every engine waits for it before
// reading results back.

// the batch launch of one fine step; grid = nb x the largest shot's tile count
template <int DIR, int EPI, int MINB>
static void launch_shots(Engine* e0, const StepBatch& b, int nb, int max_tiles) {
    const bool timed = e0->stats && (e0->step_launches + e0->pair_launches) % STATS_PERIOD == 0;
    if (timed) stats_mark(e0);
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)(nb * max_tiles));
    cfg.blockDim = dim3(NT);
    cfg.stream = e0->st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    EIO_CUDA(cudaLaunchKernelEx(&cfg, k_step_shots<DIR, EPI, MINB>, b, nb));
    if (timed) {
        stats_mark(e0);
        e0->sampled++;
    }
    e0->launches++;
    e0->step_launches++;
}

// a batch launch updates the interior cells of every shot once
static void batch_count(Engine* e0, Engine* const* es, int nb, long long launches) {
    long long cells = 0;
    for (int i = 0; i < nb; i++) cells += (long long)(es[i]->nz - 2 * FAT) * (es[i]->nx - 2 * FAT);
    e0->step_cells += cells * launches;
}

// Nonlinear forward (adj = 0) or adjoint (adj = 1) of nb shots, one engine
// each (own wavefields, point lists, windows), advanced in lockstep: one
// k_step_shots launch per fine step covers the tiles of every shot (the
// shots of a tile next to each other, reading one copy of the medium), so
// small grids fill the GPU and the per-step launch cost is paid once for all
// of them.  The steps, time weights and arithmetic
// are those of engine_nl (same stencil body), so each shot's result equals its
// single-shot propagation with the tile kernel bit for bit.  No free surface,
// no wavefield output; the launches go to the first engine's stream, which
// waits for every engine's preparation, and every engine waits for the loop
// before returning its traces.  modelReg: regular source traces, nb x 5 host
// arrays (read by the forward, written by the adjoint); dataIrreg: irregular
// receiver traces, nb host arrays (written by the forward, read by the adjoint).
void engine_nl_shots_batch(Engine* const* es, int nb, int adj, float* const* modelReg, const ShotGeom* g,
                           const SInterp* const* rec, float* const* dataIrreg) {
    if (nb < 1 || nb > STEP_BATCH) throw Error(EIO_ERR_ARG, "batch of 1 .. 8 shots");
    Engine* e0 = es[0];
    EIO_CUDA(cudaSetDevice(e0->device));
    if (!e0->tuned) engine_autotune(e0);
    const int minb = (e0->kind == 3 || e0->kind == 5) ? 4 : 3;
    std::vector<PointList> src(nb), recp(nb);
    std::vector<Levels> lv;
    lv.reserve(nb);
    StepBatch b;
    memset(&b, 0, sizeof(b));
    int max_tiles = 0;
    for (int i = 0; i < nb; i++) {
        Engine* e = es[i];
        if (e->device != e0->device || e->nts != e0->nts || e->S != e0->S)
            throw Error(EIO_ERR_ARG, "batched shots need engines of one device and one time axis");
        if (e->fs) throw Error(EIO_ERR_UNSUPPORTED, "batched shots have no free surface");
        err_reset(e);
        float* dm[5]; float* dr[5];
        for (int f = 0; f < 5; f++) {
            const size_t nm = (size_t)g[i].nSrc[kFieldGrid[f]] * e->nts;
            if (!adj) h2d(e, e->stage_a[f], modelReg[5 * i + f], nm);
            else e->stage_a[f].ensure(std::max<size_t>(16, sizeof(float) * nm));
            dm[f] = e->stage_a[f].f();
        }
        stage_receivers(e, adj, g[i], rec + 4 * i, adj ? dataIrreg[i] : nullptr, dr);
        build_points(e, g[i].srcPos, g[i].nSrc, src[i]);
        build_points(e, g[i].recPos, g[i].nRec, recp[i]);
        StepArgs& a = b.a[i];
        a = base_args(e);
        // every engine of a context holds the same medium: all shots read the first
        // engine's, so the shots' CTAs of one tile share it through L2
        for (int f = 0; f < 5; f++) a.par[f] = mpar(e0, f) + (long long)e->win_ix0 * e->nz;
        zero_wavefields(e);
        lv.emplace_back(e);
        if (!adj) {
            stage_in(e, dm, src[i].ld, e->nts, e->sig_in);
            zero_out(e, recp[i].ld, e->nts, e->sig_out);
            a.inj = upload_points(e, src[i], e->inj_ts, e->inj_ent, e->sig_in);
            a.ext = upload_points(e, recp[i], e->ext_ts, e->ext_ent, e->sig_out);
        } else {
            stage_in(e, dr, recp[i].ld, e->nts, e->sig_in);
            zero_out(e, src[i].ld, e->nts, e->sig_out);
            a.inj = upload_points(e, recp[i], e->inj_ts, e->inj_ent, e->sig_in);
            a.ext = upload_points(e, src[i], e->ext_ts, e->ext_ent, e->sig_out);
        }
        max_tiles = std::max(max_tiles, e->ntiles);
        if (i > 0) {
            EIO_CUDA(cudaEventRecord(e->ev_sync, e->st));
            EIO_CUDA(cudaStreamWaitEvent(e0->st, e->ev_sync, 0));
        }
    }
    const float* F = e0->filt.data();
    const int h = e0->h;
    Engine* const* engines = es;
    auto launch = [&] {
        if (!adj) {
            if (minb == 4) launch_shots<0, EPI_NONE, 4>(e0, b, nb, max_tiles);
            else launch_shots<0, EPI_NONE, 3>(e0, b, nb, max_tiles);
        } else {
            if (minb == 4) launch_shots<1, EPI_NONE, 4>(e0, b, nb, max_tiles);
            else launch_shots<1, EPI_NONE, 3>(e0, b, nb, max_tiles);
        }
        batch_count(e0, engines, nb, 1);
    };
    // the fine steps in propagation order, with the time weights of engine_nl
    auto step = [&](int its, int it2) {
        const int ki = adj ? it2 + 1 : it2 - 1;
        for (int i = 0; i < nb; i++) {
            StepArgs& a = b.a[i];
            lv[i].set(a);
            a.inj.t0 = its; a.inj.w0 = F[ki]; a.inj.w1 = F[h + ki];
            a.ext.t0 = its; a.ext.w0 = F[it2]; a.ext.w1 = F[h + it2];
            lv[i].single();
        }
        launch();
    };
    if (!adj) {
        for (int its = 0; its < e0->nts - 1; its++)
            for (int it2 = 1; it2 < e0->S + 1; it2++) step(its, it2);
    } else {
        for (int its = e0->nts - 2; its > -1; its--)
            for (int it2 = e0->S - 1; it2 > -1; it2--) step(its, it2);
    }
    check_launch();
    EIO_CUDA(cudaEventRecord(e0->ev_sync, e0->st));
    for (int i = 0; i < nb; i++) {
        Engine* e = es[i];
        if (i > 0) EIO_CUDA(cudaStreamWaitEvent(e->st, e0->ev_sync, 0));
        if (!adj) {
            float* dr[5];
            for (int f = 0; f < 5; f++) dr[f] = e->stage_b[f].f();
            stage_out(e, recp[i].ld, e->nts, e->sig_out, dr);
            return_receivers(e, rec + 4 * i, dataIrreg[i]);
        } else {
            float* dm[5];
            for (int f = 0; f < 5; f++) dm[f] = e->stage_a[f].f();
            stage_out(e, src[i].ld, e->nts, e->sig_out, dm);
            for (int f = 0; f < 5; f++)
                d2h(e, modelReg[5 * i + f], e->stage_a[f], (size_t)g[i].nSrc[kFieldGrid[f]] * e->nts);
        }
    }
    for (int i = 0; i < nb; i++) {
        EIO_CUDA(cudaStreamSynchronize(es[i]->st));
        err_check(es[i]);
    }
}

// ---------------------------------------------------------------- Born shots in lockstep (phases)
struct ShotBatch {
    Engine* const* es;
    int nb;
    int max_tiles = 0;
    StepBatch b;
    std::vector<Levels> lv;
    // persistent time loop: the steps of a phase are recorded here and run as one k_wave launch
    bool wave = false;
    std::vector<StepArgs> plan;
    std::vector<int> modes, ssk;
    ShotBatch(Engine* const* engines, int n) : es(engines), nb(n) {
        if (nb < 1 || nb > STEP_BATCH) throw Error(EIO_ERR_ARG, "batch of 1 .. 8 shots");
        memset(&b, 0, sizeof(b));
        Engine* e0 = es[0];
        for (int i = 0; i < nb; i++) {
            Engine* e = es[i];
            if (e->device != e0->device || e->nts != e0->nts || e->S != e0->S || e->nz != e0->nz)
                throw Error(EIO_ERR_ARG, "batched shots need engines of one device and one time axis");
            if (e->S != 2 || e->ckpt)
                throw Error(EIO_ERR_UNSUPPORTED, "batched Born shots need sub = 1 and an FP32 history");
            max_tiles = std::max(max_tiles, e->ntiles);
        }
    }
    Engine* e0() const { return es[0]; }
    // base arguments of every shot, reading the first engine's medium at its own window
    void base() {
        Engine* e0 = es[0];
        for (int i = 0; i < nb; i++) {
            Engine* e = es[i];
            b.a[i] = base_args(e);
            const long long off = (long long)e->win_ix0 * e->nz;
            for (int f = 0; f < 5; f++) b.a[i].par[f] = mpar(e0, f) + off;
        }
    }
    void levels() {
        lv.clear();
        for (int i = 0; i < nb; i++) {
            zero_wavefields(es[i]);
            lv.emplace_back(es[i]);
        }
    }
    // the first engine's stream waits for the work queued on the others, and back
    void join_in() {
        for (int i = 1; i < nb; i++) {
            EIO_CUDA(cudaEventRecord(es[i]->ev_sync, es[i]->st));
            EIO_CUDA(cudaStreamWaitEvent(es[0]->st, es[i]->ev_sync, 0));
        }
    }
    void join_out() {
        EIO_CUDA(cudaEventRecord(es[0]->ev_sync, es[0]->st));
        for (int i = 1; i < nb; i++) EIO_CUDA(cudaStreamWaitEvent(es[i]->st, es[0]->ev_sync, 0));
    }
    // one fine step: launched now, or recorded for the persistent loop (whose
    // phase runs one epilogue: EPI_TRI / EPI_TRI_IMG steps without a coarse
    // sample carry tmode 0 and are plain steps)
    template <int DIR, int EPI, int MINB>
    void step(int ss_k = -1) {
        if (wave) {
            plan.insert(plan.end(), b.a, b.a + nb);
            modes.push_back(ss_k >= 0 ? WAVE_SS : 0);
            ssk.push_back(ss_k);
        } else {
            launch_shots<DIR, EPI, MINB>(es[0], b, nb, max_tiles);
            batch_count(es[0], es, nb, 1);
        }
        for (int i = 0; i < nb; i++) lv[i].single();
    }
    // start recording a phase (bit `phase` of the first engine's persistent-loop mask)
    void begin(int phase) {
        wave = (es[0]->use_wave & phase) != 0;
        plan.clear();
        modes.clear();
        ssk.clear();
    }
    // run the recorded phase as one persistent launch of k_wave<DIR, EPI, MINB>;
    // ia / slots: the secondary-source inputs of the forward scattered phase
    template <int DIR, int EPI, int MINB>
    void run(const ImagingArgs* ia = nullptr, float* const* slots = nullptr);
};

template <int DIR, int EPI, int MINB>
static int wave_resident(Engine* e, int slot) {
    int& n = e->wave_ctas[slot];
    if (!n) {
        int per = 0;
        EIO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_wave<DIR, EPI, MINB>, NT, 0));
        if (per < 1) throw Error(EIO_ERR_CUDA, "the persistent step kernel does not fit on an SM");
        n = per * e->nsm;
    }
    return n;
}
// the wave_ctas slot of each instantiation
template <int DIR, int EPI, int MINB>
constexpr int wave_slot() {
    return EPI == EPI_TRI ? 0 : EPI == EPI_INJ_SS ? 1 : EPI == EPI_TRI_IMG ? 2 : (DIR == 0 ? 3 : 4) + (MINB == 4 ? 2 : 0);
}

template <int DIR, int EPI, int MINB>
void ShotBatch::run(const ImagingArgs* ia, float* const* slots) {
    if (!wave || modes.empty()) return;
    Engine* e0 = es[0];
    const int nsteps = (int)modes.size();
    const size_t pbytes = sizeof(StepArgs) * plan.size();
    e0->wave_plan.ensure(pbytes);
    e0->wave_mode.ensure(sizeof(int) * nsteps);
    e0->wave_ssk.ensure(sizeof(int) * nsteps);
    e0->wave_done.ensure(sizeof(int) * (size_t)nb * max_tiles);
    EIO_CUDA(cudaMemcpyAsync(e0->wave_plan.p, plan.data(), pbytes, cudaMemcpyHostToDevice, e0->st));
    EIO_CUDA(cudaMemcpyAsync(e0->wave_mode.p, modes.data(), sizeof(int) * nsteps, cudaMemcpyHostToDevice, e0->st));
    EIO_CUDA(cudaMemcpyAsync(e0->wave_ssk.p, ssk.data(), sizeof(int) * nsteps, cudaMemcpyHostToDevice, e0->st));
    EIO_CUDA(cudaMemsetAsync(e0->wave_done.p, 0, sizeof(int) * (size_t)nb * max_tiles, e0->st));
    WaveArgs w;
    memset(&w, 0, sizeof(w));
    w.plan = static_cast<const StepArgs*>(e0->wave_plan.p);
    w.mode = static_cast<const int*>(e0->wave_mode.p);
    w.ss_k = static_cast<const int*>(e0->wave_ssk.p);
    for (int i = 0; i < nb; i++) {
        if (ia) w.img[i] = ia[i];
        if (slots)
            for (int k = 0; k < 2; k++)
                for (int f = 0; f < 5; f++) w.ss[i][k][f] = slots[(i * 2 + k) * 5 + f];
    }
    w.done = static_cast<int*>(e0->wave_done.p);
    w.err = static_cast<int*>(e0->err.p);
    w.wait_limit = e0->wait_limit * 4;
    w.nsteps = nsteps;
    w.nb = nb;
    w.max_tiles = max_tiles;
    const int units = nb * max_tiles;
    const bool timed = e0->stats;
    if (timed) stats_mark(e0);
    void* args[] = {&w};
    const int g = std::min(units, wave_resident<DIR, EPI, MINB>(e0, wave_slot<DIR, EPI, MINB>()));
    EIO_CUDA(cudaLaunchCooperativeKernel((const void*)k_wave<DIR, EPI, MINB>, g, NT, args, 0, e0->st));
    if (timed) {
        stats_mark(e0);
        e0->sampled += nsteps;   // the event pair covers every step of the phase
    }
    e0->launches++;
    e0->step_launches += nsteps;
    batch_count(e0, es, nb, nsteps);
    // the host arrays are read by the copies above: keep them until the stream has passed them
    EIO_CUDA(cudaStreamSynchronize(e0->st));
}

// Phase 1 of every shot: the source wavefield and its coarse Vx/Vz history
// (born_source with two fine steps per sample).  src: per-shot source lists
// (fine-time Born sources, or the nonlinear operators' coarse traces when ext
// holds the receiver lists of a nonlinear forward that also records).
static void batch_source(ShotBatch& B, std::vector<PointList>& src, const SparseOp* ext) {
    Engine* e0 = B.e0();
    for (int i = 0; i < B.nb; i++) {
        Engine* e = B.es[i];
        const size_t wbytes = sizeof(float) * 2 * (size_t)e->nts * e->n;
        const bool fresh = e->W.cap < wbytes;
        e->W.ensure(wbytes, e->hist_where);
        if (fresh || !e->w_clean || e->w_n != e->n) EIO_CUDA(cudaMemsetAsync(e->W.p, 0, wbytes, e->st));
        e->w_clean = true;
        e->w_n = e->n;
        StepArgs& a = B.b.a[i];
        a.inj = upload_points(e, src[i], e->inj_ts, e->inj_ent, e->sig_in);
        if (ext) a.ext = ext[i];
        else memset(&a.ext, 0, sizeof(a.ext));
        a.W0 = e->W.f();
        a.W1 = e->W.f() + (long long)e->nts * e->n;
    }
    B.levels();
    B.join_in();
    const SrcWeights weights{e0, ext != nullptr};
    const float* F = e0->filt.data();
    const int h = e0->h;
    B.begin(1);
    for (int its = 0; its < e0->nts - 1; its++)
        for (int it2 = 1; it2 < 3; it2++) {
            const bool last = (its == e0->nts - 2 && it2 == 2);
            for (int i = 0; i < B.nb; i++) {
                StepArgs& a = B.b.a[i];
                B.lv[i].set(a);
                weights(a, its, it2);
                if (it2 == 1) {          // row its = o*f[h+1] + c*f[h+2] + n*f[1]
                    a.tmode = 1; a.wt = its; a.tw_o = F[h + 1]; a.tw_c = F[h + 2]; a.tw_n = F[1];
                } else if (last) {       // row nts-1 = c*f[h+1] + n*f[h+2]
                    a.tmode = 2; a.wt = its + 1; a.tw_o = 0.f; a.tw_c = F[h + 1]; a.tw_n = F[h + 2];
                } else {
                    a.tmode = 0;         // no coarse sample: a plain step
                }
            }
            if (it2 == 1 || last || B.wave) B.step<0, EPI_TRI, 4>();
            else B.step<0, EPI_NONE, 4>();
        }
    B.run<0, EPI_TRI, 3>();
    check_launch();
    B.join_out();   // phase 2 prepares on the engines' own streams
}

// Phase 2 of the Born forward for every shot: the scattered wavefield with the
// secondary sources of the perturbation dm[i] (per shot, windowed views);
// imaging kernels on the first engine's imaging stream fill each shot's ring
// up to R-1 coarse samples ahead; rec: receiver lists (extraction).
static void batch_scatter(ShotBatch& B, std::vector<PointList>& rec, float* const* dm) {
    Engine* e0 = B.e0();
    constexpr int R = 4;
    ImagingBatch ib;
    memset(&ib, 0, sizeof(ib));
    int img_tiles = 0;
    for (int i = 0; i < B.nb; i++) {
        Engine* e = B.es[i];
        for (int k = 0; k < R; k++)
            for (int f = 0; f < 5; f++) e->ss[k * 5 + f].ensure(sizeof(float) * e->n);
        for (int f = 0; f < 10; f++) EIO_CUDA(cudaMemsetAsync(e->ss[f].p, 0, sizeof(float) * e->n, e->st));
        zero_out(e, rec[i].ld, e->nts, e->sig_out);
        StepArgs& a = B.b.a[i];
        memset(&a.inj, 0, sizeof(a.inj));
        a.ext = upload_points(e, rec[i], e->ext_ts, e->ext_ent, e->sig_out);
        ImagingArgs& ia = ib.a[i];
        ia.h = whist(e);
        ia.nz = e->nz; ia.nx = e->nx;
        for (int q = 0; q < 4; q++) { ia.cz[q] = e->zc[q]; ia.cx[q] = e->xc[q]; }
        ia.dts_inv = e->dts_inv;
        for (int f = 0; f < 5; f++) ia.dm[f] = dm[5 * i + f];
        img_tiles = std::max(img_tiles, ((e->nz - 2 * FAT + TZ - 1) / TZ) * ((e->nx - 2 * FAT) / TX));
    }
    B.levels();
    B.join_in();
    const float* F = e0->filt.data();
    const int h = e0->h;
    B.begin(2);
    if (B.wave) {
        // persistent loop: the owning CTA computes the secondary sources of sample k
        // for its tile into ring slot k % 2 right before the first step that uses them
        std::vector<float*> slots((size_t)B.nb * 2 * 5);
        for (int i = 0; i < B.nb; i++)
            for (int k = 0; k < 2; k++)
                for (int f = 0; f < 5; f++) slots[(i * 2 + k) * 5 + f] = B.es[i]->ss[k * 5 + f].f();
        for (int its = 0; its < e0->nts - 1; its++)
            for (int it2 = 1; it2 < 3; it2++) {
                for (int i = 0; i < B.nb; i++) {
                    StepArgs& a = B.b.a[i];
                    B.lv[i].set(a);
                    for (int f = 0; f < 5; f++) {
                        a.ssL[f] = slots[(i * 2 + (its & 1)) * 5 + f];
                        a.ssR[f] = slots[(i * 2 + ((its + 1) & 1)) * 5 + f];
                    }
                    a.sw0 = F[it2 - 1]; a.sw1 = F[h + it2 - 1];
                    a.ext.t0 = its; a.ext.w0 = F[it2]; a.ext.w1 = F[h + it2];
                }
                // sample 0 before the first step; sample its+1 before (its, 2), its first reader
                const int k = (its == 0 && it2 == 1) ? 0 : (it2 == 2 ? its + 1 : -1);
                B.step<0, EPI_INJ_SS, 4>(k);
            }
        B.run<0, EPI_INJ_SS, 3>(ib.a, slots.data());
        check_launch();
        return;
    }
    EIO_CUDA(cudaEventRecord(e0->ev_sync, e0->st));
    EIO_CUDA(cudaStreamWaitEvent(e0->st2, e0->ev_sync, 0));
    for (int k = 0; k < R; k++) {
        EIO_CUDA(cudaEventRecord(e0->ev_free[k], e0->st2));
        EIO_CUDA(cudaEventRecord(e0->ev_ready[k], e0->st2));
    }
    auto image = [&](int k) {
        const int sl = k % R;
        EIO_CUDA(cudaStreamWaitEvent(e0->st2, e0->ev_free[sl], 0));
        for (int i = 0; i < B.nb; i++) {
            ib.a[i].its = k;
            for (int f = 0; f < 5; f++) ib.a[i].ss[f] = B.es[i]->ss[sl * 5 + f].f();
        }
        k_imaging_shots<0, 0><<<B.nb * img_tiles, NT, 0, e0->st2>>>(ib, B.nb);
        e0->launches++;
        EIO_CUDA(cudaEventRecord(e0->ev_ready[sl], e0->st2));
    };
    for (int k = 0; k < R - 1 && k < e0->nts; k++) image(k);
    for (int its = 0; its < e0->nts - 1; its++) {
        if (its + R - 1 < e0->nts) image(its + R - 1);
        const int l = its % R, r = (its + 1) % R;
        EIO_CUDA(cudaStreamWaitEvent(e0->st, e0->ev_ready[l], 0));
        EIO_CUDA(cudaStreamWaitEvent(e0->st, e0->ev_ready[r], 0));
        for (int it2 = 1; it2 < 3; it2++) {
            for (int i = 0; i < B.nb; i++) {
                StepArgs& a = B.b.a[i];
                B.lv[i].set(a);
                for (int f = 0; f < 5; f++) { a.ssL[f] = B.es[i]->ss[l * 5 + f].f(); a.ssR[f] = B.es[i]->ss[r * 5 + f].f(); }
                a.sw0 = F[it2 - 1]; a.sw1 = F[h + it2 - 1];
                a.ext.t0 = its; a.ext.w0 = F[it2]; a.ext.w1 = F[h + it2];
            }
            B.step<0, EPI_INJ_SS, 4>();
        }
        EIO_CUDA(cudaEventRecord(e0->ev_free[l], e0->st));
    }
    EIO_CUDA(cudaEventRecord(e0->ev_sync, e0->st2));
    EIO_CUDA(cudaStreamWaitEvent(e0->st, e0->ev_sync, 0));
    check_launch();
}

// Phase 2 of the Born adjoint for every shot: the adjoint wavefield of the
// regular receiver traces (inj), the imaging condition fused into the
// coarse-sample steps (EPI_TRI_IMG) against each shot's history, into the
// per-shot images img[i] (windowed views; shots of a batch never share one).
static void batch_adjoint(ShotBatch& B, std::vector<PointList>& rec, float* const* img) {
    Engine* e0 = B.e0();
    for (int i = 0; i < B.nb; i++) {
        Engine* e = B.es[i];
        StepArgs& a = B.b.a[i];
        a.inj = upload_points(e, rec[i], e->inj_ts, e->inj_ent, e->sig_in);
        memset(&a.ext, 0, sizeof(a.ext));
        a.wh = whist(e);
        a.dts_inv = e->dts_inv;
        for (int f = 0; f < 5; f++) a.img[f] = img[5 * i + f];
    }
    B.levels();
    B.join_in();
    const float* F = e0->filt.data();
    const int h = e0->h;
    B.begin(4);
    for (int its = e0->nts - 2; its > -1; its--)
        for (int it2 = 1; it2 > -1; it2--) {
            int T = -1;
            for (int i = 0; i < B.nb; i++) {
                StepArgs& a = B.b.a[i];
                B.lv[i].set(a);
                a.inj.t0 = its; a.inj.w0 = F[it2 + 1]; a.inj.w1 = F[h + it2 + 1];
                if (it2 == 1) {          // sample its+1 = (p(2T+1) f[1] + p(2T) f[0]) + p(2T-1) f[h+1]
                    T = its + 1; a.tmode = 1; a.tw_o = F[1]; a.tw_c = F[0]; a.tw_n = F[h + 1];
                } else if (its == 0) {   // sample 0 = p(1) f[1] + p(0) f[0]
                    T = 0; a.tmode = 2; a.tw_o = 0.f; a.tw_c = F[1]; a.tw_n = F[0];
                } else {
                    a.tmode = 0;         // no coarse sample: a plain step
                }
                a.img_its = T;
            }
            if (T >= 0 || B.wave) B.step<1, EPI_TRI_IMG, 3>();
            else B.step<1, EPI_NONE, 4>();
        }
    B.run<1, EPI_TRI_IMG, 3>();
    check_launch();
}

// Born forward (adj = 0) or adjoint (adj = 1) of nb shots in lockstep, device
// inputs and outputs.  ds: per shot 5 device arrays of fine-time regular
// source traces (trace-major); dm: per shot 5 device pointers (forward: the
// perturbation slices; adjoint: the shot's own image, accumulated), both
// already offset to the shot's window; dr: per shot 5 device arrays of regular
// receiver traces (trace-major; written by the forward, read by the adjoint).
// Returns with the work queued on every engine's stream.
static void born_batch_queue(Engine* const* es, int nb, int adj, float* const* ds, float* const* dm,
                             float* const* dr, const ShotGeom* g) {
    Engine* e0 = es[0];
    if (!e0->tuned) engine_autotune(e0);
    ShotBatch B(es, nb);
    std::vector<PointList> src(nb), recp(nb);
    for (int i = 0; i < nb; i++) {
        Engine* e = es[i];
        err_reset(e);
        build_points(e, g[i].srcPos, g[i].nSrc, src[i]);
        build_points(e, g[i].recPos, g[i].nRec, recp[i]);
        stage_in(e, ds + 5 * i, src[i].ld, e->ntw, e->sig_in);
    }
    B.base();
    batch_source(B, src, nullptr);
    B.base();
    if (!adj) {
        batch_scatter(B, recp, dm);
    } else {
        for (int i = 0; i < nb; i++)   // on each engine's stream, after phase 1 (batch_source joined out)
            stage_in(es[i], dr + 5 * i, recp[i].ld, es[i]->nts, es[i]->sig_in);
        batch_adjoint(B, recp, dm);
    }
    B.join_out();
    if (!adj)
        for (int i = 0; i < nb; i++) stage_out(es[i], recp[i].ld, es[i]->nts, es[i]->sig_out, dr + 5 * i);
}

static void batch_finish(Engine* const* es, int nb) {
    for (int i = 0; i < nb; i++) {
        EIO_CUDA(cudaStreamSynchronize(es[i]->st));
        stats_flush(es[i]);
        err_check(es[i]);
    }
}

void engine_born_batch_dev(Engine* const* es, int nb, int adj, float* const* ds, float* const* dm, float* const* dr,
                           const ShotGeom* g) {
    EIO_CUDA(cudaSetDevice(es[0]->device));
    born_batch_queue(es, nb, adj, ds, dm, dr, g);
    batch_finish(es, nb);
}

// The same with host inputs and outputs, as engine_born_shot: srcDtw per shot
// 5 host arrays of fine-time regular source traces; rec per shot 4 receiver
// interpolators; dataIrreg per shot host traces [5][nIrreg][nts] (written by
// the forward, read by the adjoint).  The receivers are interpolated on the GPU.
void engine_born_shots_batch(Engine* const* es, int nb, int adj, float* const* srcDtw, float* const* dm,
                             const ShotGeom* g, const SInterp* const* rec, float* const* dataIrreg) {
    EIO_CUDA(cudaSetDevice(es[0]->device));
    std::vector<float*> ds((size_t)5 * nb), dr((size_t)5 * nb);
    for (int i = 0; i < nb; i++) {
        Engine* e = es[i];
        for (int f = 0; f < 5; f++) {
            h2d(e, e->stage_a[f], srcDtw[5 * i + f], (size_t)g[i].nSrc[kFieldGrid[f]] * e->ntw);
            ds[5 * i + f] = e->stage_a[f].f();
        }
        stage_receivers(e, adj, g[i], rec + 4 * i, adj ? dataIrreg[i] : nullptr, dr.data() + 5 * i);
    }
    born_batch_queue(es, nb, adj, ds.data(), dm, dr.data(), g);
    if (!adj)
        for (int i = 0; i < nb; i++) return_receivers(es[i], rec + 4 * i, dataIrreg[i]);
    batch_finish(es, nb);
}

// the image buffers of this lane, offset to the current shot window
void engine_dm_window(Engine* e, float* out[5]) {
    for (int f = 0; f < 5; f++) out[f] = e->stage_c[f].f() + (long long)e->win_ix0 * e->nz;
}

void engine_nl_shot(Engine* e, int adj, float* const modelReg[5], const ShotGeom& g, const SInterp* const rec[4],
                    float* dataIrreg, float* wfld) {
    EIO_CUDA(cudaSetDevice(e->device));
    float* dm[5]; float* dr[5];
    size_t nm[5];
    for (int f = 0; f < 5; f++) {
        nm[f] = (size_t)g.nSrc[kFieldGrid[f]] * e->nts;
        if (!adj) h2d(e, e->stage_a[f], modelReg[f], nm[f]);
        else e->stage_a[f].ensure(std::max<size_t>(16, sizeof(float) * nm[f]));
        dm[f] = e->stage_a[f].f();
    }
    stage_receivers(e, adj, g, rec, dataIrreg, dr);
    float* wdev = nullptr;
    const size_t wcount = (size_t)5 * e->nts * e->n;
    if (wfld) {
        e->wsave.ensure(sizeof(float) * wcount);
        EIO_CUDA(cudaMemsetAsync(e->wsave.p, 0, sizeof(float) * wcount, e->st));
        wdev = e->wsave.f();
    }
    engine_nl(e, adj, dm, dr, g, wdev);
    if (wfld) d2h(e, wfld, e->wsave, wcount);
    if (!adj) return_receivers(e, rec, dataIrreg);
    else
        for (int f = 0; f < 5; f++) d2h(e, modelReg[f], e->stage_a[f], nm[f]);
    EIO_CUDA(cudaStreamSynchronize(e->st));
}

}  // namespace eio

// ============================================================================
// Allocation-free nonlinear forward propagation (eio_nl_fwd_noalloc).
//
// Some callers cannot call cudaMalloc: code whose device memory is owned by
// another allocator (a framework's caching allocator that must see every
// byte), processes that forbid allocation after start-up (real-time or
// latency-critical services), or plug-ins that must not grow the device
// footprint of their host process.  For them this entry point runs the same
// nonlinear forward propagation as eio_nl_fwd_reg_dev with the same kernels,
// but every scratch buffer (both wavefield time levels, the taper tables, the
// sparse point lists and the time-major trace copies) lives in ONE
// file-scope device array of fixed size.  The array is reserved when the
// library's device code is loaded on a GPU and stays reserved on every GPU
// that loads it until the process exits.  The caller passes the inputs
// (medium, source traces) and the output (receiver traces) in its own device
// memory.  Calls share the array: two calls that overlap on the GPU (other
// host threads, other streams) race on it and must be serialised by the
// caller.
// ============================================================================
namespace eio {
namespace noalloc {

constexpr long long MAX_CELLS = 262144;        // nz * nx (e.g. 312 x 520 fits)
constexpr int MAX_AXIS = 16384;                // nz, nx each
constexpr long long MAX_SIGNAL = 4LL << 20;    // floats of time-major trace copies (sources + receivers)
constexpr int MAX_TILES = 8192;                // tile buckets per point list
constexpr int MAX_POINTS = 65536;              // entries per point list

constexpr long long OFF_WF = 0;
constexpr long long OFF_TAPER = OFF_WF + 10 * MAX_CELLS;
constexpr long long OFF_SIG = OFF_TAPER + 2LL * MAX_AXIS;
constexpr long long OFF_TS = OFF_SIG + MAX_SIGNAL;                   // 2 x (MAX_TILES + 1) ints
constexpr long long OFF_ENT = OFF_TS + 2LL * (MAX_TILES + 4);        // 2 x MAX_POINTS PointEntry
constexpr long long TOTAL = OFF_ENT + 2LL * MAX_POINTS * 2;          // in 4-byte words

static __device__ __align__(256) float g_noalloc_scratch[TOTAL];

static std::mutex g_mu;
// per device ordinal: the address found at set-up and the id of the CUDA
// context it belongs to (a cudaDeviceReset ends that context; the next one
// loads the library's device code anew, possibly at another address)
struct ScratchSlot {
    unsigned long long ctx = 0;
    float* p = nullptr;
};
static ScratchSlot g_dev_addr[256];

// id of the context current on this thread (driver entry points through the
// runtime, so nothing links libcuda); false when there is none or the driver
// cannot tell
static bool current_context_id(unsigned long long* id) {
    static PFN_cuCtxGetCurrent_v4000 get_cur = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_cur = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(p);
    }
    if (!get_cur || !get_id) return false;
    CUcontext c = nullptr;
    if (get_cur(&c) != CUDA_SUCCESS || !c) return false;
    return get_id(c, id) == CUDA_SUCCESS;
}

// Device address of the scratch array on the current device.  Set-up, once
// per device: the first call looks it up with cudaGetSymbolAddress (the host
// symbol itself is only a stand-in, never a device address) and keeps it
// with the id of the device's context; later calls in that context reuse it.
// After a cudaDeviceReset the context id differs and the address is looked
// up again.  Where the driver cannot report context ids, every call looks it
// up (cheap: no allocation).
static float* scratch_on_current_device() {
    int dev = 0;
    EIO_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) throw Error(EIO_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    unsigned long long id = 0;
    ScratchSlot& slot = g_dev_addr[dev];
    if (slot.p && current_context_id(&id) && id == slot.ctx) return slot.p;
    void* p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess || !p)
        throw Error(EIO_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(err));
    // the lookup made the device's primary context current on this thread
    if (current_context_id(&id)) {
        slot.ctx = id;
        slot.p = static_cast<float*>(p);
    } else {
        slot = ScratchSlot();
    }
    return static_cast<float*>(p);
}

// Per-tile buckets of the tile kernel (TZ x TX tiles numbered z-fastest).
static int bucket(int nz, int nx, const int* const pos[4], const int npos[4], std::vector<int>& ts,
                  std::vector<PointEntry>& ent, int ld[5]) {
    const int ntz = (nz - 2 * FAT + TZ - 1) / TZ, ntx = (nx - 2 * FAT) / TX, ntiles = ntz * ntx;
    std::vector<std::pair<int, PointEntry>> tmp;
    for (int f = 0; f < 5; f++) {
        const int g = kFieldGrid[f];
        ld[f] = npos[g];
        for (int k = 0; k < npos[g]; k++) {
            const int cell = pos[g][k];
            const int ix = cell / nz, iz = cell % nz;
            if (cell < 0 || ix < FAT || ix >= nx - FAT || iz < FAT || iz >= nz - FAT)
                throw Error(EIO_ERR_BOUNDS, "acquisition point " + std::to_string(cell) +
                                                " lies outside the updated interior of the grid");
            PointEntry pe;
            pe.key = (f << 16) | (((ix - FAT) % TX) << 8) | ((iz - FAT) % TZ);
            pe.col = k;
            tmp.push_back({((ix - FAT) / TX) * ntz + (iz - FAT) / TZ, pe});
        }
    }
    ts.assign(ntiles + 1, 0);
    for (auto& t : tmp) ts[t.first + 1]++;
    for (int i = 0; i < ntiles; i++) ts[i + 1] += ts[i];
    ent.resize(tmp.size());
    std::vector<int> cur(ts.begin(), ts.end() - 1);
    for (auto& t : tmp) ent[cur[t.first]++] = t.second;
    return ntiles;
}

static void nl_fwd(const eio_fd_params& p, float* const med[5], float* const model[5], float* const data[5],
                   const int* const srcPos[4], const int nSrc[4], const int* const recPos[4], const int nRec[4],
                   cudaStream_t st) {
    const int nz = p.nz, nx = p.nx, nts = p.nts;
    if (nz < 2 * FAT + 16 || nx < 2 * FAT + 16 || (nz - 2 * FAT) % 16 || (nx - 2 * FAT) % 16)
        throw Error(EIO_ERR_QC, "nz-2*fat and nx-2*fat must be positive multiples of 16");
    if ((long long)nz * nx > MAX_CELLS || nz > MAX_AXIS || nx > MAX_AXIS)
        throw Error(EIO_ERR_ARG, "grid " + std::to_string(nz) + "x" + std::to_string(nx) +
                                     " exceeds the allocation-free limit of " + std::to_string(MAX_CELLS) +
                                     " cells (and " + std::to_string(MAX_AXIS) + " per axis)");
    if (p.sub < 1 || 2 * p.sub >= SUB_MAX || nts < 2) throw Error(EIO_ERR_ARG, "invalid nts / sub");
    if (p.fat != 4 || p.blockSize != 16 || p.surfaceCondition != 0)
        throw Error(EIO_ERR_UNSUPPORTED, "fat 4, blockSize 16 and surfaceCondition 0 only");
    for (int k = 0; k < 4; k++)
        if (nSrc[k] < 0 || nRec[k] < 0) throw Error(EIO_ERR_ARG, "negative point count");
    // constants, same formulas as build_fdparam (nonlinearPropElasticGpuFunctions.cu:155-202)
    const int S = 2 * p.sub, h = S + 1;
    const int ntw = (nts - 1) * S + 1;
    float dz = p.dz, dx = p.dx;
    if (p.mod_par == 2) { dz *= 1000.f; dx *= 1000.f; }
    static const double C[4] = {1.196289062541883, -0.079752604188901, 0.009570312506634, -6.975446437140719e-04};
    std::vector<float> filt(2 * h);
    const float sc = std::sqrt(float(ntw) / float(nts));
    for (int i = 0; i < h; i++) {
        const float a0 = (float)(1.0 - 1.0 * i / S), b0 = (float)(1.0 - a0);
        filt[i] = (float)(a0 * (1.0 / sc));
        filt[i + h] = (float)(b0 * (1.0 / sc));
    }
    const int minPad = std::min(std::min(p.zPadMinus, p.zPadPlus), std::min(p.xPadMinus, p.xPadPlus));
    if (minPad < 0 || minPad >= PAD_MAX) throw Error(EIO_ERR_QC, "**** ERROR: Padding value is too high ****");
    std::vector<float> damp(std::max(minPad, 1), 1.f), tz(nz, 1.f), tx(nx, 1.f);
    for (int i = 0; i < minPad; i++) {
        float arg = (float)(M_PI / (1.0 * minPad) * 1.0 * (minPad - i));
        damp[i] = (float)(p.alphaCos + (1.0 - p.alphaCos) * std::cos(arg));
    }
    for (int iz = FAT; iz < nz - FAT; iz++) {
        const int d = std::min(iz - FAT, nz - iz - 1 - FAT);
        if (d < minPad) tz[iz] = damp[d];
    }
    for (int ix = FAT; ix < nx - FAT; ix++) {
        const int d = std::min(ix - FAT, nx - ix - 1 - FAT);
        if (d < minPad) tx[ix] = damp[d];
    }
    // sparse point lists
    std::vector<int> ts_i, ts_e;
    std::vector<PointEntry> en_i, en_e;
    int ld_i[5], ld_e[5];
    const int ntiles = bucket(nz, nx, srcPos, nSrc, ts_i, en_i, ld_i);
    bucket(nz, nx, recPos, nRec, ts_e, en_e, ld_e);
    if (ntiles > MAX_TILES) throw Error(EIO_ERR_ARG, "too many tiles for the allocation-free scratch");
    if ((long long)en_i.size() > MAX_POINTS || (long long)en_e.size() > MAX_POINTS)
        throw Error(EIO_ERR_ARG, "more than " + std::to_string(MAX_POINTS) + " sparse points in one list");
    long long sig_total = 0;
    for (int f = 0; f < 5; f++) sig_total += (long long)(ld_i[f] + ld_e[f]) * nts;
    if (sig_total > MAX_SIGNAL)
        throw Error(EIO_ERR_ARG, "source + receiver traces (" + std::to_string(sig_total) +
                                     " floats) exceed the allocation-free limit of " + std::to_string(MAX_SIGNAL));

    // carve the scratch array
    float* base = scratch_on_current_device();
    const long long n = (long long)nz * nx;
    float* wf = base + OFF_WF;
    float* dampz = base + OFF_TAPER;
    float* dampx = dampz + nz;
    float* sig = base + OFF_SIG;
    int* ts_dev_i = reinterpret_cast<int*>(base + OFF_TS);
    int* ts_dev_e = ts_dev_i + (MAX_TILES + 2);
    PointEntry* ent_dev_i = reinterpret_cast<PointEntry*>(base + OFF_ENT);
    PointEntry* ent_dev_e = ent_dev_i + MAX_POINTS;
    float* sin_f[5];
    float* sout_f[5];
    {
        float* q = sig;
        for (int f = 0; f < 5; f++) { sin_f[f] = q; q += (long long)ld_i[f] * nts; }
        for (int f = 0; f < 5; f++) { sout_f[f] = q; q += (long long)ld_e[f] * nts; }
    }
    // set-up copies and clears (no allocation anywhere below)
    EIO_CUDA(cudaMemcpyAsync(dampz, tz.data(), sizeof(float) * nz, cudaMemcpyHostToDevice, st));
    EIO_CUDA(cudaMemcpyAsync(dampx, tx.data(), sizeof(float) * nx, cudaMemcpyHostToDevice, st));
    EIO_CUDA(cudaMemcpyAsync(ts_dev_i, ts_i.data(), sizeof(int) * ts_i.size(), cudaMemcpyHostToDevice, st));
    EIO_CUDA(cudaMemcpyAsync(ts_dev_e, ts_e.data(), sizeof(int) * ts_e.size(), cudaMemcpyHostToDevice, st));
    if (!en_i.empty())
        EIO_CUDA(cudaMemcpyAsync(ent_dev_i, en_i.data(), sizeof(PointEntry) * en_i.size(), cudaMemcpyHostToDevice, st));
    if (!en_e.empty())
        EIO_CUDA(cudaMemcpyAsync(ent_dev_e, en_e.data(), sizeof(PointEntry) * en_e.size(), cudaMemcpyHostToDevice, st));
    EIO_CUDA(cudaMemsetAsync(wf, 0, sizeof(float) * 10 * n, st));   // both time levels start at zero
    for (int f = 0; f < 5; f++) {
        if (ld_e[f]) EIO_CUDA(cudaMemsetAsync(sout_f[f], 0, sizeof(float) * ld_e[f] * nts, st));
        if (ld_i[f]) {
            dim3 b(32, 8), g((nts + 31) / 32, (ld_i[f] + 31) / 32);
            k_transpose<<<g, b, 0, st>>>(model[f], sin_f[f], ld_i[f], nts);
        }
    }
    StepArgs a;
    memset(&a, 0, sizeof(a));
    for (int f = 0; f < 5; f++) a.par[f] = med[f];
    a.dampz = dampz;
    a.dampx = dampx;
    a.nz = nz;
    a.nx = nx;
    a.ntz = (nz - 2 * FAT + TZ - 1) / TZ;
    for (int k = 0; k < 4; k++) { a.cz[k] = (float)(C[k] / dz); a.cx[k] = (float)(C[k] / dx); }
    if (!en_i.empty()) {
        a.inj.tile_start = ts_dev_i;
        a.inj.ent = ent_dev_i;
        for (int f = 0; f < 5; f++) { a.inj.sig[f] = sin_f[f]; a.inj.ld[f] = ld_i[f]; }
    }
    if (!en_e.empty()) {
        a.ext.tile_start = ts_dev_e;
        a.ext.ent = ent_dev_e;
        for (int f = 0; f < 5; f++) { a.ext.sig[f] = sout_f[f]; a.ext.ld[f] = ld_e[f]; }
    }
    float* p0[5];
    float* p1[5];
    for (int f = 0; f < 5; f++) { p0[f] = wf + f * n; p1[f] = wf + (5 + f) * n; }
    for (int its = 0; its < nts - 1; its++)
        for (int it2 = 1; it2 < S + 1; it2++) {
            for (int f = 0; f < 5; f++) { a.o[f] = p0[f]; a.c[f] = p1[f]; }
            a.inj.t0 = its; a.inj.w0 = filt[it2 - 1]; a.inj.w1 = filt[h + it2 - 1];
            a.ext.t0 = its; a.ext.w0 = filt[it2]; a.ext.w1 = filt[h + it2];
            k_step<0, EPI_NONE><<<ntiles, NT, 0, st>>>(a);
            std::swap(p0, p1);
        }
    for (int f = 0; f < 5; f++) {
        if (!ld_e[f]) continue;
        dim3 b(32, 8), g((ld_e[f] + 31) / 32, (nts + 31) / 32);
        k_transpose<<<g, b, 0, st>>>(sout_f[f], data[f], nts, ld_e[f]);
    }
    cudaError_t lerr = cudaGetLastError();
    if (lerr != cudaSuccess) throw Error(EIO_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(lerr));
    EIO_CUDA(cudaStreamSynchronize(st));
}

}  // namespace noalloc
}  // namespace eio

extern "C" __attribute__((visibility("default"))) int eio_nl_fwd_noalloc(
    const eio_fd_params* p, float* const medium[5], float* const model[5], float* const data[5],
    const int* const srcPos[4], const int nSrc[4], const int* const recPos[4], const int nRec[4], void* stream) {
    try {
        if (!p || !medium || !model || !data || !srcPos || !nSrc || !recPos || !nRec)
            throw eio::Error(EIO_ERR_ARG, "null argument");
        eio::noalloc::nl_fwd(*p, medium, model, data, srcPos, nSrc, recPos, nRec, static_cast<cudaStream_t>(stream));
        return EIO_OK;
    } catch (const eio::Error& e) {
        eio::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        eio::set_last_error(e.what());
        return EIO_ERR_ARG;
    }
}
