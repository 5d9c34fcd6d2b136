// Internal declarations shared by the host-preparation code (eio_host.cpp) and
// the device engine (eio_engine.cu).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "eio_b200.h"

namespace eio {

constexpr int SUB_MAX = 100;   // varDeclare.h:11 (2*sub must stay below it)
constexpr int PAD_MAX = 500;   // varDeclare.h:10

// message returned by eio_last_error() on the calling thread
void set_last_error(const std::string& msg);

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// ---------------------------------------------------------------- host prep
struct FdParam {
    eio_fd_params p;
    int S = 0;            // internal sub-steps per coarse sample (2*sub)
    int ntw = 0;
    float dtw = 0.f;
    int minPad = 0;
    float zc[4], xc[4];   // FD coefficients
    std::vector<float> filt;   // 2*(S+1) time-interpolation filter
    std::vector<float> damp;   // [minPad] cosine taper
    float dts_inv = 0.f;       // Born: 1/(2 dts)
    float minVpVs = 0.f, maxVpVs = 0.f;
    std::vector<float> par[5]; // rhoxDtw, rhozDtw, lamb2MuDtw, lambDtw, muxzDtw
    std::vector<float> fsc;    // [nx] free surface: sigmaxx coefficient on the surface row
};

// Builds the FD parameters, checks the QC of fdParamElastic and prepares the
// scaled staggered medium.  Throws Error(EIO_ERR_QC, ...) on QC failure.
void build_fdparam(const eio_fd_params& p, const float* elasticParam, FdParam& out);
void stagger_x(int adj, int add, int nz, int nx, float* model, float* data);
void stagger_z(int adj, int add, int nz, int nx, float* model, float* data);
void time_interp(int adj, int add, int nts, float dts, float ots, int S, int nDev, float* coarse, float* fine);

struct SInterp {
    int nIrreg = 0, nReg = 0, nft = 0, nt = 0;
    std::vector<int> gpi;      // [nIrreg*nft]
    std::vector<float> w;      // [nIrreg*nft]
    std::vector<int> slot;     // unique slot of every (device, filter) entry
    std::vector<int> uniq;     // [nReg] unique regular positions, first-seen order
    int nz = 0, nx = 0;
};
void build_sinterp(const float* zc, const float* xc, int nDev, int nz, float oz, float dz, int nx, float ox,
                   float dx, int nt, const std::string& method, int nFilt, int dipole, float zDip, float xDip,
                   SInterp& out);
void sinterp_forward(const SInterp& s, bool add, const float* reg, float* irreg);
void sinterp_adjoint(const SInterp& s, bool add, float* reg, const float* irreg);

// ---------------------------------------------------------------- device engine
struct Engine;   // opaque, defined in eio_engine.cu
Engine* engine_create(int device, const FdParam& fd);
void engine_destroy(Engine* e);
void engine_set_medium(Engine* e, const FdParam& fd);
void engine_set_checkpoint(Engine* e, int mode);
// step-kernel selection: kind 0 tile kernel, 1 TMA sweep (tz, cw, cpr); autotune times the candidates
void engine_set_kernel(Engine* e, int kind, int tz, int cw, int cpr);
void engine_set_wait_limit(Engine* e, long long polls);   // < 0: the default
void engine_share_medium(Engine* e, const Engine* from);   // e's kernels read from's medium arrays
void engine_set_persistent(Engine* e, int mask);          // phases of the shot groups run as persistent loops
int engine_get_persistent(const Engine* e);
long long engine_get_wait_limit(const Engine* e);
void engine_get_kernel(const Engine* e, int* kind, int* tz, int* cw, int* cpr);
void engine_autotune(Engine* e);
void* engine_stream(Engine* e);
// launch statistics: enable = 1/0 (-1 leaves it), reset = 1 zeroes the counters after reading
void engine_set_graphs(Engine* e, int enable);
void engine_set_window(Engine* e, int ix0, int nxw);   // nxw = 0: the whole grid
bool engine_is_tuned(const Engine* e);
size_t engine_history_bytes(const Engine* e);
int engine_get_checkpoint(const Engine* e);
int engine_get_graphs(const Engine* e);
size_t engine_cells(const Engine* e);
void engine_dm_ptrs(Engine* e, float* out[5]);          // this lane's own image buffers
void engine_dm_add(Engine* e, float* const dst[5]);     // dst += this lane's image (device)
int engine_window_ix0(const Engine* e);
// FP64 sum of x*y (op 0) or (x-y)^2 (op 1) over n values (dtype 0 FP32, 1 FP64) on GPU `device`
double reduce64(int device, int op, int dtype, const void* x, const void* y, long long n, bool on_device);

// learned preconditioner (eio_cnn.cu); device pointers, work queued on `stream`
constexpr int CNN_MSE_PARTIALS = 1024;
void cnn_conv3x3(int n, int h, int w, int cin, int cout, const void* x, const void* wt, const void* mask, int relu,
                 void* y, float* y32, void* stream);
long long cnn_wgrad_scratch(int n, int h, int w, int cin, int cout);
void cnn_set_conv_path(int path);
int cnn_get_conv_path();
int cnn_status(int reset);
void cnn_set_wait_limit(long long polls);   // < 0: the default
long long cnn_get_wait_limit();
void cnn_conv3x3_wgrad(int n, int h, int w, int cin, int cout, const void* x, const void* dy, float* dw,
                       float* scratch, long long scratchFloats, void* stream);
void cnn_flip(int cin, int cout, const void* w, void* wt, void* stream);
void cnn_mse(long long npix, int c, int nc, const float* y32, const float* target, void* dz, double* part,
             double* loss, void* stream);
void cnn_adam(long long n, float* p, float* m, float* v, const float* g, float lr, float b1, float b2, float eps,
              int step, void* pb, void* stream);
void engine_stats(Engine* e, int enable, int reset, long long* launches, long long* step_launches, double* step_ms,
                  long long* pair_launches, double* pair_ms);

struct ShotGeom {
    const int* srcPos[4]; int nSrc[4];
    const int* recPos[4]; int nRec[4];
};
// all float arrays are device pointers
// wfld (device, [nts][5][nx][nz], zeroed by the caller) receives the coarse
// samples of every fine step's new level when not null
void engine_nl(Engine* e, int adj, float* const model[5], float* const data[5], const ShotGeom& g,
               float* wfld = nullptr);
void engine_nl_record(Engine* e, float* const model[5], float* const data[5], const ShotGeom& g);
// reuse_history: the history of the shot is already in place (engine_nl_record); srcDtw unused
void engine_born(Engine* e, int adj, float* const srcDtw[5], float* const dm[5], float* const data[5],
                 const ShotGeom& g, bool reuse_history = false);
// host-pointer convenience wrappers (copy in/out through the engine's staging buffers)
// wfld: host [nts][5][nx][nz], overwritten with the saved wavefield when not null
void engine_nl_host(Engine* e, int adj, float* const model[5], float* const data[5], const ShotGeom& g,
                    float* wfld = nullptr);
// Multi-shot paths: the Born perturbation / gradient grids stay on the device
// across shots (stage with engine_dm_upload or engine_dm_zero, read back with
// engine_dm_download); receiver traces go in and out as irregular traces
// [5][nIrreg][nts] on the host, interpolated on the device with rec[grid].
void engine_dm_upload(Engine* e, float* const dm[5]);
void engine_dm_zero(Engine* e);
void engine_dm_download(Engine* e, float* const dm[5]);
void engine_born_shot(Engine* e, int adj, float* const srcDtw[5], const ShotGeom& g, const SInterp* const rec[4],
                      float* dataIrreg);
// modelReg: regular source traces, read (forward) or written (adjoint)
double engine_fwi_shot(Engine* e, float* const modelReg[5], const ShotGeom& g, const SInterp* const rec[4],
                       float* dataIrreg, float* resid, double (*residual)(void*, const float*, float*), void* ctx,
                       float* const dm[5]);
void engine_dm_window(Engine* e, float* out[5]);
constexpr int STEP_BATCH = 8;   // shots of one lockstep launch (k_step_batch)
void engine_nl_shots_batch(Engine* const* es, int nb, int adj, float* const* modelReg, const ShotGeom* g,
                           const SInterp* const* rec, float* const* dataIrreg);
// Born forward / adjoint of nb shots in lockstep (one engine per shot; sub = 1,
// FP32 history, no free surface); dm: per shot 5 device pointers (the
// perturbation, or the shot's own image), offset to the shot's window.
// Host traces (receivers interpolated on the GPU, like engine_born_shot):
void engine_born_shots_batch(Engine* const* es, int nb, int adj, float* const* srcDtw, float* const* dm,
                             const ShotGeom* g, const SInterp* const* rec, float* const* dataIrreg);
// device traces: ds fine-time regular sources, dr regular receiver traces, per shot 5 arrays each
void engine_born_batch_dev(Engine* const* es, int nb, int adj, float* const* ds, float* const* dm, float* const* dr,
                           const ShotGeom* g);
bool engine_batchable(const Engine* e);   // sub = 1 and an FP32 history
long long engine_step_cells(const Engine* e);
void engine_set_history_where(Engine* e, int where);
int engine_history_where(const Engine* e);
void set_device_memory_cap(long long bytes);
long long device_memory_used();
void engine_nl_shot(Engine* e, int adj, float* const modelReg[5], const ShotGeom& g, const SInterp* const rec[4],
                    float* dataIrreg, float* wfld = nullptr);
void engine_born_host(Engine* e, int adj, float* const srcDtw[5], float* const dm[5], float* const data[5],
                      const ShotGeom& g);

// U-Net layers (eio_gemm.cu)
void gemm_bf16(long long M, long long N, long long K, const void* A, long long lda, const void* B, long long ldb,
               float* C32, void* C16, const void* mask, int relu, int splits, float* scratch, void* stream);
void gemm_set_wait_limit(long long polls);
int gemm_status(int reset);
void unet_set_tma(int on);
int unet_get_tma();
void unet_conv3x3(int n, int h, int w, int cin, int cout, const void* x, const void* wt, float* y32, void* y16,
                  int relu, void* stream);
long long unet_wgrad_scratch(int n, int h, int w, int cin, int cout);
void unet_conv3x3_wgrad(int n, int h, int w, int cin, int cout, const void* x, const void* dz, float* dw,
                        float* scratch, long long scratch_floats, void* stream);
void unet_flip(int cout, int cin, const void* w, void* wf, void* stream);
void unet_resample(int op, int n, int h, int w, int c, const void* in, void* out, int add, void* stream);
void unet_concat(int adj, long long pixels, int ca, int cb, void* a, int add_a, void* b, int add_b, void* z,
                 void* stream);
void unet_relu_adj(long long n, const void* src, const void* mask, void* dst, int add, void* stream);
}  // namespace eio
