// Tensor-core GEMM and the layer kernels of the U-Net preconditioner
// (precond.UNet; no reference counterpart).
//
// k_gemm_tc: C[M][N] = A[M][K] . B[N][K]^T, BF16 operands, FP32 accumulation
// in tensor memory, on tcgen05.  A tile of C is 128 x BN (BN = 32, 64, 128 or
// 256 TMEM columns, twice over); its K range (the whole K, or one slice of a
// split-K grid) streams through a 4- to 8-stage shared-memory ring in
// 64-wide slices, each filled by 16-byte cp.async copies into the
// non-swizzled UMMA operand layouts (K-major, or MN-major for operands whose
// rows are contiguous in memory) and consumed by four tcgen05.mma.kind::f16
// (M = 128, N = BN, K = 16) that one thread issues and commits to the
// stage's mbarrier.  A stage is refilled once the MMAs that read it have
// arrived.  Rows past M, columns past N and K past K read zeros.  The
// epilogue reads the accumulator with tcgen05.ld (each warp its 32 lanes) and
// writes FP32 and/or BF16 (optional ReLU, or a multiply by (mask > 0), the
// ReLU derivative of the backward pass).  Split-K grids write FP32 partials
// that k_sum_splits adds in a fixed order.  The kernel is persistent: CTA b
// takes tiles b, b + grid, ...; the copy ring runs on across tile boundaries
// and two TMEM accumulators let a tile's epilogue overlap the next tile's
// MMAs.  Every mbarrier wait is bounded; after a timeout the CTA drains its
// MMAs and copies, frees its tensor memory and returns with the error flag
// set (eio_gemm_status).
//
// Convolutions (3x3, stride 1, zero padding 1, NHWC) are implicit GEMMs on
// the same kernel, the operand chunks gathered by the copy loop (no column
// matrix in memory):
// forward  Y[p][co]   = sum_{tap, ci} X[p + off(tap)][ci] W[co][tap][ci]   (A rows = pixels, K-major gather)
// data     dX[p][ci]  = the same with dY and the flipped weights Wf[ci][tap][co]
// weights  dW^T[tap ci][co] = sum_p X[p + off(tap)][ci] dY[p][co]          (A gathered MN-major, B = dY MN-major)
// with W stored [co][tap][ci], tap = 3 dy + dx; the weight gradient splits
// the pixels over the grid and its partial sums are added (and transposed)
// in a fixed order.  Small kernels, 8 channels (16 bytes) per thread: weight
// flip, 2x2 average pooling and nearest 2x upsampling (forward and adjoint),
// channel concatenation and its adjoint (adding into the skip connection's
// gradient), the ReLU derivative.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "eio_internal.h"

namespace eio {

namespace {

using bf16 = __nv_bfloat16;

#define GCUDA(x)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) throw Error(EIO_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr int G_BM = 128;                    // rows of a CTA tile (TMEM lanes)
constexpr int G_BK = 64;                     // K of one ring stage
constexpr int G_THREADS = 128;
constexpr long long G_WAIT = 1LL << 22;      // default polls of an accumulator wait
constexpr long long G_DRAIN = 1LL << 24;     // polls of a drain wait after a timeout

__device__ int g_gemm_err;                   // 1: a wait timed out (drained), 2: the drain timed out too
long long g_gemm_wait = G_WAIT;

// Where an operand's 16-byte chunks come from.
enum : int {
    OP_PLAIN = 0,   // K-major matrix [rows][ld]
    OP_CONV = 1,    // K-major, rows = pixels p of an NHWC tensor X, K = tap * C + c: X[p + off(tap)][c] (0 outside)
    OP_CONVT = 2,   // MN-major, rows = tap * C + c, K = pixels p: X[p + off(tap)][c] (0 outside)
    OP_MN = 3       // MN-major matrix stored [K][ld] (the rows contiguous)
};

template <int BN>
struct GCfg {
    static constexpr int STAGES = BN >= 256 ? 4 : (BN >= 128 ? 6 : 8);
    static constexpr int A_BYTES = G_BM * G_BK * 2;
    static constexpr int B_BYTES = BN * G_BK * 2;
    static constexpr int STAGE = A_BYTES + B_BYTES;
    static constexpr int BAR = STAGES * STAGE;            // STAGES mbarriers, then the TMEM address
    static constexpr int SMEM = BAR + 8 * STAGES + 16;
};

__device__ __forceinline__ unsigned g_smem(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ unsigned long long g_desc(unsigned addr, unsigned lbo, unsigned sbo)
{
    return (unsigned long long)((addr >> 4) & 0x3FFF) | ((unsigned long long)((lbo >> 4) & 0x3FFF) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Operand descriptor of the kk-th K16 step of a stage holding `rows` rows.
// Non-swizzled layouts of core matrices (8 rows x 16 bytes), the leading
// byte offset being the K-direction stride between core matrices and the
// stride byte offset the M/N-direction one:
//   K-major:  chunk (row r, K chunk c) at (c * rows + r) * 16       (LBO rows x 16, SBO 128)
//   MN-major: chunk (row group g, k) at (k / 16) * rows * 32 + (2 g + (k / 8) % 2) * 128 + (k % 8) * 16
//             (LBO 128, SBO 256)
// Both put the kk-th K16 step at byte kk * rows * 32.
__device__ __forceinline__ unsigned long long g_opdesc(unsigned base, int rows, int kk, bool mn)
{
    return mn ? g_desc(base + (unsigned)(kk * rows * 32), 128, 256)
              : g_desc(base + (unsigned)(kk * rows * 32), (unsigned)(rows * 16), 128);
}
__device__ __forceinline__ unsigned g_mn_off(int rows, int g, int k)
{
    return (unsigned)((k >> 4) * rows * 32 + (2 * g + ((k >> 3) & 1)) * 128 + (k & 7) * 16);
}

// instruction descriptor: F32 accumulator, BF16 A and B (K-major unless
// amn / bmn: MN-major), N = BN, M = 128
template <int BN>
__device__ __forceinline__ unsigned g_idesc(bool amn, bool bmn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (amn ? 1u << 15 : 0u) | (bmn ? 1u << 16 : 0u) |
           ((unsigned)(BN >> 3) << 17) | ((unsigned)(G_BM >> 4) << 24);
}

__device__ __forceinline__ bool g_wait(unsigned bar, unsigned parity, long long limit)
{
    for (long long it = 0; it < limit; it++) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void g_ld16(unsigned taddr, float* v)
{
    unsigned r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// 16 bytes from global memory into shared memory, zeros when !in (src is then
// only a valid address, nothing is read)
__device__ __forceinline__ void g_cp16(unsigned dst, const void* src, bool in)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(in ? 16 : 0) : "memory");
}

struct GemmArgs {
    const bf16* A; const bf16* B;
    long long M, N, K, lda, ldb;
    int amode, bmode;        // OP_PLAIN / OP_CONV / OP_CONVT for A, OP_PLAIN / OP_MN for B
    int cw, ch, cc;          // width, height, channels of the NHWC tensor A gathers from
    float* C32;              // optional [splits][M][N] (ldc = N)
    bf16* C16;               // optional [M][N]
    const bf16* mask;        // optional [M][N]: C *= (mask > 0)
    int relu;
    long long kchunk;        // K per split (a multiple of G_BK)
    int mt, nt, splits;      // tile grid: M tiles, N tiles, K splits
    long long wait;
};

// Source pixel of tap t (3 dy + dx) for pixel p at (y, x), or -1 outside the
// image (zero padding)
__device__ __forceinline__ long long g_tap_src(long long p, int y, int x, int tap, int H, int W)
{
    const int dy = tap / 3 - 1, dx = tap - 3 * (tap / 3) - 1;
    const int sy = y + dy, sx = x + dx;
    return (sy >= 0 && sy < H && sx >= 0 && sx < W) ? p + (long long)dy * W + dx : -1;
}

// Slice [k0, k0 + 64) (K < ke) of A's rows [m0, m0 + 128) into stage dst.
// Pixel indices stay below 2^31 + 128 (pixel counts are capped at 2^31).
__device__ __forceinline__ void g_load_a(const GemmArgs& g, long long m0, long long k0, long long ke, unsigned dst)
{
    const int tid = threadIdx.x;
    if (g.amode == OP_PLAIN) {
        const long long row = m0 + tid;
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const long long k = k0 + 8 * c;
            const bool in = row < g.M && k < ke;
            g_cp16(dst + (unsigned)(c * G_BM + tid) * 16, in ? g.A + row * g.lda + k : g.A, in);
        }
    } else if (g.amode == OP_CONV) {
        // thread = pixel row; 8 consecutive K chunks (channel groups of one or more taps)
        const long long p = m0 + tid;
        const unsigned pu = (unsigned)p, cw = (unsigned)g.cw;
        const int x = (int)(pu % cw), y = (int)((pu / cw) % (unsigned)g.ch);
        int tap = (int)((unsigned)k0 / (unsigned)g.cc), c8 = (int)(k0 - (long long)tap * g.cc);
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const long long k = k0 + 8 * c;
            long long src = -1;
            if (p < g.M && k < ke) src = g_tap_src(p, y, x, tap, g.ch, g.cw);
            g_cp16(dst + (unsigned)(c * G_BM + tid) * 16, src >= 0 ? g.A + src * g.cc + c8 : g.A, src >= 0);
            c8 += 8;
            if (c8 == g.cc) {
                c8 = 0;
                tap++;
            }
        }
    } else {   // OP_CONVT: rows tap * C + c, K = pixels; thread = pixel k0 + tid % 64, row groups tid / 64 + 2 j
        const int kp = tid & 63;
        const long long p = k0 + kp;
        const unsigned pu = (unsigned)p, cw = (unsigned)g.cw;
        const int x = (int)(pu % cw), y = (int)((pu / cw) % (unsigned)g.ch);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int gr = (tid >> 6) + 2 * j;
            const long long m = m0 + 8 * gr;
            long long src = -1;
            int c8 = 0;
            if (p < ke && m < g.M) {
                const int tap = (int)((unsigned)m / (unsigned)g.cc);
                c8 = (int)(m - (long long)tap * g.cc);
                src = g_tap_src(p, y, x, tap, g.ch, g.cw);
            }
            g_cp16(dst + g_mn_off(G_BM, gr, kp), src >= 0 ? g.A + src * g.cc + c8 : g.A, src >= 0);
        }
    }
}

// Slice [k0, k0 + 64) of B's rows [n0, n0 + BN) into stage dst
template <int BN>
__device__ __forceinline__ void g_load_b(const GemmArgs& g, long long n0, long long k0, long long ke, unsigned dst)
{
    const int tid = threadIdx.x;
    if (g.bmode == OP_PLAIN) {
#pragma unroll
        for (int i = tid; i < BN * 8; i += G_THREADS) {
            const int r = i % BN, c = i / BN;
            const long long row = n0 + r, k = k0 + 8 * c;
            const bool in = row < g.N && k < ke;
            g_cp16(dst + (unsigned)(c * BN + r) * 16, in ? g.B + row * g.ldb + k : g.B, in);
        }
    } else {   // OP_MN: B[k][n] at k * ldb + n
#pragma unroll
        for (int i = tid; i < BN * 8; i += G_THREADS) {
            const int kp = i & 63, gr = i >> 6;
            const long long k = k0 + kp, n = n0 + 8 * gr;
            const bool in = k < ke && n < g.N;
            g_cp16(dst + g_mn_off(BN, gr, kp), in ? g.B + k * g.ldb + n : g.B, in);
        }
    }
}

// Accumulator buffer -> C (rows of this warp's 32 TMEM lanes)
template <int BN>
__device__ __forceinline__ void g_epilogue(const GemmArgs& g, unsigned tbuf, long long m0, long long n0, int z)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long row = m0 + warp * 32 + lane;
    float* c32 = g.C32 ? g.C32 + (long long)z * g.M * g.N : nullptr;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
        float v[16];
        g_ld16(tbuf + ((unsigned)(warp * 32) << 16) + (unsigned)c, v);
        const long long col = n0 + c;
        if (row >= g.M || col >= g.N) continue;
        const int nv = (int)min((long long)16, g.N - col);
        const bool vec = nv == 16 && (g.N & 7) == 0;
        if (g.mask) {
            const bf16* mk = g.mask + row * g.N + col;
            if (vec) {
                uint4 u[2];
                u[0] = *reinterpret_cast<const uint4*>(mk);
                u[1] = *reinterpret_cast<const uint4*>(mk + 8);
                const bf16* mb = reinterpret_cast<const bf16*>(u);
#pragma unroll
                for (int i = 0; i < 16; i++)
                    if (!(__bfloat162float(mb[i]) > 0.f)) v[i] = 0.f;
            } else {
                for (int i = 0; i < nv; i++)
                    if (!(__bfloat162float(mk[i]) > 0.f)) v[i] = 0.f;
            }
        } else if (g.relu) {
#pragma unroll
            for (int i = 0; i < 16; i++) v[i] = fmaxf(v[i], 0.f);
        }
        if (c32) {
            float* dst = c32 + row * g.N + col;
            if (vec) {
#pragma unroll
                for (int i = 0; i < 16; i += 4)
                    *reinterpret_cast<float4*>(dst + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
            } else {
                for (int i = 0; i < nv; i++) dst[i] = v[i];
            }
        }
        if (g.C16) {
            bf16* dst = g.C16 + row * g.N + col;
            if (vec) {
                uint4 u[2];
                bf16* ub = reinterpret_cast<bf16*>(u);
#pragma unroll
                for (int i = 0; i < 16; i++) ub[i] = __float2bfloat16_rn(v[i]);
                *reinterpret_cast<uint4*>(dst) = u[0];
                *reinterpret_cast<uint4*>(dst + 8) = u[1];
            } else {
                for (int i = 0; i < nv; i++) dst[i] = __float2bfloat16_rn(v[i]);
            }
        }
    }
}

// Persistent tcgen05 GEMM (tile id: N tile fastest, then M tile, then K split)
template <int BN>
__global__ void __launch_bounds__(G_THREADS, 1) k_gemm_tc(const __grid_constant__ GemmArgs g)
{
    using Cf = GCfg<BN>;
    constexpr int S = Cf::STAGES;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem + Cf::BAR);
    unsigned* tslot = reinterpret_cast<unsigned*>(smem + Cf::BAR + 8 * S);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int tiles = g.mt * g.nt * g.splits;

    if (tid == 0) {
        for (int s = 0; s < S; s++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(g_smem(bar + s)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(g_smem(tslot)),
                     "r"(2 * BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *tslot;
    const unsigned s0 = g_smem(smem);
    auto stageA = [&](int s) { return s0 + (unsigned)(s * Cf::STAGE); };
    auto stageB = [&](int s) { return s0 + (unsigned)(s * Cf::STAGE + Cf::A_BYTES); };
    auto t_m0 = [&](int id) { return (long long)((id / g.nt) % g.mt) * G_BM; };
    auto t_n0 = [&](int id) { return (long long)(id % g.nt) * BN; };
    auto t_z = [&](int id) { return id / (g.nt * g.mt); };
    auto t_kb = [&](int id) { return (long long)t_z(id) * g.kchunk; };
    auto t_ke = [&](int id) { return min(g.K, t_kb(id) + g.kchunk); };
    auto t_kt = [&](int id) { return (int)((t_ke(id) - t_kb(id) + G_BK - 1) / G_BK); };

    // copy cursor: the next slice to load is slice l_t of tile l_tile, the
    // l_n-th of this CTA (stage l_n % S); one copy group per slice, empty
    // groups past the last tile
    int l_tile = blockIdx.x, l_t = 0, l_n = 0;
    auto load_next = [&]() {
        if (l_tile < tiles) {
            const int s = l_n % S;
            const long long k0 = t_kb(l_tile) + (long long)l_t * G_BK, ke = t_ke(l_tile);
            g_load_a(g, t_m0(l_tile), k0, ke, stageA(s));
            g_load_b<BN>(g, t_n0(l_tile), k0, ke, stageB(s));
            if (++l_t == t_kt(l_tile)) {
                l_t = 0;
                l_tile += gridDim.x;
            }
        }
        l_n++;
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    for (int i = 0; i < S - 1; i++) load_next();

    const bool amn = g.amode == OP_CONVT, bmn = g.bmode == OP_MN;
    const unsigned idesc = g_idesc<BN>(amn, bmn);
    bool bad = false;
    int q = 0, pend_a = -1, pend_b = -1, it = 0, prev = -1;
    for (int tile = blockIdx.x; tile < tiles && !bad; tile += gridDim.x, it++) {
        const int KT = t_kt(tile);
        const unsigned acc_buf = tmem + (unsigned)((it & 1) * BN);
        for (int t = 0; t < KT; t++, q++) {
            const int s = q % S;
            asm volatile("cp.async.wait_group %0;" ::"n"(S - 2) : "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                for (int kk = 0; kk < G_BK / 16; kk++) {
                    const unsigned long long ad = g_opdesc(stageA(s), G_BM, kk, amn);
                    const unsigned long long bd = g_opdesc(stageB(s), BN, kk, bmn);
                    const unsigned acc = (t | kk) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                        :
                        : "r"(acc_buf), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                        : "memory");
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 g_smem(bar + s))
                             : "memory");
            }
            pend_b = pend_a;
            pend_a = q;
            // the stage of slice q - 1 is refilled next: its MMAs must have read it
            if (q >= 1) {
                const int p = q - 1;
                const bool ok = g_wait(g_smem(bar + p % S), (unsigned)((p / S) & 1), g.wait);
                if (__syncthreads_or(!ok)) {
                    bad = true;
                    break;
                }
                pend_b = -1;
            }
            load_next();
            if (t == 0 && prev >= 0) {   // every MMA of the previous tile has completed
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                g_epilogue<BN>(g, tmem + (unsigned)(((it - 1) & 1) * BN), t_m0(prev), t_n0(prev), t_z(prev));
            }
        }
        prev = tile;
    }
    if (!bad && q > 0) {
        const int p = q - 1;
        const bool ok = g_wait(g_smem(bar + p % S), (unsigned)((p / S) & 1), g.wait);
        if (__syncthreads_or(!ok)) {
            bad = true;
        } else {
            pend_a = -1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            g_epilogue<BN>(g, tmem + (unsigned)(((it - 1) & 1) * BN), t_m0(prev), t_n0(prev), t_z(prev));
        }
    }
    if (bad) {
        // drain the MMAs that may still run and the copies in flight before the
        // tensor memory is freed and the CTA leaves
        bool drained = true;
        if (pend_a >= 0) drained = g_wait(g_smem(bar + pend_a % S), (unsigned)((pend_a / S) & 1), G_DRAIN) && drained;
        if (pend_b >= 0) drained = g_wait(g_smem(bar + pend_b % S), (unsigned)((pend_b / S) & 1), G_DRAIN) && drained;
        asm volatile("cp.async.wait_all;" ::: "memory");
        drained = !__syncthreads_or(!drained);
        if (tid == 0) atomicMax(&g_gemm_err, drained ? 1 : 2);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN) : "memory");
}

// out = sum_s part[s] in split order (FP32; optional ReLU, optional BF16
// copy); part is [splits][M][N], out [M][N], or [N][M] when trans
__global__ void __launch_bounds__(256) k_sum_splits(const float* __restrict__ part, int splits, long long M, long long N,
                                                   int trans, int relu, float* __restrict__ out, bf16* __restrict__ out16)
{
    const long long n = M * N;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float acc = 0.f;
        for (int s = 0; s < splits; s++) acc += part[(long long)s * n + i];
        if (relu) acc = fmaxf(acc, 0.f);
        const long long o = trans ? (i % N) * M + i / N : i;
        if (out) out[o] = acc;
        if (out16) out16[o] = __float2bfloat16_rn(acc);
    }
}

// Wf[ci][tap][co] = W[co][8 - tap][ci]
__global__ void k_flip_ct(const bf16* __restrict__ W, int Cout, int Cin, bf16* __restrict__ Wf)
{
    const long long total = 9LL * Cout * Cin;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int co = (int)(i % Cout);
        const long long r = i / Cout;
        const int tap = (int)(r % 9), ci = (int)(r / 9);
        Wf[i] = W[((long long)co * 9 + (8 - tap)) * Cin + ci];
    }
}

// 8 BF16 values (16 bytes) <-> FP32
struct F8 {
    float v[8];
};
__device__ __forceinline__ F8 ld8(const bf16* p)
{
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    const bf16* b = reinterpret_cast<const bf16*>(&u);
    F8 r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = __bfloat162float(b[i]);
    return r;
}
__device__ __forceinline__ void st8(bf16* p, const F8& f)
{
    uint4 u;
    bf16* b = reinterpret_cast<bf16*>(&u);
#pragma unroll
    for (int i = 0; i < 8; i++) b[i] = __float2bfloat16_rn(f.v[i]);
    *reinterpret_cast<uint4*>(p) = u;
}

// Thread i of the layer kernels handles the 8-channel chunk i of its output
// (or input) tensor; chunk counts stay below 2^31 (checked on the host).

// 2x2 average pooling y[n][h/2][w/2][c] of x[n][h][w][c] (h, w: the input size)
__global__ void __launch_bounds__(256) k_pool2(const bf16* __restrict__ x, int H, int W, int C, unsigned total,
                                              bf16* __restrict__ y)
{
    const unsigned c8 = (unsigned)C / 8, Wo = (unsigned)W / 2, Ho = (unsigned)H / 2;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const unsigned cc = i % c8, p = i / c8;
        const unsigned xo = p % Wo, r = p / Wo, yo = r % Ho, n = r / Ho;
        const long long b = (((long long)n * H + 2 * yo) * W + 2 * xo) * C + cc * 8;
        const F8 a = ld8(x + b), bb = ld8(x + b + C), c = ld8(x + b + (long long)W * C),
                 d = ld8(x + b + (long long)W * C + C);
        F8 o;
#pragma unroll
        for (int k = 0; k < 8; k++) o.v[k] = 0.25f * (a.v[k] + bb.v[k] + c.v[k] + d.v[k]);
        st8(y + (long long)i * 8, o);
    }
}
// its adjoint dx[n][y][x][c] (+)= dy[n][y/2][x/2][c] / 4 (h, w: the output size)
__global__ void __launch_bounds__(256) k_pool2_adj(const bf16* __restrict__ dy, int H, int W, int C, unsigned total,
                                                  bf16* __restrict__ dx, int add)
{
    const unsigned c8 = (unsigned)C / 8;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const unsigned cc = i % c8, p = i / c8;
        const unsigned x = p % (unsigned)W, r = p / (unsigned)W, y = r % (unsigned)H, n = r / (unsigned)H;
        F8 v = ld8(dy + (((long long)n * (H / 2) + y / 2) * (W / 2) + x / 2) * C + cc * 8);
        F8 o = add ? ld8(dx + (long long)i * 8) : F8{};
#pragma unroll
        for (int k = 0; k < 8; k++) o.v[k] = add ? o.v[k] + 0.25f * v.v[k] : 0.25f * v.v[k];
        st8(dx + (long long)i * 8, o);
    }
}
// nearest 2x upsampling y[n][2h][2w][c] = x[n][h][w][c] (h, w: the input size)
__global__ void __launch_bounds__(256) k_up2(const bf16* __restrict__ x, int H, int W, int C, unsigned total,
                                            bf16* __restrict__ y)
{
    const unsigned c8 = (unsigned)C / 8, W2 = 2u * W, H2 = 2u * H;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const unsigned cc = i % c8, p = i / c8;
        const unsigned xo = p % W2, r = p / W2, yo = r % H2, n = r / H2;
        *reinterpret_cast<uint4*>(y + (long long)i * 8) =
            *reinterpret_cast<const uint4*>(x + (((long long)n * H + yo / 2) * W + xo / 2) * C + cc * 8);
    }
}
// its adjoint dx[n][y][x][c] (+)= the sum of the four dy values it feeds (h, w: the output size)
__global__ void __launch_bounds__(256) k_up2_adj(const bf16* __restrict__ dy, int H, int W, int C, unsigned total,
                                                bf16* __restrict__ dx, int add)
{
    const unsigned c8 = (unsigned)C / 8;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const unsigned cc = i % c8, p = i / c8;
        const unsigned x = p % (unsigned)W, r = p / (unsigned)W, y = r % (unsigned)H, n = r / (unsigned)H;
        const long long b = (((long long)n * 2 * H + 2 * y) * 2 * W + 2 * x) * C + cc * 8;
        const F8 a = ld8(dy + b), bb = ld8(dy + b + C), c = ld8(dy + b + 2LL * W * C), d = ld8(dy + b + 2LL * W * C + C);
        F8 o = add ? ld8(dx + (long long)i * 8) : F8{};
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const float s = a.v[k] + bb.v[k] + c.v[k] + d.v[k];
            o.v[k] = add ? o.v[k] + s : s;
        }
        st8(dx + (long long)i * 8, o);
    }
}

// z[p] = [a[p], b[p]] (channels Ca + Cb); adjoint: da[p] (+)= z[p][0:Ca], db[p] (+)= z[p][Ca:]
__global__ void __launch_bounds__(256) k_concat(const bf16* __restrict__ a, int Ca, const bf16* __restrict__ b, int Cb,
                                               unsigned total, bf16* __restrict__ z)
{
    const unsigned c8 = (unsigned)(Ca + Cb) / 8, a8 = (unsigned)Ca / 8, b8 = (unsigned)Cb / 8;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const unsigned cc = i % c8;
        const long long p = i / c8;
        const bf16* src = cc < a8 ? a + (p * a8 + cc) * 8 : b + (p * b8 + (cc - a8)) * 8;
        *reinterpret_cast<uint4*>(z + (long long)i * 8) = *reinterpret_cast<const uint4*>(src);
    }
}
__global__ void __launch_bounds__(256) k_concat_adj(const bf16* __restrict__ dz, int Ca, int Cb, unsigned total,
                                                   bf16* __restrict__ da, int add_a, bf16* __restrict__ db, int add_b)
{
    const unsigned c8 = (unsigned)(Ca + Cb) / 8, a8 = (unsigned)Ca / 8, b8 = (unsigned)Cb / 8;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const unsigned cc = i % c8;
        const long long p = i / c8;
        const bool first = cc < a8;
        bf16* d = first ? da + (p * a8 + cc) * 8 : db + (p * b8 + (cc - a8)) * 8;
        const int add = first ? add_a : add_b;
        if (!add) {
            *reinterpret_cast<uint4*>(d) = *reinterpret_cast<const uint4*>(dz + (long long)i * 8);
        } else {
            const F8 v = ld8(dz + (long long)i * 8);
            F8 o = ld8(d);
#pragma unroll
            for (int k = 0; k < 8; k++) o.v[k] += v.v[k];
            st8(d, o);
        }
    }
}

// dst (+)= src * (mask > 0) (ReLU derivative), 8 values per thread
__global__ void __launch_bounds__(256) k_relu_adj(const bf16* __restrict__ src, const bf16* __restrict__ mask,
                                                 unsigned total, bf16* __restrict__ dst, int add)
{
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const F8 s = ld8(src + (long long)i * 8), m = ld8(mask + (long long)i * 8);
        F8 o = add ? ld8(dst + (long long)i * 8) : F8{};
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const float v = m.v[k] > 0.f ? s.v[k] : 0.f;
            o.v[k] = add ? o.v[k] + v : v;
        }
        st8(dst + (long long)i * 8, o);
    }
}

int g_sms()
{
    int dev = 0, n = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}
unsigned g_grid(long long total, int per = 256)
{
    return (unsigned)std::max<long long>(1, std::min<long long>((total + per - 1) / per, 16LL * g_sms()));
}

template <int BN>
void launch_gemm(GemmArgs& a, cudaStream_t st)
{
    static int opened[64] = {};
    int dev = 0;
    GCUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error(EIO_ERR_ARG, "device index above 63");
    if (!opened[dev]) {
        GCUDA(cudaFuncSetAttribute(k_gemm_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, GCfg<BN>::SMEM));
        opened[dev] = 1;
    }
    const long long mt = (a.M + G_BM - 1) / G_BM, nt = (a.N + BN - 1) / BN;
    if (mt * nt * a.splits > (1LL << 30)) throw Error(EIO_ERR_ARG, "GEMM tile count out of range");
    a.mt = (int)mt;
    a.nt = (int)nt;
    const long long tiles = mt * nt * a.splits;
    k_gemm_tc<BN><<<(unsigned)std::min<long long>(tiles, g_sms()), G_THREADS, GCfg<BN>::SMEM, st>>>(a);
    GCUDA(cudaGetLastError());
}

void launch_any(GemmArgs& a, cudaStream_t st)
{
    if (a.N <= 32) launch_gemm<32>(a, st);
    else if (a.N <= 64) launch_gemm<64>(a, st);
    else if (a.N <= 128) launch_gemm<128>(a, st);
    else launch_gemm<256>(a, st);
}

void check16(const void* p, const char* what)
{
    if (!p) throw Error(EIO_ERR_ARG, std::string("null ") + what);
    if (reinterpret_cast<uintptr_t>(p) % 16) throw Error(EIO_ERR_ARG, std::string(what) + " not 16-byte aligned");
}
void check16opt(const void* p, const char* what)
{
    if (p && reinterpret_cast<uintptr_t>(p) % 16) throw Error(EIO_ERR_ARG, std::string(what) + " not 16-byte aligned");
}

// K slices per split for at most `splits` splits, none of them empty; returns the split count
int fit_splits(long long kt, int splits, long long* kchunk)
{
    const long long per = (kt + splits - 1) / splits;
    *kchunk = per * G_BK;
    return (int)((kt + per - 1) / per);
}

// K splits of a weight gradient: enough tiles for two per SM, each split at
// least four slices (256 pixels)
int wgrad_splits(long long M, long long N, long long K)
{
    const long long bn = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
    const long long base = ((M + G_BM - 1) / G_BM) * ((N + bn - 1) / bn);
    const long long kt = (K + G_BK - 1) / G_BK;
    long long s = (2LL * g_sms() + base - 1) / base;
    s = std::max<long long>(1, std::min<long long>(s, kt / 4));
    long long kc;
    return fit_splits(kt, (int)std::min<long long>(s, 4096), &kc);
}

void conv_geometry(int n, int h, int w, int cin, int cout)
{
    if (n < 1 || h < 1 || w < 1 || cin < 8 || cout < 8 || cin % 8 || cout % 8)
        throw Error(EIO_ERR_ARG, "conv3x3: positive sizes, channel counts multiples of 8");
    if ((long long)n * h * w > (1LL << 31)) throw Error(EIO_ERR_ARG, "conv3x3: too many pixels");
}

unsigned chunks(long long values, const char* what)
{
    if (values % 8) throw Error(EIO_ERR_ARG, std::string(what) + ": value counts must be multiples of 8");
    if (values / 8 >= (1LL << 31)) throw Error(EIO_ERR_ARG, std::string(what) + ": tensor too large");
    return (unsigned)(values / 8);
}

}  // namespace

// C = A . B^T (see k_gemm_tc).  splits > 1: split-K over at most `splits`
// slices into scratch (splits x M x N floats), then summed in slice order
// into C32 / C16 (no mask or ReLU epilogue with splits > 1).
void gemm_bf16(long long M, long long N, long long K, const void* A, long long lda, const void* B, long long ldb,
               float* C32, void* C16, const void* mask, int relu, int splits, float* scratch, void* stream)
{
    if (M < 1 || N < 1 || K < 1 || N > (1LL << 24)) throw Error(EIO_ERR_ARG, "GEMM sizes out of range");
    if (K % 8 || lda % 8 || ldb % 8 || lda < K || ldb < K)
        throw Error(EIO_ERR_ARG, "K and the leading dimensions must be multiples of 8 (16-byte rows), lda, ldb >= K");
    check16(A, "A");
    check16(B, "B");
    if (!C32 && !C16) throw Error(EIO_ERR_ARG, "no output");
    check16opt(C32, "C32");
    check16opt(C16, "C16");
    check16opt(mask, "mask");
    check16opt(scratch, "scratch");
    if (splits < 1 || splits > 4096) throw Error(EIO_ERR_ARG, "splits must be 1 .. 4096");
    const long long kt = (K + G_BK - 1) / G_BK;
    splits = (int)std::min<long long>(splits, kt);
    if (splits > 1 && (mask || relu)) throw Error(EIO_ERR_ARG, "split-K GEMMs have no mask or ReLU epilogue");
    if (splits > 1 && !scratch) throw Error(EIO_ERR_ARG, "split-K needs scratch (splits x M x N floats)");
    GemmArgs a{};
    a.A = static_cast<const bf16*>(A);
    a.B = static_cast<const bf16*>(B);
    a.M = M; a.N = N; a.K = K; a.lda = lda; a.ldb = ldb;
    a.amode = OP_PLAIN;
    a.bmode = OP_PLAIN;
    a.splits = fit_splits(kt, splits, &a.kchunk);
    a.C32 = a.splits > 1 ? scratch : C32;
    a.C16 = a.splits > 1 ? nullptr : static_cast<bf16*>(C16);
    a.mask = static_cast<const bf16*>(mask);
    a.relu = relu;
    a.wait = g_gemm_wait;
    auto st = static_cast<cudaStream_t>(stream);
    launch_any(a, st);
    if (a.splits > 1) {
        k_sum_splits<<<g_grid(M * N), 256, 0, st>>>(scratch, a.splits, M, N, 0, 0, C32, static_cast<bf16*>(C16));
        GCUDA(cudaGetLastError());
    }
}

void gemm_set_wait_limit(long long polls) { g_gemm_wait = polls < 0 ? G_WAIT : polls; }

int gemm_status(int reset)
{
    int e = 0;
    GCUDA(cudaMemcpyFromSymbol(&e, g_gemm_err, sizeof(int)));
    if (reset) {
        const int z = 0;
        GCUDA(cudaMemcpyToSymbol(g_gemm_err, &z, sizeof(int)));
    }
    return e;
}

// y[p][co] = sum_{tap, ci} x[p + off(tap)][ci] w[co][tap][ci]: the implicit GEMM
void unet_conv3x3(int n, int h, int w, int cin, int cout, const void* x, const void* wt, float* y32, void* y16,
                  int relu, void* stream)
{
    conv_geometry(n, h, w, cin, cout);
    check16(x, "input");
    check16(wt, "weights");
    if (!y32 && !y16) throw Error(EIO_ERR_ARG, "conv3x3: no output");
    check16opt(y32, "FP32 output");
    check16opt(y16, "BF16 output");
    GemmArgs a{};
    a.A = static_cast<const bf16*>(x);
    a.B = static_cast<const bf16*>(wt);
    a.M = (long long)n * h * w; a.N = cout; a.K = 9LL * cin;
    a.lda = 0; a.ldb = 9LL * cin;
    a.amode = OP_CONV;
    a.bmode = OP_PLAIN;
    a.cw = w; a.ch = h; a.cc = cin;
    a.splits = 1;
    a.kchunk = ((a.K + G_BK - 1) / G_BK) * G_BK;
    a.C32 = y32;
    a.C16 = static_cast<bf16*>(y16);
    a.relu = relu;
    a.wait = g_gemm_wait;
    launch_any(a, static_cast<cudaStream_t>(stream));
}

long long unet_wgrad_scratch(int n, int h, int w, int cin, int cout)
{
    conv_geometry(n, h, w, cin, cout);
    const long long M = 9LL * cin, N = cout, K = (long long)n * h * w;
    return (long long)wgrad_splits(M, N, K) * M * N;
}

// dw[co][tap][ci] = sum_p dz[p][co] x[p + off(tap)][ci]: C[tap ci][co] with A
// gathered MN-major from x and B = dz read MN-major, the pixels split over the
// grid into scratch, the splits added in a fixed order and transposed into dw
void unet_conv3x3_wgrad(int n, int h, int w, int cin, int cout, const void* x, const void* dz, float* dw,
                        float* scratch, long long scratch_floats, void* stream)
{
    conv_geometry(n, h, w, cin, cout);
    check16(x, "input");
    check16(dz, "output gradient");
    check16(dw, "weight gradient");
    check16(scratch, "scratch");
    GemmArgs a{};
    a.A = static_cast<const bf16*>(x);
    a.B = static_cast<const bf16*>(dz);
    a.M = 9LL * cin; a.N = cout; a.K = (long long)n * h * w;
    a.lda = 0; a.ldb = cout;
    a.amode = OP_CONVT;
    a.bmode = OP_MN;
    a.cw = w; a.ch = h; a.cc = cin;
    const long long kt = (a.K + G_BK - 1) / G_BK;
    a.splits = fit_splits(kt, wgrad_splits(a.M, a.N, a.K), &a.kchunk);
    if ((long long)a.splits * a.M * a.N > scratch_floats)
        throw Error(EIO_ERR_ARG, "conv3x3 weight gradient: scratch too small (eio_unet_wgrad_scratch)");
    a.C32 = scratch;
    a.wait = g_gemm_wait;
    auto st = static_cast<cudaStream_t>(stream);
    launch_any(a, st);
    k_sum_splits<<<g_grid(a.M * a.N), 256, 0, st>>>(scratch, a.splits, a.M, a.N, 1, 0, dw, nullptr);
    GCUDA(cudaGetLastError());
}

void unet_flip(int cout, int cin, const void* w, void* wf, void* stream)
{
    if (cout < 1 || cin < 1 || !w || !wf) throw Error(EIO_ERR_ARG, "flip: sizes or pointers");
    k_flip_ct<<<g_grid(9LL * cout * cin), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const bf16*>(w), cout,
                                                                                       cin, static_cast<bf16*>(wf));
    GCUDA(cudaGetLastError());
}

void unet_resample(int op, int n, int h, int w, int c, const void* in, void* out, int add, void* stream)
{
    if (n < 1 || h < 1 || w < 1 || c < 8 || c % 8) throw Error(EIO_ERR_ARG, "resample: positive sizes, channels a multiple of 8");
    check16(in, "resample input");
    check16(out, "resample output");
    if ((op == 0 || op == 1) && (h % 2 || w % 2)) throw Error(EIO_ERR_ARG, "pooling needs even sizes");
    auto st = static_cast<cudaStream_t>(stream);
    auto i = static_cast<const bf16*>(in);
    auto o = static_cast<bf16*>(out);
    const long long full = (long long)n * h * w * c;
    switch (op) {
        case 0: {   // h, w: the input size
            const unsigned t = chunks(full / 4, "pooling");
            k_pool2<<<g_grid(t), 256, 0, st>>>(i, h, w, c, t, o);
            break;
        }
        case 1: {   // h, w: the output size
            const unsigned t = chunks(full, "pooling adjoint");
            k_pool2_adj<<<g_grid(t), 256, 0, st>>>(i, h, w, c, t, o, add);
            break;
        }
        case 2: {   // h, w: the input size
            const unsigned t = chunks(full * 4, "upsampling");
            k_up2<<<g_grid(t), 256, 0, st>>>(i, h, w, c, t, o);
            break;
        }
        case 3: {   // h, w: the output size
            const unsigned t = chunks(full, "upsampling adjoint");
            k_up2_adj<<<g_grid(t), 256, 0, st>>>(i, h, w, c, t, o, add);
            break;
        }
        default: throw Error(EIO_ERR_ARG, "resample op must be 0 .. 3");
    }
    GCUDA(cudaGetLastError());
}

void unet_concat(int adj, long long pixels, int ca, int cb, void* a, int add_a, void* b, int add_b, void* z,
                 void* stream)
{
    if (pixels < 1 || ca < 8 || cb < 8 || ca % 8 || cb % 8)
        throw Error(EIO_ERR_ARG, "concat: positive sizes, channels multiples of 8");
    check16(a, "concat first part");
    check16(b, "concat second part");
    check16(z, "concat whole");
    const unsigned t = chunks(pixels * (ca + cb), "concat");
    auto st = static_cast<cudaStream_t>(stream);
    if (!adj)
        k_concat<<<g_grid(t), 256, 0, st>>>(static_cast<const bf16*>(a), ca, static_cast<const bf16*>(b), cb, t,
                                            static_cast<bf16*>(z));
    else
        k_concat_adj<<<g_grid(t), 256, 0, st>>>(static_cast<const bf16*>(z), ca, cb, t, static_cast<bf16*>(a), add_a,
                                                static_cast<bf16*>(b), add_b);
    GCUDA(cudaGetLastError());
}

void unet_relu_adj(long long n, const void* src, const void* mask, void* dst, int add, void* stream)
{
    if (n < 1) throw Error(EIO_ERR_ARG, "relu adjoint: sizes");
    check16(src, "relu adjoint input");
    check16(mask, "relu adjoint mask");
    check16(dst, "relu adjoint output");
    const unsigned t = chunks(n, "relu adjoint");
    k_relu_adj<<<g_grid(t), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const bf16*>(src), static_cast<const bf16*>(mask), t, static_cast<bf16*>(dst), add);
    GCUDA(cudaGetLastError());
}

}  // namespace eio
