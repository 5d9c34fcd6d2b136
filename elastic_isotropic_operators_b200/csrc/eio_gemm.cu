// Tensor-core GEMM and the layer kernels of the U-Net preconditioner
// (precond.UNet; no reference counterpart).
//
// k_gemm_tc: C[M][N] = A[M][K] . B[N][K]^T, BF16 operands, FP32 accumulation
// in tensor memory, on tcgen05.  A tile of C is 128 x BN (BN = 32, 64, 128 or
// 256 TMEM columns, twice over); its K range (the whole K, or one slice of a
// split-K grid) streams through a 4- to 10-stage shared-memory ring in
// 64-wide slices, each filled by 16-byte cp.async copies into the 128-byte
// swizzled UMMA operand layouts (K-major, or MN-major for operands whose rows
// are contiguous in memory; 8 lanes copy one 128-byte row) and consumed by four tcgen05.mma.kind::f16
// (M = 128, N = BN, K = 16) that one thread issues and commits to the
// stage's mbarrier (256 threads copy and run the epilogue).  A stage is refilled once the MMAs that read it have
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
#include <cuda.h>   // CUtensorMap and the tensor-map encoder's types (the encoder is fetched at run time)
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
constexpr int G_THREADS = 256;                // 8 warps: copies and epilogue; thread 0 issues the MMAs
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
    static constexpr int STAGES = BN >= 256 ? 4 : (BN >= 128 ? 6 : (BN >= 64 ? 8 : 10));
    static constexpr int LAG = STAGES >= 8 ? 3 : (STAGES >= 6 ? 2 : 1);   // MMA batches in flight
    static constexpr int AHEAD = STAGES - LAG;                              // slices of copies in flight
    static constexpr int A_BYTES = G_BM * G_BK * 2;
    static constexpr int B_BYTES = BN * G_BK * 2;
    static constexpr int STAGE = A_BYTES + B_BYTES;                         // multiple of 1024
    static constexpr int BAR = 1024 + STAGES * STAGE;                       // after the 1024-byte alignment slack
    static constexpr int SMEM = BAR + 8 * STAGES + 16;
};

__device__ __forceinline__ unsigned g_smem(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor, 128-byte swizzle (sm_100 encoding: version
// 1 at bit 46, swizzle mode 2 at bits 61-63)
__device__ __forceinline__ unsigned long long g_desc(unsigned addr, unsigned lbo, unsigned sbo)
{
    return (unsigned long long)((addr >> 4) & 0x3FFF) | ((unsigned long long)((lbo >> 4) & 0x3FFF) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46) | (2ull << 61);
}

// Operand layouts of a stage holding `rows` rows x 64 K (all 128-byte
// swizzled, 1024-byte atoms of 8 x 128 bytes, chunk position XOR row % 8):
//   K-major:  row r is 128 bytes of K; chunk c (K 8c .. 8c+7) of row r at
//             (r / 8) * 1024 + (r % 8) * 128 + ((c ^ r % 8) * 16).
//             Descriptor of K16 step kk: start + 32 kk, SBO 1024 (8-row groups).
//   MN-major: K row k holds 64 consecutive rows (MN) in 128 bytes; chunk of MN
//             group g (rows 8g .. 8g+7) at K k sits in atom (k / 8, g / 8) at
//             ((k / 8) * (rows / 64) + g / 8) * 1024 + (k % 8) * 128 + (((g ^ k) % 8) * 16).
//             Descriptor of K16 step kk: start + 2 kk (rows / 64) 1024,
//             LBO 1024 (MN atoms), SBO (rows / 64) * 1024 (K groups of 8).
__device__ __forceinline__ unsigned g_kmaj(int r, int c)
{
    return (unsigned)((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4));
}
__device__ __forceinline__ unsigned g_mnmaj(int rows, int g, int k)
{
    return (unsigned)(((k >> 3) * (rows >> 6) + (g >> 3)) * 1024 + (k & 7) * 128 + (((g ^ k) & 7) << 4));
}
__device__ __forceinline__ unsigned long long g_opdesc(unsigned base, int rows, int kk, bool mn)
{
    return mn ? g_desc(base + (unsigned)(kk * 2 * (rows >> 6) * 1024), 1024, (unsigned)((rows >> 6) * 1024))
              : g_desc(base + (unsigned)(kk * 32), 16, 1024);
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

// 32 accumulator columns of this warp's 32 lanes
__device__ __forceinline__ void g_ld32(unsigned taddr, float* v)
{
    unsigned r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
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

// K-major copy loops: thread t copies chunk t % 8 of rows t / 8 + 32 j, so
// that 8 lanes read the 128 contiguous bytes of one row.  For OP_CONV, yx[j]
// holds (y << 16 | x) of row t / 8 + 32 j's pixel, -1 past M (set per tile;
// widths and heights below 2^15).  Pixel indices stay below 2^31 + 128
// (pixel counts are capped at 2^31).
constexpr int G_RPT = G_BM * 8 / G_THREADS;   // A rows per thread (4)
__device__ __forceinline__ void g_tile_pixels(const GemmArgs& g, long long m0, int* yx)
{
    const int r0 = threadIdx.x >> 3;
#pragma unroll
    for (int j = 0; j < G_RPT; j++) {
        const long long p = m0 + r0 + (G_THREADS / 8) * j;
        const unsigned pu = (unsigned)p, cw = (unsigned)g.cw;
        yx[j] = p < g.M ? (int)((((pu / cw) % (unsigned)g.ch) << 16) | (pu % cw)) : -1;
    }
}

// Slice [k0, k0 + 64) (K < ke) of A's rows [m0, m0 + 128) into stage dst
__device__ __forceinline__ void g_load_a(const GemmArgs& g, long long m0, long long k0, long long ke, unsigned dst,
                                         const int* yx)
{
    const int tid = threadIdx.x;
    if (g.amode == OP_PLAIN) {
        const int c = tid & 7;
        const long long k = k0 + 8 * c;
#pragma unroll
        for (int j = 0; j < G_RPT; j++) {
            const int r = (tid >> 3) + (G_THREADS / 8) * j;
            const long long row = m0 + r;
            const bool in = row < g.M && k < ke;
            g_cp16(dst + g_kmaj(r, c), in ? g.A + row * g.lda + k : g.A, in);
        }
    } else if (g.amode == OP_CONV) {
        const int c = tid & 7;
        const long long k = k0 + 8 * c;
        const int tap = (int)((unsigned)k / (unsigned)g.cc), c8 = (int)(k - (long long)tap * g.cc);
        const bool kin = k < ke;
#pragma unroll
        for (int j = 0; j < G_RPT; j++) {
            const int r = (tid >> 3) + (G_THREADS / 8) * j;
            long long src = -1;
            if (kin && yx[j] >= 0) src = g_tap_src(m0 + r, yx[j] >> 16, yx[j] & 0xFFFF, tap, g.ch, g.cw);
            g_cp16(dst + g_kmaj(r, c), src >= 0 ? g.A + src * g.cc + c8 : g.A, src >= 0);
        }
    } else {
        // OP_CONVT: rows (M) = tap * C + c, K = pixels.  Thread t copies MN
        // group t % 16 (8 channels of one tap) of pixels k0 + t / 16 + 16 j, so
        // that lanes read consecutive channels of one pixel.
        const int gr = tid & 15;
        const long long m = m0 + 8 * gr;
        const bool min_ = m < g.M;
        const int tap = min_ ? (int)((unsigned)m / (unsigned)g.cc) : 0;
        const int c8 = (int)(m - (long long)tap * g.cc);
        const int kp0 = tid >> 4;
        long long p = k0 + kp0;
        const unsigned pu = (unsigned)p, cw = (unsigned)g.cw, chh = (unsigned)g.ch;
        int x = (int)(pu % cw), y = (int)((pu / cw) % chh);
        constexpr int STEP = G_THREADS / 16;  // pixels between a thread's copies
#pragma unroll
        for (int j = 0; j < 64 / STEP; j++) {
            long long src = -1;
            if (min_ && p < ke) src = g_tap_src(p, y, x, tap, g.ch, g.cw);
            g_cp16(dst + g_mnmaj(G_BM, gr, kp0 + STEP * j), src >= 0 ? g.A + src * g.cc + c8 : g.A, src >= 0);
            p += STEP;
            x += STEP;
            while (x >= g.cw) {
                x -= g.cw;
                if (++y == g.ch) y = 0;
            }
        }
    }
}

// Slice [k0, k0 + 64) of B's rows [n0, n0 + BN) into stage dst
template <int BN>
__device__ __forceinline__ void g_load_b(const GemmArgs& g, long long n0, long long k0, long long ke, unsigned dst)
{
    const int tid = threadIdx.x;
    if (g.bmode == OP_PLAIN) {
        const int c = tid & 7;
        const long long k = k0 + 8 * c;
#pragma unroll
        for (int j = 0; j < BN * 8 / G_THREADS; j++) {
            const int r = (tid >> 3) + (G_THREADS / 8) * j;
            const long long row = n0 + r;
            const bool in = row < g.N && k < ke;
            g_cp16(dst + g_kmaj(r, c), in ? g.B + row * g.ldb + k : g.B, in);
        }
    } else {   // OP_MN: B[k][n] at k * ldb + n; lanes read consecutive 8-column groups of one k
        constexpr int G = BN / 8;
#pragma unroll
        for (int j = 0; j < BN * 8 / G_THREADS; j++) {
            const int i = threadIdx.x + G_THREADS * j;
            const int gr = i % G, kp = i / G;
            const long long k = k0 + kp, n = n0 + 8 * gr;
            const bool in = k < ke && n < g.N;
            g_cp16(dst + g_mnmaj(BN, gr, kp), in ? g.B + k * g.ldb + n : g.B, in);
        }
    }
}

// Accumulator buffer -> C: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its
// quarter) and the 32-column groups (w / 4) + 2 i
template <int BN>
__device__ __forceinline__ void g_epilogue(const GemmArgs& g, unsigned tbuf, long long m0, long long n0, int z)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, quarter = warp & 3;
    const long long row = m0 + quarter * 32 + lane;
    float* c32 = g.C32 ? g.C32 + (long long)z * g.M * g.N : nullptr;
#pragma unroll 1
    for (int c = (warp >> 2) * 32; c < BN; c += 64) {
        float v[32];
        g_ld32(tbuf + ((unsigned)(quarter * 32) << 16) + (unsigned)c, v);
        const long long col = n0 + c;
        if (row >= g.M || col >= g.N) continue;
        const int nv = (int)min((long long)32, g.N - col);
        const bool vec = (g.N & 7) == 0;      // 8-column groups stay 16-byte aligned
        if (g.mask) {
            const bf16* mk = g.mask + row * g.N + col;
            for (int i = 0; i < nv; i++)
                if (!(__bfloat162float(mk[i]) > 0.f)) v[i] = 0.f;
        } else if (g.relu) {
#pragma unroll
            for (int i = 0; i < 32; i++) v[i] = fmaxf(v[i], 0.f);
        }
        if (c32) {
            float* dst = c32 + row * g.N + col;
            if (vec) {
#pragma unroll
                for (int i = 0; i < 32; i += 8)
                    if (i < nv) {
                        *reinterpret_cast<float4*>(dst + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
                        *reinterpret_cast<float4*>(dst + i + 4) = make_float4(v[i + 4], v[i + 5], v[i + 6], v[i + 7]);
                    }
            } else {
                for (int i = 0; i < nv; i++) dst[i] = v[i];
            }
        }
        if (g.C16) {
            bf16* dst = g.C16 + row * g.N + col;
            if (vec) {
#pragma unroll
                for (int i = 0; i < 32; i += 8)
                    if (i < nv) {
                        uint4 u;
                        bf16* ub = reinterpret_cast<bf16*>(&u);
#pragma unroll
                        for (int e = 0; e < 8; e++) ub[e] = __float2bfloat16_rn(v[i + e]);
                        *reinterpret_cast<uint4*>(dst + i) = u;
                    }
            } else {
                for (int i = 0; i < nv; i++) dst[i] = __float2bfloat16_rn(v[i]);
            }
        }
    }
}

// Persistent tcgen05 GEMM (tile id: N tile fastest, then M tile, then K split).
// Slice q of this CTA lives in stage q % S; its MMAs commit to that stage's
// mbarrier.  After issuing slice q's MMAs the CTA refills the stage of slice
// q - LAG (waiting for those MMAs) with slice q + AHEAD, so LAG batches of
// MMAs and AHEAD slices of copies are in flight.  A tile's accumulator is
// read out once its last MMAs are known complete, while the next tile
// accumulates in the other TMEM buffer.
template <int BN>
__global__ void __launch_bounds__(G_THREADS, 1) k_gemm_tc(const __grid_constant__ GemmArgs g)
{
    using Cf = GCfg<BN>;
    constexpr int S = Cf::STAGES, LAG = Cf::LAG, AHEAD = Cf::AHEAD;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const unsigned raw = g_smem(smem_raw);
    unsigned char* smem = smem_raw + ((1024u - (raw & 1023u)) & 1023u);   // 1024-byte aligned stages
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_raw + Cf::BAR);
    unsigned* tslot = reinterpret_cast<unsigned*>(smem_raw + Cf::BAR + 8 * S);
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
    int l_tile = blockIdx.x, l_t = 0, l_n = 0, l_kt = 0;
    long long l_m0 = 0, l_n0 = 0, l_kb = 0, l_ke = 0;
    int yx[G_RPT];
    auto load_next = [&]() {
        if (l_tile < tiles) {
            const int s = l_n % S;
            if (l_t == 0) {                    // a new tile: its coordinates once
                l_m0 = t_m0(l_tile);
                l_n0 = t_n0(l_tile);
                l_kb = t_kb(l_tile);
                l_ke = t_ke(l_tile);
                l_kt = t_kt(l_tile);
                if (g.amode == OP_CONV) g_tile_pixels(g, l_m0, yx);
            }
            const long long k0 = l_kb + (long long)l_t * G_BK;
            g_load_a(g, l_m0, k0, l_ke, stageA(s), yx);
            g_load_b<BN>(g, l_n0, k0, l_ke, stageB(s));
            if (++l_t == l_kt) {
                l_t = 0;
                l_tile += gridDim.x;
            }
        }
        l_n++;
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    for (int i = 0; i < AHEAD; i++) load_next();

    const bool amn = g.amode == OP_CONVT, bmn = g.bmode == OP_MN;
    const unsigned idesc = g_idesc<BN>(amn, bmn);
    bool bad = false;
    int q = 0, it = 0;
    int ep_tile[2] = {-1, -1}, ep_last[2] = {0, 0};   // per TMEM buffer: tile awaiting its epilogue, its last slice
    auto epilogue = [&](int b) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        g_epilogue<BN>(g, tmem + (unsigned)(b * BN), t_m0(ep_tile[b]), t_n0(ep_tile[b]), t_z(ep_tile[b]));
        ep_tile[b] = -1;
    };
    // epilogues of tiles whose last slice is <= done (older tile first)
    auto drain_epilogues = [&](int done) {
        const int o = (ep_tile[0] >= 0 && ep_tile[1] >= 0) ? (ep_last[0] < ep_last[1] ? 0 : 1)
                                                           : (ep_tile[0] >= 0 ? 0 : 1);
        if (ep_tile[o] >= 0 && ep_last[o] <= done) epilogue(o);
        if (ep_tile[o ^ 1] >= 0 && ep_last[o ^ 1] <= done) epilogue(o ^ 1);
    };
    for (int tile = blockIdx.x; tile < tiles && !bad; tile += gridDim.x, it++) {
        const int b = it & 1;
        if (ep_tile[b] >= 0) {
            // the buffer still holds an older tile's sums: every MMA issued so far
            // is complete once the latest one is
            const bool ok = g_wait(g_smem(bar + (q - 1) % S), (unsigned)(((q - 1) / S) & 1), g.wait);
            if (__syncthreads_or(!ok)) {
                bad = true;
                break;
            }
            drain_epilogues(q - 1);
        }
        const int KT = t_kt(tile);
        const unsigned acc_buf = tmem + (unsigned)(b * BN);
        for (int t = 0; t < KT; t++, q++) {
            const int s = q % S;
            asm volatile("cp.async.wait_group %0;" ::"n"(AHEAD - 1) : "memory");
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
            // the stage of slice q - LAG is refilled next (with slice q + AHEAD):
            // its MMAs must have read it
            if (q >= LAG) {
                const int p = q - LAG;
                const bool ok = g_wait(g_smem(bar + p % S), (unsigned)((p / S) & 1), g.wait);
                if (__syncthreads_or(!ok)) {
                    bad = true;
                    q++;
                    break;
                }
                drain_epilogues(p);
            }
            load_next();
        }
        if (!bad) {
            ep_tile[b] = tile;
            ep_last[b] = q - 1;
        }
    }
    if (!bad && q > 0) {
        const bool ok = g_wait(g_smem(bar + (q - 1) % S), (unsigned)(((q - 1) / S) & 1), g.wait);
        if (__syncthreads_or(!ok)) bad = true;
        else drain_epilogues(q - 1);
    }
    if (bad) {
        // drain: every MMA issued is complete once the latest one is; then the
        // copies in flight; then the tensor memory is freed and the CTA leaves
        bool drained = true;
        if (q > 0) drained = g_wait(g_smem(bar + (q - 1) % S), (unsigned)(((q - 1) / S) & 1), G_DRAIN);
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


// ---------------------------------------------------------------------------
// k_conv_tma: the 3x3 convolutions with their operands brought in by TMA.
// When the pixels of a 128-row tile (or of a 64-pixel weight-gradient slice)
// form a rectangle of the NHWC image (widths that divide the box or are
// divided by it), the 3x3 gather of one tap and one block of 16 / 32 / 64
// channels is ONE 4-D tiled TMA box of the activation tensor at the tile's
// origin shifted by the tap; the tensor's out-of-bounds fill supplies the
// zero padding.  Roles: warp 0 (one lane) issues the copies, warp 1 (one
// lane) the MMAs, warps 2-5 read the accumulators out (one TMEM lane quarter
// each).  Stages are handed over through full / empty mbarriers, the two
// TMEM accumulators through their own pair; every wait is bounded and a role
// that gives up raises a shared abort flag that ends the others' waits.
//   conv (forward, data gradient): A = boxes {cb channels, bw x bh pixels}
//     (K-major, swizzle 2 cb bytes), up to 64 K per stage; B = the weights
//     [cout][9 cin] as one 2-D box {64 K, BN rows} (K-major, 128-byte swizzle).
//   weight gradient: A = boxes {cb channels, 64 pixels} of the input shifted by
//     the tap of each 128-row tile's channel blocks (MN-major), B = boxes
//     {cbB channels, 64 pixels} of dz (MN-major); K = pixels, split over the grid.
constexpr int T_THREADS = 192;

struct ConvTma {
    int wgrad;                 // 0: convolution, 1: weight gradient
    int C, cb;                 // channels of the gathered tensor, channel block of its boxes
    int W, H;                  // image size
    long long M, N, K;         // GEMM sizes; K = 9 C (convolution) or pixels (weight gradient)
    int mt, nt, splits;        // tiles: M, N, K splits
    long long kchunk;          // weight gradient: pixels per split (a multiple of 64)
    int cbB;                   // weight gradient: channel block of dz's boxes
    float* C32;                // optional [splits][M][N]
    bf16* C16;                 // optional [M][N]
    int relu;
    long long wait;
};

// CPS CTAs per SM (1, 2, 3 or 4): fewer stages each, and every CTA's TMEM
// allocation fits next to the others' (BN <= 128 for 2, <= 64 for 3 and 4);
// more CTAs keep more copies in flight per SM, which the small-channel
// layers' short box rows need
template <int BN, int CPS = 1>
struct TCfg {
    static constexpr int A_BYTES = 16384;
    static constexpr int B_BYTES = BN * 128;
    static constexpr int STAGE = A_BYTES + B_BYTES;        // multiple of 1024
    static constexpr int S0 = ((CPS == 1 ? 200 : CPS == 2 ? 96 : CPS == 3 ? 64 : 46) * 1024) / STAGE;
    static constexpr int STAGES = S0 > 8 ? 8 : S0;
    static constexpr int COLS = BN < 32 ? 32 : BN;          // TMEM columns of one accumulator buffer
    static constexpr int TALLOC = 2 * COLS <= 64 ? 64 : 2 * COLS <= 128 ? 128 : 2 * COLS <= 256 ? 256 : 512;
    static constexpr int BAR = 1024 + STAGES * STAGE;       // after the 1024-byte alignment slack
    static constexpr int SMEM = BAR + 8 * (2 * STAGES + 4) + 32;
};

__device__ __forceinline__ unsigned long long t_desc(unsigned addr, unsigned lbo, unsigned sbo, int swz)
{
    const unsigned long long mode = swz == 128 ? 2 : (swz == 64 ? 4 : 6);
    return (unsigned long long)((addr >> 4) & 0x3FFF) | ((unsigned long long)((lbo >> 4) & 0x3FFF) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46) | (mode << 61);
}
__device__ __forceinline__ void t_load4(unsigned dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                        unsigned bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(dst), "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void t_load2(unsigned dst, const CUtensorMap* map, int c0, int c1, unsigned bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 ::"r"(dst), "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void t_expect(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void t_arrive(unsigned bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// bounded wait; also gives up once another role raised the abort flag
__device__ __forceinline__ bool t_wait(unsigned bar, unsigned parity, long long limit, const volatile int* abort)
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
        if ((it & 255) == 255 && *abort) return false;
    }
    return false;
}
__device__ __forceinline__ void t_mma(unsigned acc, unsigned long long ad, unsigned long long bd, unsigned idesc,
                                      bool accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(acc), "l"(ad), "l"(bd), "r"(idesc), "r"(accumulate ? 1u : 0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void t_commit(unsigned bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

template <int BN, int CPS>
__global__ void __launch_bounds__(T_THREADS, CPS) k_conv_tma(const __grid_constant__ CUtensorMap ta,
                                                            const __grid_constant__ CUtensorMap tb,
                                                            const __grid_constant__ ConvTma g)
{
    using Cf = TCfg<BN, CPS>;
    static_assert(Cf::STAGES >= 2, "at least two stages");
    static_assert(Cf::TALLOC * CPS <= 512, "the CTAs of an SM share its 512 TMEM columns");
    constexpr int S = Cf::STAGES;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const unsigned raw = g_smem(smem_raw);
    const unsigned s0 = raw + ((1024u - (raw & 1023u)) & 1023u);   // 1024-byte aligned stages
    const unsigned bars = raw + Cf::BAR;                            // full[S], empty[S], tfull[2], tempty[2]
    auto full = [&](int s) { return bars + 8u * s; };
    auto empty = [&](int s) { return bars + 8u * (S + s); };
    auto tfull = [&](int b) { return bars + 8u * (2 * S + b); };
    auto tempty = [&](int b) { return bars + 8u * (2 * S + 2 + b); };
    unsigned* tslot = reinterpret_cast<unsigned*>(smem_raw + Cf::BAR + 8 * (2 * S + 4));
    volatile int* abort = reinterpret_cast<volatile int*>(tslot + 1);
    int* qprod = reinterpret_cast<int*>(tslot + 2);
    int* qmma = reinterpret_cast<int*>(tslot + 3);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles = g.mt * g.nt * g.splits;
    const int cpt = g.C / g.cb;                  // channel blocks per tap
    const int nbox = 9 * cpt, nbs = 64 / g.cb;   // convolution: boxes per tile, boxes per stage

    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full(s)) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty(s)) : "memory");
        }
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tfull(b)) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(tempty(b)) : "memory");
        }
        *abort = 0;
        *qprod = 0;
        *qmma = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(g_smem(tslot)),
                     "r"(Cf::TALLOC)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *tslot;
    auto stageA = [&](int s) { return s0 + (unsigned)(s * Cf::STAGE); };
    auto stageB = [&](int s) { return s0 + (unsigned)(s * Cf::STAGE + Cf::A_BYTES); };
    auto t_mi = [&](int id) { return (id / g.nt) % g.mt; };
    auto t_ni = [&](int id) { return id % g.nt; };
    auto t_z = [&](int id) { return id / (g.nt * g.mt); };
    auto slices = [&](int id) {
        if (!g.wgrad) return (nbox + nbs - 1) / nbs;
        const long long kb = (long long)t_z(id) * g.kchunk, ke = min(g.K, kb + g.kchunk);
        return (int)((ke - kb) / 64);
    };
    const long long HW = (long long)g.H * g.W;

    if (warp == 0 && lane == 0) {
        // ---- copies
        int q = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
            const int mi = t_mi(tile), ni = t_ni(tile), ns = slices(tile);
            const long long m0 = (long long)mi * G_BM;
            for (int j = 0; j < ns; j++, q++) {
                const int s = q % S;
                if (!t_wait(empty(s), (unsigned)(((q / S) & 1) ^ 1), g.wait, abort)) {
                    ok = false;
                    break;
                }
                if (!g.wgrad) {
                    // pixels m0 .. m0 + 127: a bw x bh rectangle at (n, y0, x0)
                    const int n = (int)(m0 / HW);
                    const long long rem = m0 - n * HW;
                    const int y0 = (int)(rem / g.W), x0 = (int)(rem - (long long)y0 * g.W);
                    const int b0 = j * nbs, nb = min(nbox - b0, nbs);
                    t_expect(full(s), (unsigned)(nb * G_BM * g.cb * 2 + BN * 128));
                    for (int i = 0; i < nb; i++) {
                        const int b = b0 + i, tap = b / cpt, c0 = (b - tap * cpt) * g.cb;
                        t_load4(stageA(s) + (unsigned)(i * G_BM * g.cb * 2), &ta, c0, x0 + tap % 3 - 1,
                                y0 + tap / 3 - 1, n, full(s));
                    }
                    t_load2(stageB(s), &tb, b0 * g.cb, ni * BN, full(s));
                } else {
                    const long long p0 = (long long)t_z(tile) * g.kchunk + 64LL * j;
                    const int n = (int)(p0 / HW);
                    const long long rem = p0 - n * HW;
                    const int y = (int)(rem / g.W), x = (int)(rem - (long long)y * g.W);
                    const int na = (int)min((long long)(G_BM / g.cb), (g.M - m0 + g.cb - 1) / g.cb);
                    const int nbB = BN / g.cbB;
                    t_expect(full(s), (unsigned)(na * 64 * g.cb * 2 + nbB * 64 * g.cbB * 2));
                    for (int i = 0; i < na; i++) {
                        const long long m = m0 + (long long)i * g.cb;
                        const int tap = (int)(m / g.C), c0 = (int)(m - (long long)tap * g.C);
                        t_load4(stageA(s) + (unsigned)(i * 64 * g.cb * 2), &ta, c0, x + tap % 3 - 1, y + tap / 3 - 1,
                                n, full(s));
                    }
                    for (int i = 0; i < nbB; i++)
                        t_load2(stageB(s) + (unsigned)(i * 64 * g.cbB * 2), &tb, i * g.cbB, (int)p0, full(s));
                }
            }
        }
        *qprod = q;
        if (!ok) *abort = 1;
    } else if (warp == 1 && lane == 0) {
        // ---- MMAs
        const unsigned idesc = (1u << 4) | (1u << 7) | (1u << 10) | (g.wgrad ? (1u << 15) | (1u << 16) : 0u) |
                               ((unsigned)(BN >> 3) << 17) | ((unsigned)(G_BM >> 4) << 24);
        const int swA = 2 * g.cb, swB = g.wgrad ? 2 * g.cbB : 128;
        int q = 0, it = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, it++) {
            const int b = it & 1, ns = slices(tile);
            if (!t_wait(tempty(b), (unsigned)(((it >> 1) & 1) ^ 1), g.wait, abort)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned acc = tmem + (unsigned)(b * Cf::COLS);
            for (int j = 0; j < ns; j++, q++) {
                const int s = q % S;
                if (!t_wait(full(s), (unsigned)((q / S) & 1), g.wait, abort)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                if (!g.wgrad) {
                    const int nb = min(nbox - j * nbs, nbs), steps = nb * g.cb / 16;
                    for (int kk = 0; kk < steps; kk++) {
                        const int i = kk * 16 / g.cb, off = (kk * 16 % g.cb) * 2;
                        const unsigned long long ad =
                            t_desc(stageA(s) + (unsigned)(i * G_BM * swA + off), 16, (unsigned)(8 * swA), swA);
                        const unsigned long long bd = t_desc(stageB(s) + (unsigned)(kk * 32), 16, 1024, 128);
                        t_mma(acc, ad, bd, idesc, (j | kk) != 0);
                    }
                } else {
                    for (int kk = 0; kk < 4; kk++) {
                        const unsigned long long ad = t_desc(stageA(s) + (unsigned)(kk * 16 * swA),
                                                             (unsigned)(64 * swA), (unsigned)(8 * swA), swA);
                        const unsigned long long bd = t_desc(stageB(s) + (unsigned)(kk * 16 * swB),
                                                             (unsigned)(64 * swB), (unsigned)(8 * swB), swB);
                        t_mma(acc, ad, bd, idesc, (j | kk) != 0);
                    }
                }
                t_commit(empty(s));   // the stage is free once these MMAs have read it
            }
            if (!ok) break;
            t_commit(tfull(b));       // the accumulator is complete once every MMA so far is
        }
        *qmma = q;
        if (!ok) *abort = 1;
    } else if (warp >= 2) {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31
        const int quarter = warp & 3;
        int it = 0;
        for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, it++) {
            const int b = it & 1;
            // every lane waits (and acquires); the warp goes on only if all lanes saw the
            // accumulator complete (tcgen05.ld is warp-collective)
            const bool seen = t_wait(tfull(b), (unsigned)((it >> 1) & 1), g.wait, abort);
            if (!__all_sync(0xffffffffu, seen)) {
                if (lane == 0) *abort = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const long long row = (long long)t_mi(tile) * G_BM + quarter * 32 + lane;
            const long long n0 = (long long)t_ni(tile) * BN;
            float* c32 = g.C32 ? g.C32 + (long long)t_z(tile) * g.M * g.N : nullptr;
#pragma unroll 1
            for (int c = 0; c < BN; c += 32) {
                float v[32];
                g_ld32(tmem + (unsigned)(b * Cf::COLS + c) + ((unsigned)(quarter * 32) << 16), v);
                const long long col = n0 + c;
                if (row >= g.M || col >= g.N) continue;
                const int nv = (int)min((long long)32, g.N - col);
                if (g.relu) {
#pragma unroll
                    for (int i = 0; i < 32; i++) v[i] = fmaxf(v[i], 0.f);
                }
                if (c32) {
                    float* dst = c32 + row * g.N + col;
#pragma unroll
                    for (int i = 0; i < 32; i += 8)
                        if (i < nv) {
                            *reinterpret_cast<float4*>(dst + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
                            *reinterpret_cast<float4*>(dst + i + 4) =
                                make_float4(v[i + 4], v[i + 5], v[i + 6], v[i + 7]);
                        }
                }
                if (g.C16) {
                    bf16* dst = g.C16 + row * g.N + col;
#pragma unroll
                    for (int i = 0; i < 32; i += 8)
                        if (i < nv) {
                            uint4 u;
                            bf16* ub = reinterpret_cast<bf16*>(&u);
#pragma unroll
                            for (int e = 0; e < 8; e++) ub[e] = __float2bfloat16_rn(v[i + e]);
                            *reinterpret_cast<uint4*>(dst + i) = u;
                        }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) t_arrive(tempty(b));
        }
    }
    __syncthreads();
    if (*abort && tid == 0) {
        // drain: copies issued but never consumed, then the MMAs (all complete
        // once the last committed batch is), before the tensor memory is freed
        bool drained = true;
        const volatile int never = 0;
        for (int q = *qmma; q < *qprod; q++)
            drained = t_wait(full(q % S), (unsigned)((q / S) & 1), G_DRAIN, &never) && drained;
        if (*qmma > 0) {
            const int q = *qmma - 1;
            drained = t_wait(empty(q % S), (unsigned)((q / S) & 1), G_DRAIN, &never) && drained;
        }
        atomicMax(&g_gemm_err, drained ? 1 : 2);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cf::TALLOC) : "memory");
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
    if (a.N <= 32 && a.bmode != OP_MN) launch_gemm<32>(a, st);   // MN-major operands come in 64-row atoms
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
    const long long bn = N <= 64 ? 64 : N <= 128 ? 128 : 256;     // the B operand is MN-major: BN >= 64
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
    if (h >= (1 << 15) || w >= (1 << 15)) throw Error(EIO_ERR_ARG, "conv3x3: height and width below 32768");
}

// ---- TMA path (k_conv_tma): tensor maps and eligibility
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
int g_use_tma = 3;   // TMA kernel, up to four CTAs per SM where the tile width allows

EncodeTiledFn tma_encoder()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        GCUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) throw Error(EIO_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// BF16 tensor map: dims / box innermost first, strides (bytes) of dims 1 ..;
// swizzle = the box's inner extent in bytes (32, 64 or 128); out-of-bounds reads give zeros
void tma_map(CUtensorMap* m, const void* base, int rank, const cuuint64_t* dims, const cuuint64_t* strides,
             const cuuint32_t* box, int swz)
{
    const cuuint32_t es[4] = {1, 1, 1, 1};
    const CUtensorMapSwizzle sw = swz == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                                  : swz == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                              : CU_TENSOR_MAP_SWIZZLE_32B;
    const CUresult r = tma_encoder()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, const_cast<void*>(base),
                                     dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(EIO_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

// the largest of 64 / 32 / 16 channels dividing c (0: none)
int chan_block(long long c) { return c % 64 == 0 ? 64 : c % 32 == 0 ? 32 : c % 16 == 0 ? 16 : 0; }

// a box of px pixels as a bw x bh rectangle that tiles the h x w image
bool rect_box(int h, int w, int px, int* bw, int* bh)
{
    if (w % px == 0) {
        *bw = px;
        *bh = 1;
        return true;
    }
    if (px % w == 0 && h % (px / w) == 0) {
        *bw = w;
        *bh = px / w;
        return true;
    }
    return false;
}

int tma_bn(long long n)
{
    const int opts[] = {16, 32, 64, 96, 128, 192, 256};
    for (int b : opts)
        if (n <= b) return b;
    return 192;
}

template <int BN, int CPS>
void launch_tma(const CUtensorMap& ta, const CUtensorMap& tb, const ConvTma& a, cudaStream_t st)
{
    static int opened[64] = {};
    int dev = 0;
    GCUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error(EIO_ERR_ARG, "device index above 63");
    if (!opened[dev]) {
        GCUDA(cudaFuncSetAttribute(k_conv_tma<BN, CPS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   TCfg<BN, CPS>::SMEM));
        opened[dev] = 1;
    }
    const long long tiles = (long long)a.mt * a.nt * a.splits;
    const long long ctas = std::min<long long>(tiles, (long long)CPS * g_sms());
    k_conv_tma<BN, CPS><<<(unsigned)ctas, T_THREADS, TCfg<BN, CPS>::SMEM, st>>>(ta, tb, a);
    GCUDA(cudaGetLastError());
}
// tile widths each CTA count takes: 4 per SM up to 32 columns, 3 up to 64, 2 up to 128
template <int CPS>
bool launch_tma_cps(int bn, const CUtensorMap& ta, const CUtensorMap& tb, const ConvTma& a, cudaStream_t st)
{
    constexpr int maxbn = CPS == 4 ? 32 : CPS == 3 ? 64 : CPS == 2 ? 128 : 256;
    if (bn > maxbn) return false;
    if (bn == 16) {
        launch_tma<16, CPS>(ta, tb, a, st);
        return true;
    }
    if (bn == 32) {
        launch_tma<32, CPS>(ta, tb, a, st);
        return true;
    }
    if constexpr (maxbn >= 64) {
        if (bn == 64) {
            launch_tma<64, CPS>(ta, tb, a, st);
            return true;
        }
    }
    if constexpr (maxbn >= 128) {
        if (bn == 96) {
            launch_tma<96, CPS>(ta, tb, a, st);
            return true;
        }
        if (bn == 128) {
            launch_tma<128, CPS>(ta, tb, a, st);
            return true;
        }
    }
    if constexpr (maxbn >= 256) {
        if (bn == 192) launch_tma<192, CPS>(ta, tb, a, st);
        else launch_tma<256, CPS>(ta, tb, a, st);
        return true;
    }
    return false;
}
// g_use_tma: 1 one CTA per SM; 2 up to two; 3 up to four (as many as the tile width allows)
void launch_tma_any(int bn, const CUtensorMap& ta, const CUtensorMap& tb, const ConvTma& a, cudaStream_t st)
{
    if (g_use_tma >= 3 && (launch_tma_cps<4>(bn, ta, tb, a, st) || launch_tma_cps<3>(bn, ta, tb, a, st))) return;
    if (g_use_tma >= 2 && launch_tma_cps<2>(bn, ta, tb, a, st)) return;
    launch_tma_cps<1>(bn, ta, tb, a, st);
}

// eligibility and splits of the two TMA forms
bool tma_conv_ok(int h, int w, int cin)
{
    int bw, bh;
    return g_use_tma && chan_block(cin) && rect_box(h, w, 128, &bw, &bh);
}
bool tma_wgrad_ok(int h, int w, int cin, int cout)
{
    int bw, bh;
    return g_use_tma && chan_block(cin) && cout % 16 == 0 && cout <= 256 && rect_box(h, w, 64, &bw, &bh);
}
int tma_wgrad_splits(long long M, long long P, long long* kchunk)
{
    const long long base = (M + G_BM - 1) / G_BM, kt = P / 64;
    long long s = (2LL * g_sms() + base - 1) / base;
    s = std::max<long long>(1, std::min<long long>(s, kt / 4));
    return fit_splits(kt, (int)std::min<long long>(s, 4096), kchunk);
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

void unet_set_tma(int on)
{
    if (on < 0 || on > 3)
        throw Error(EIO_ERR_ARG, "TMA mode: 0 copy loop, 1 TMA, 2 up to two CTAs per SM, 3 up to four");
    g_use_tma = on;
}
int unet_get_tma() { return g_use_tma; }

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
    if (tma_conv_ok(h, w, cin)) {
        int bw, bh;
        rect_box(h, w, 128, &bw, &bh);
        ConvTma t{};
        t.wgrad = 0;
        t.C = cin;
        t.cb = chan_block(cin);
        t.W = w;
        t.H = h;
        t.M = (long long)n * h * w;
        t.N = cout;
        t.K = 9LL * cin;
        const int bn = tma_bn(cout);
        t.mt = (int)(t.M / G_BM);
        t.nt = (int)((cout + bn - 1) / bn);
        t.splits = 1;
        t.C32 = y32;
        t.C16 = static_cast<bf16*>(y16);
        t.relu = relu;
        t.wait = g_gemm_wait;
        CUtensorMap ta, tb;
        const cuuint64_t da[4] = {(cuuint64_t)cin, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
        const cuuint64_t sa[3] = {(cuuint64_t)cin * 2, (cuuint64_t)w * cin * 2, (cuuint64_t)h * w * cin * 2};
        const cuuint32_t ba[4] = {(cuuint32_t)t.cb, (cuuint32_t)bw, (cuuint32_t)bh, 1};
        tma_map(&ta, x, 4, da, sa, ba, 2 * t.cb);
        const cuuint64_t db[2] = {(cuuint64_t)(9LL * cin), (cuuint64_t)cout};
        const cuuint64_t sb[1] = {(cuuint64_t)(9LL * cin * 2)};
        const cuuint32_t bb[2] = {64, (cuuint32_t)bn};
        tma_map(&tb, wt, 2, db, sb, bb, 128);
        launch_tma_any(bn, ta, tb, t, static_cast<cudaStream_t>(stream));
        return;
    }
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
    long long need = (long long)wgrad_splits(M, N, K) * M * N;
    if (tma_wgrad_ok(h, w, cin, cout)) {
        long long kc;
        need = std::max(need, (long long)tma_wgrad_splits(M, K, &kc) * M * N);
    }
    return need;
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
    auto st = static_cast<cudaStream_t>(stream);
    if (tma_wgrad_ok(h, w, cin, cout)) {
        int bw, bh;
        rect_box(h, w, 64, &bw, &bh);
        ConvTma t{};
        t.wgrad = 1;
        t.C = cin;
        t.cb = chan_block(cin);
        t.W = w;
        t.H = h;
        t.M = 9LL * cin;
        t.N = cout;
        t.K = (long long)n * h * w;
        const int bn = tma_bn(cout);
        t.cbB = chan_block(bn);
        t.mt = (int)((t.M + G_BM - 1) / G_BM);
        t.nt = 1;
        t.splits = tma_wgrad_splits(t.M, t.K, &t.kchunk);
        if ((long long)t.splits * t.M * t.N > scratch_floats)
            throw Error(EIO_ERR_ARG, "conv3x3 weight gradient: scratch too small (eio_unet_wgrad_scratch)");
        t.C32 = scratch;
        t.wait = g_gemm_wait;
        CUtensorMap ta, tb;
        const cuuint64_t da[4] = {(cuuint64_t)cin, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
        const cuuint64_t sa[3] = {(cuuint64_t)cin * 2, (cuuint64_t)w * cin * 2, (cuuint64_t)h * w * cin * 2};
        const cuuint32_t ba[4] = {(cuuint32_t)t.cb, (cuuint32_t)bw, (cuuint32_t)bh, 1};
        tma_map(&ta, x, 4, da, sa, ba, 2 * t.cb);
        const cuuint64_t db[2] = {(cuuint64_t)cout, (cuuint64_t)t.K};
        const cuuint64_t sb[1] = {(cuuint64_t)cout * 2};
        const cuuint32_t bb[2] = {(cuuint32_t)t.cbB, 64};
        tma_map(&tb, dz, 2, db, sb, bb, 2 * t.cbB);
        launch_tma_any(bn, ta, tb, t, st);
        k_sum_splits<<<g_grid(t.M * t.N), 256, 0, st>>>(scratch, t.splits, t.M, t.N, 1, 0, dw, nullptr);
        GCUDA(cudaGetLastError());
        return;
    }
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
