// Kernels of the learned FWI preconditioner: a small fully convolutional
// network (3x3 convolutions, stride 1, zero padding 1, no biases, ReLU between
// layers) that maps an FWI gradient to an approximate Gauss-Newton model
// update.  The reference has no learned component; this network is trained on
// pairs (J^T J dm, dm) that the Born operators of this library produce.
//
// Layout: activations NHWC in BF16, C = 16 or 32 channels per pixel (32 or
// 64 bytes, so a pixel is whole 16-byte vectors); weights [9][Cout][Cin] BF16
// (tap = 3 dy + dx) with FP32 master copies for the optimiser.  Products run
// on the tensor cores as implicit GEMMs with FP32 accumulation
// (mma.sync m16n8k16 BF16):
//
// * k_conv3: y[p][co] = sum_tap sum_ci x[p + off(tap)][ci] w[tap][co][ci],
//   off(tap) = (dy - 1, dx - 1).  M = pixels (16 per fragment), N = Cout,
//   K = 9 Cin.  A CTA computes 8 rows x 32 columns of output pixels, one warp
//   per row; the input tile with its one-pixel halo and all weights sit in
//   shared memory, each pixel row padded by 8 BF16 so that the 32-bit
//   fragment loads of 8 consecutive pixels hit 32 distinct banks.  Epilogue:
//   optional ReLU, or a multiply by (mask > 0) (the ReLU derivative of the
//   layer below, for the backward pass), BF16 store and an optional FP32 copy.
// * the data gradient is the same kernel on the flipped, transposed weights
//   wt[tap][ci][co] = w[8 - tap][co][ci] (k_flip).
// * k_conv3_wgrad: dw[tap][co][ci] = sum_p dy[p][co] x[p + off(tap)][ci],
//   M = Cout, N = Cin, K = pixels; one warp per tap, both operands fetched
//   with ldmatrix.trans from the staged tiles.  A persistent grid keeps its
//   partial sums in registers over all its tiles and writes them once; the
//   partials are then summed in a fixed order (16 chunks of consecutive
//   blocks in parallel, then the chunks), so the weight gradient does not
//   change from run to run.
// * k_mse: loss 0.5 sum (y - t)^2 / count over the first nc channels, its
//   derivative in BF16; k_adam: Adam step on the FP32 master weights with the
//   BF16 copy written alongside.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "eio_internal.h"

namespace eio {

namespace {

using bf16 = __nv_bfloat16;

constexpr int CT_H = 8;     // output rows of a CTA (one warp each)
constexpr int CT_W = 32;    // output columns of a CTA (two 16-pixel fragments per warp)
constexpr int SR = CT_H + 2, SC = CT_W + 2;   // staged input tile with its halo
constexpr int FWD_THREADS = 32 * CT_H;
constexpr int WG_THREADS = 32 * 9;            // weight gradient: one warp per tap

__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldsm_x4_trans(uint32_t* r, const bf16* p)
{
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

__device__ __forceinline__ uint32_t lds32(const bf16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// rows x cols pixels of image n starting at (y0 - halo, x0 - halo) into shared
// memory (pixel stride C + 8); pixels outside the image are zero
template <int C>
__device__ __forceinline__ void stage_pixels(const bf16* __restrict__ x, int H, int W, int n, int y0, int x0,
                                             int halo, int rows, int cols, bf16* s, int nthr)
{
    constexpr int V = C / 8;
    constexpr int CP = C + 8;
    const int total = rows * cols * V;
    for (int i = threadIdx.x; i < total; i += nthr) {
        const int v = i % V, p = i / V;
        const int r = p / cols, c = p - r * cols;
        const int gy = y0 - halo + r, gx = x0 - halo + c;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (gy >= 0 && gy < H && gx >= 0 && gx < W)
            val = *reinterpret_cast<const uint4*>(x + (((size_t)n * H + gy) * W + gx) * C + v * 8);
        *reinterpret_cast<uint4*>(s + (size_t)p * CP + v * 8) = val;
    }
}

template <int CIN, int COUT>
constexpr int conv_smem() { return (SR * SC * (CIN + 8) + 9 * COUT * (CIN + 8)) * 2; }

template <int CIN, int COUT>
constexpr int wgrad_smem() { return (SR * SC * (CIN + 8) + CT_H * CT_W * (COUT + 8)) * 2; }

// EPI 0: optional ReLU; EPI 1: multiply by (mask > 0), mask NHWC with COUT channels
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(FWD_THREADS) k_conv3(const bf16* __restrict__ x, const bf16* __restrict__ w,
                                                      const bf16* __restrict__ mask, int relu, int H, int W,
                                                      bf16* __restrict__ y, float* __restrict__ y32)
{
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int CP = CIN + 8;
    constexpr int NT = COUT / 8;
    bf16* sx = reinterpret_cast<bf16*>(smem);
    bf16* sw = sx + SR * SC * CP;
    const int n = blockIdx.z, y0 = blockIdx.y * CT_H, x0 = blockIdx.x * CT_W;
    for (int i = threadIdx.x; i < 9 * COUT * (CIN / 8); i += FWD_THREADS) {
        const int v = i % (CIN / 8), row = i / (CIN / 8);
        *reinterpret_cast<uint4*>(sw + row * CP + v * 8) = *reinterpret_cast<const uint4*>(w + row * CIN + v * 8);
    }
    stage_pixels<CIN>(x, H, W, n, y0, x0, 1, SR, SC, sx, FWD_THREADS);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float acc[2][NT][4];
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
        for (int j = 0; j < NT; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[m][j][q] = 0.f;
#pragma unroll 1
    for (int tap = 0; tap < 9; tap++) {
        const int dy = tap / 3, dx = tap - 3 * dy;
        const bf16* srow = sx + ((warp + dy) * SC + dx) * CP;
#pragma unroll
        for (int kc = 0; kc < CIN / 16; kc++) {
            uint32_t a[2][4];
#pragma unroll
            for (int m = 0; m < 2; m++) {
                const bf16* p0 = srow + (m * 16 + g) * CP + kc * 16 + 2 * t;
                const bf16* p1 = p0 + 8 * CP;
                a[m][0] = lds32(p0);
                a[m][1] = lds32(p1);
                a[m][2] = lds32(p0 + 8);
                a[m][3] = lds32(p1 + 8);
            }
#pragma unroll
            for (int j = 0; j < NT; j++) {
                const bf16* pw = sw + (tap * COUT + j * 8 + g) * CP + kc * 16 + 2 * t;
                const uint32_t b0 = lds32(pw), b1 = lds32(pw + 8);
                mma_bf16(acc[0][j], a[0], b0, b1);
                mma_bf16(acc[1][j], a[1], b0, b1);
            }
        }
    }
    const int oy = y0 + warp;
    if (oy >= H) return;
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
        for (int half = 0; half < 2; half++) {
            const int ox = x0 + m * 16 + g + 8 * half;
            if (ox >= W) continue;
            const size_t pix = ((size_t)n * H + oy) * W + ox;
#pragma unroll
            for (int j = 0; j < NT; j++) {
                const int co = j * 8 + 2 * t;
                float v0 = acc[m][j][2 * half], v1 = acc[m][j][2 * half + 1];
                if constexpr (EPI == 0) {
                    if (relu) { v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); }
                } else {
                    const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162*>(mask + pix * COUT + co);
                    if (!(__bfloat162float(mk.x) > 0.f)) v0 = 0.f;
                    if (!(__bfloat162float(mk.y) > 0.f)) v1 = 0.f;
                }
                *reinterpret_cast<__nv_bfloat162*>(y + pix * COUT + co) = __floats2bfloat162_rn(v0, v1);
                if (y32) *reinterpret_cast<float2*>(y32 + pix * COUT + co) = make_float2(v0, v1);
            }
        }
}

// ---------------------------------------------------------------- tcgen05 path
// The same convolution on the 5th-generation tensor cores.  A CTA (4 warps)
// walks down a strip of TC_STRIP image rows, 128 output pixels wide; a
// persistent grid loops over the strips.  Input rows (with a one-pixel halo)
// sit in a ring of five shared-memory slots as [8-channel chunk][130
// pixels][8 BF16], which is the K-major, non-swizzled operand layout of
// tcgen05.mma: the A operand of tap (dy, dx) and 16 channels is a descriptor
// onto slot (y - 1 + dy) shifted by dx pixels (8 pixels x 16 B core matrices,
// the next 8 pixels 128 B on, the next 8 channels one chunk = 2080 B on), so
// no im2col copy is made and each input row is loaded once per strip.  The
// weights sit as [tap][chunk][Cout][8 BF16] (B operand, K-major).  One thread
// issues the 9 * Cin / 16 MMAs (M = 128, N = Cout, K = 16) of a row into one of
// two 32-column TMEM accumulators and commits them to that accumulator's
// mbarrier.  Software pipeline per row y: wait for input row y + 2 (cp.async;
// row y + 3 may still be in flight), barrier, issue the MMAs of row y + 1,
// wait (bounded) for those of row y, start the copies of row y + 4 into the
// slot those MMAs have released, epilogue of row y (each warp reads its 32
// lanes = pixels with tcgen05.ld): copies run two rows ahead, the tensor
// cores one row ahead of the epilogue.
// Operand and descriptor layout follow the PTX ISA's tcgen05 matrix
// descriptor (start, leading and stride byte offsets >> 4, version 1 at bit
// 46, no swizzle) and instruction descriptor (F32 accumulator, BF16 A and B,
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24).
constexpr int TC_PIX = 128;                 // output pixels of a row tile
constexpr int TC_HP = TC_PIX + 2;           // staged pixels of a row (halo)
constexpr int TC_THREADS = 128;
constexpr int TC_STRIP = 16;                // rows of a strip
constexpr int TC_SLOTS = 5;                 // input-row ring: rows y-1 .. y+3 of output row y
constexpr long long TC_WAIT_LIMIT = 1LL << 22;   // default try_wait polls of an accumulator wait
constexpr long long TC_DRAIN_LIMIT = 1LL << 24;  // polls of a drain wait after a timeout (never shortened)
constexpr int TC_TMEM_COLS = 64;            // two 32-column accumulators

// set when an mbarrier wait gives up: 1 = an accumulator wait timed out (the
// CTA drained its MMAs and copies and stopped; that call's output is
// incomplete), 2 = even the drain timed out (the context should be dropped)
__device__ int g_cnn_err;

// bounded wait on phase `parity` of the mbarrier at shared address `bar`
__device__ __forceinline__ bool tc_wait(unsigned bar, unsigned parity, long long limit)
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

template <int CIN, int COUT>
struct TcLayout {
    static constexpr int ROW_BYTES = (CIN / 8) * TC_HP * 16;
    static constexpr int A_BYTES = TC_SLOTS * ROW_BYTES;
    static constexpr int B_OFF = (A_BYTES + 127) / 128 * 128;
    static constexpr int B_BYTES = 9 * (CIN / 8) * COUT * 16;
    static constexpr int BAR_OFF = B_OFF + B_BYTES;   // 2 mbarriers, then the TMEM address
    static constexpr int SMEM = BAR_OFF + 32;
};

__device__ __forceinline__ unsigned cnn_smem_u32(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long umma_desc(unsigned addr, unsigned lbo, unsigned sbo)
{
    return (unsigned long long)((addr >> 4) & 0x3FFF) | ((unsigned long long)((lbo >> 4) & 0x3FFF) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

template <int COUT>
__device__ __forceinline__ constexpr unsigned umma_idesc()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(COUT >> 3) << 17) | ((unsigned)(TC_PIX >> 4) << 24);
}

template <int N>
__device__ __forceinline__ void tmem_ld(unsigned taddr, float* v);

template <>
__device__ __forceinline__ void tmem_ld<16>(unsigned taddr, float* v)
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

template <>
__device__ __forceinline__ void tmem_ld<32>(unsigned taddr, float* v)
{
    tmem_ld<16>(taddr, v);
    tmem_ld<16>(taddr + 16, v + 16);
}

// input row gy of image n, pixels x0-1 .. x0+128, into ring slot `slot` by
// 16-byte cp.async copies (zero-filled outside the image); the caller waits
template <int CIN>
__device__ __forceinline__ void tc_stage_row(const bf16* __restrict__ x, int H, int W, int n, int gy, int x0,
                                             unsigned char* slot)
{
    constexpr int KC = CIN / 8;
    const bool row_in = gy >= 0 && gy < H;
    for (int i = threadIdx.x; i < KC * TC_HP; i += TC_THREADS) {
        const int kc = i % KC, c = i / KC;
        const int gx = x0 - 1 + c;
        const bool in = row_in && gx >= 0 && gx < W;
        const bf16* src = in ? x + (((size_t)n * H + gy) * W + gx) * CIN + kc * 8 : x;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                         cnn_smem_u32(slot + ((size_t)kc * TC_HP + c) * 16)),
                     "l"(src), "r"(in ? 16 : 0)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ int tc_slot(int row) { return (row + TC_SLOTS) % TC_SLOTS; }   // row >= -1

__device__ __forceinline__ void tc_commit_empty() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// copy groups up to all but the newest `pending` have landed, then a barrier
template <int PENDING>
__device__ __forceinline__ void tc_rows_landed()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic writes -> tensor-core reads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
}

// the MMAs of output row y (ring slots of rows y-1 .. y+1) into accumulator buf, committed to bar
template <int CIN, int COUT>
__device__ __forceinline__ void tc_issue_row(unsigned a0, unsigned b0, int y, unsigned tmem_buf, unsigned bar)
{
    using Ly = TcLayout<CIN, COUT>;
    constexpr int KC = CIN / 8;
    constexpr unsigned idesc = umma_idesc<COUT>();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
    for (int tap = 0; tap < 9; tap++) {
        const int dy = tap / 3, dx = tap - 3 * dy;
        const unsigned slot = a0 + (unsigned)(tc_slot(y - 1 + dy) * Ly::ROW_BYTES);
#pragma unroll
        for (int kk = 0; kk < CIN / 16; kk++) {
            const unsigned long long ad = umma_desc(slot + (2 * kk * TC_HP + dx) * 16, TC_HP * 16, 128);
            const unsigned long long bd = umma_desc(b0 + ((tap * KC + 2 * kk) * COUT) * 16, COUT * 16, 128);
            const unsigned acc = (tap | kk) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                :
                : "r"(tmem_buf), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                : "memory");
        }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(TC_THREADS) k_conv3_tc(const bf16* __restrict__ x, const bf16* __restrict__ w,
                                                        const bf16* __restrict__ mask, int relu, int N, int H,
                                                        int W, bf16* __restrict__ y, float* __restrict__ y32,
                                                        long long wait_limit)
{
    using Ly = TcLayout<CIN, COUT>;
    constexpr int KC = CIN / 8;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sA = smem;
    unsigned char* sB = smem + Ly::B_OFF;
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem + Ly::BAR_OFF);
    unsigned* tslot = reinterpret_cast<unsigned*>(smem + Ly::BAR_OFF + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    for (int i = tid; i < 9 * COUT * KC; i += TC_THREADS) {   // weights -> [tap][chunk][co][8]
        const int kc = i % KC, row = i / KC;                   // row = tap * COUT + co
        const int tap = row / COUT, co = row - tap * COUT;
        *reinterpret_cast<uint4*>(sB + (((size_t)tap * KC + kc) * COUT + co) * 16) =
            *reinterpret_cast<const uint4*>(w + (size_t)row * CIN + kc * 8);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(cnn_smem_u32(bar)), "r"(1) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(cnn_smem_u32(bar + 1)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(cnn_smem_u32(tslot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *tslot;
    const unsigned a0 = cnn_smem_u32(sA), b0 = cnn_smem_u32(sB);
    const unsigned bar0 = cnn_smem_u32(bar);

    const int tilesX = (W + TC_PIX - 1) / TC_PIX, strips = (H + TC_STRIP - 1) / TC_STRIP;
    const long long units = (long long)N * strips * tilesX;
    unsigned phase[2] = {0u, 0u};
    unsigned k = 0;                          // rows done by this CTA: accumulator k & 1
    bool bad = false;
    for (long long u = blockIdx.x; u < units && !bad; u += gridDim.x) {
        const int xt = (int)(u % tilesX);
        const long long r = u / tilesX;
        const int sy = (int)(r % strips), n = (int)(r / strips);
        const int x0 = xt * TC_PIX, yb = sy * TC_STRIP, ye = min(H, yb + TC_STRIP);
        // prologue: rows yb-1 .. yb+1, the MMAs of row yb, then rows yb+2 and
        // yb+3 in flight, one copy group each (empty past the strip)
        for (int gy = yb - 1; gy <= yb + 1; gy++)
            tc_stage_row<CIN>(x, H, W, n, gy, x0, sA + tc_slot(gy) * Ly::ROW_BYTES);
        tc_rows_landed<0>();
        if (tid == 0) tc_issue_row<CIN, COUT>(a0, b0, yb, tmem + (k & 1) * 32, bar0 + (k & 1) * 8);
        for (int gy = yb + 2; gy <= yb + 3; gy++) {
            if (gy - 1 < ye) tc_stage_row<CIN>(x, H, W, n, gy, x0, sA + tc_slot(gy) * Ly::ROW_BYTES);
            else tc_commit_empty();
        }
        for (int yy = yb; yy < ye; yy++, k++) {
            // row yy+2 has landed (its group is the second newest; the epilogue
            // of row yy-1 is done): MMAs of row yy+1
            tc_rows_landed<1>();
            if (yy + 1 < ye && tid == 0)
                tc_issue_row<CIN, COUT>(a0, b0, yy + 1, tmem + ((k + 1) & 1) * 32, bar0 + ((k + 1) & 1) * 8);
            // bounded wait for the accumulator of row yy
            const unsigned b = k & 1;
            const bool ok = tc_wait(bar0 + b * 8, phase[b], wait_limit);
            if (__syncthreads_or(!ok)) {
                // Timed out.  The MMAs of row yy (buffer b) and, when issued,
                // of row yy+1 (buffer b^1) may still be running and write TMEM
                // and arrive on the barriers; the cp.async copies of the ring
                // may still be landing.  Drain both before the CTA frees TMEM
                // and leaves, with a long fixed bound.
                bool drained = tc_wait(bar0 + b * 8, phase[b], TC_DRAIN_LIMIT);
                if (yy + 1 < ye) drained = tc_wait(bar0 + (b ^ 1) * 8, phase[b ^ 1], TC_DRAIN_LIMIT) && drained;
                asm volatile("cp.async.wait_all;" ::: "memory");
                drained = !__syncthreads_or(!drained);
                if (tid == 0) atomicMax(&g_cnn_err, drained ? 1 : 2);
                bad = true;
                break;
            }
            phase[b] ^= 1u;
            // the MMAs of row yy have read slot (yy-1): row yy+4 goes there, under
            // the epilogue and the next row (one group per row, empty past the strip)
            if (yy + 3 < ye) tc_stage_row<CIN>(x, H, W, n, yy + 4, x0, sA + tc_slot(yy + 4) * Ly::ROW_BYTES);
            else tc_commit_empty();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float v[COUT];
            tmem_ld<COUT>(tmem + b * 32 + ((unsigned)(warp * 32) << 16), v);
            const int gx = x0 + warp * 32 + lane;
            if (gx < W) {
                const size_t pix = ((size_t)n * H + yy) * W + gx;
                if constexpr (EPI == 0) {
                    if (relu) {
#pragma unroll
                        for (int c = 0; c < COUT; c++) v[c] = fmaxf(v[c], 0.f);
                    }
                } else {
#pragma unroll
                    for (int c8 = 0; c8 < COUT / 8; c8++) {
                        const uint4 mk = *reinterpret_cast<const uint4*>(mask + pix * COUT + c8 * 8);
                        const __nv_bfloat162* m2 = reinterpret_cast<const __nv_bfloat162*>(&mk);
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            if (!(__bfloat162float(m2[q].x) > 0.f)) v[c8 * 8 + 2 * q] = 0.f;
                            if (!(__bfloat162float(m2[q].y) > 0.f)) v[c8 * 8 + 2 * q + 1] = 0.f;
                        }
                    }
                }
#pragma unroll
                for (int c8 = 0; c8 < COUT / 8; c8++) {
                    uint4 o;
                    __nv_bfloat162* o2 = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
                    for (int q = 0; q < 4; q++) o2[q] = __floats2bfloat162_rn(v[c8 * 8 + 2 * q], v[c8 * 8 + 2 * q + 1]);
                    *reinterpret_cast<uint4*>(y + pix * COUT + c8 * 8) = o;
                }
                if (y32) {
#pragma unroll
                    for (int c4 = 0; c4 < COUT / 4; c4++)
                        *reinterpret_cast<float4*>(y32 + pix * COUT + c4 * 4) =
                            make_float4(v[4 * c4], v[4 * c4 + 1], v[4 * c4 + 2], v[4 * c4 + 3]);
                }
            }
        }
        // the next strip's prologue overwrites the ring: its barrier orders the
        // last epilogue's TMEM reads before the next MMAs
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS)
                     : "memory");
}

// partial weight gradients of the tiles tile = blockIdx.x, + gridDim.x, ...
// into part[blockIdx.x][9][COUT][CIN]
template <int CIN, int COUT>
__global__ void __launch_bounds__(WG_THREADS) k_conv3_wgrad(const bf16* __restrict__ x, const bf16* __restrict__ dy,
                                                           int N, int H, int W, float* __restrict__ part)
{
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int CPX = CIN + 8, CPY = COUT + 8;
    constexpr int MT = COUT / 16, NT = CIN / 8;
    bf16* sx = reinterpret_cast<bf16*>(smem);
    bf16* sd = sx + SR * SC * CPX;
    const int tap = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int ty = tap / 3, tx = tap - 3 * ty;
    const int tilesX = (W + CT_W - 1) / CT_W, tilesY = (H + CT_H - 1) / CT_H;
    const int ntiles = tilesX * tilesY * N;
    float acc[MT][NT][4];
#pragma unroll
    for (int m = 0; m < MT; m++)
#pragma unroll
        for (int j = 0; j < NT; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[m][j][q] = 0.f;
    const int mat = lane >> 3, mrow = lane & 7;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int n = tile / (tilesX * tilesY);
        const int rem = tile - n * tilesX * tilesY;
        const int y0 = (rem / tilesX) * CT_H, x0 = (rem % tilesX) * CT_W;
        __syncthreads();   // the previous tile's fragments are read
        stage_pixels<CIN>(x, H, W, n, y0, x0, 1, SR, SC, sx, WG_THREADS);
        stage_pixels<COUT>(dy, H, W, n, y0, x0, 0, CT_H, CT_W, sd, WG_THREADS);
        __syncthreads();
#pragma unroll 1
        for (int chunk = 0; chunk < CT_H * CT_W / 16; chunk++) {
            const int r = chunk / (CT_W / 16), c0 = (chunk % (CT_W / 16)) * 16;
            uint32_t a[MT][4];
#pragma unroll
            for (int m = 0; m < MT; m++)
                ldsm_x4_trans(a[m], sd + (r * CT_W + c0 + (mat >> 1) * 8 + mrow) * CPY + m * 16 + (mat & 1) * 8);
            uint32_t b[NT][2];
#pragma unroll
            for (int j2 = 0; j2 < NT / 2; j2++) {
                uint32_t q[4];
                ldsm_x4_trans(q, sx + ((r + ty) * SC + c0 + tx + (mat & 1) * 8 + mrow) * CPX + (2 * j2 + (mat >> 1)) * 8);
                b[2 * j2][0] = q[0];
                b[2 * j2][1] = q[1];
                b[2 * j2 + 1][0] = q[2];
                b[2 * j2 + 1][1] = q[3];
            }
#pragma unroll
            for (int m = 0; m < MT; m++)
#pragma unroll
                for (int j = 0; j < NT; j++) mma_bf16(acc[m][j], a[m], b[j][0], b[j][1]);
        }
    }
    float* out = part + (size_t)blockIdx.x * 9 * COUT * CIN + (size_t)tap * COUT * CIN;
#pragma unroll
    for (int m = 0; m < MT; m++)
#pragma unroll
        for (int j = 0; j < NT; j++) {
            const int co = m * 16 + g, ci = j * 8 + 2 * t;
            *reinterpret_cast<float2*>(out + co * CIN + ci) = make_float2(acc[m][j][0], acc[m][j][1]);
            *reinterpret_cast<float2*>(out + (co + 8) * CIN + ci) = make_float2(acc[m][j][2], acc[m][j][3]);
        }
}

constexpr int SUM_CHUNKS = 16;   // the block partials are summed in 16 chunks, then the chunks in order

// mid[c][j] = sum over the blocks b of chunk c (in order) of part[b][j]
__global__ void k_sum_partials(const float* __restrict__ part, int nblk, int len, float* __restrict__ mid)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (j >= len) return;
    const int b0 = (int)((long long)nblk * c / SUM_CHUNKS), b1 = (int)((long long)nblk * (c + 1) / SUM_CHUNKS);
    float s = 0.f;
    for (int b = b0; b < b1; b++) s += part[(size_t)b * len + j];
    mid[(size_t)c * len + j] = s;
}

__global__ void k_sum_chunks(const float* __restrict__ mid, int len, float* __restrict__ out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= len) return;
    float s = 0.f;
    for (int c = 0; c < SUM_CHUNKS; c++) s += mid[(size_t)c * len + j];
    out[j] = s;
}

// wt[tap][ci][co] = w[8 - tap][co][ci]
__global__ void k_flip(const bf16* __restrict__ w, int cin, int cout, bf16* __restrict__ wt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 9 * cin * cout) return;
    const int tap = i / (cin * cout), rem = i - tap * cin * cout;
    const int ci = rem / cout, co = rem - ci * cout;
    wt[i] = w[((size_t)(8 - tap) * cout + co) * cin + ci];
}

constexpr int MSE_THREADS = 256;

// dz = (y - t) * scale on channels < nc (0 elsewhere), partial sums of (y - t)^2 per block
__global__ void __launch_bounds__(MSE_THREADS) k_mse(const float* __restrict__ y, const float* __restrict__ tgt,
                                                     long long npix, int C, int nc, float scale,
                                                     bf16* __restrict__ dz, double* __restrict__ part)
{
    double acc = 0.0;
    const long long n = npix * C;
    for (long long i = (long long)blockIdx.x * MSE_THREADS + threadIdx.x; i < n;
         i += (long long)gridDim.x * MSE_THREADS) {
        const long long p = i / C;
        const int c = (int)(i - p * C);
        float d = 0.f;
        if (c < nc) {
            d = y[i] - tgt[p * nc + c];
            acc += (double)d * d;
        }
        dz[i] = __float2bfloat16_rn(d * scale);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __shared__ double ws[MSE_THREADS / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < MSE_THREADS / 32; k++) s += ws[k];
        part[blockIdx.x] = s;
    }
}

// one warp: lane l sums part[l], part[l + 32], ... in order, then a fixed shuffle tree
__global__ void k_sum_double(const double* __restrict__ part, int m, double scale, double* __restrict__ out)
{
    double s = 0.0;
    for (int i = threadIdx.x; i < m; i += 32) s += part[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *out = s * scale;
}

__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, long long n, float lr, float b1, float b2, float eps, float c1,
                       float c2, bf16* __restrict__ pb)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    p[i] = pi;
    if (pb) pb[i] = __float2bfloat16_rn(pi);
}

#define CCUDA(x)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (x);                                                                          \
        if (e_ != cudaSuccess) throw Error(EIO_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void check_channels(int cin, int cout)
{
    if ((cin != 16 && cin != 32) || (cout != 16 && cout != 32))
        throw Error(EIO_ERR_ARG, "convolution channels must be 16 or 32 (got " + std::to_string(cin) + " -> " +
                                     std::to_string(cout) + ")");
}

void check_dims(int n, int h, int w)
{
    if (n < 1 || h < 1 || w < 1 || n > 65535 || (h + CT_H - 1) / CT_H > 65535)
        throw Error(EIO_ERR_ARG, "bad batch or image size");
}

void check_ptr(const void* p, const char* what)
{
    if (!p) throw Error(EIO_ERR_ARG, std::string("null ") + what);
    if (reinterpret_cast<uintptr_t>(p) % 16) throw Error(EIO_ERR_ARG, std::string(what) + " not 16-byte aligned");
}

// Launch shape of kernel `K` on the current device: the dynamic shared-memory
// attribute set once per device, and the SM count times the CTAs that fit on
// an SM (at most `cap`).  Cached per device.
struct KernelSlots {
    int resident[64] = {};   // 0: not opened on that device yet
};

template <class K>
int open_kernel(KernelSlots& ks, K kernel, int threads, int smem, int cap)
{
    int dev = 0;
    CCUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error(EIO_ERR_ARG, "device index above 63");
    if (!ks.resident[dev]) {
        CCUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int nsm = 0, per = 0;
        CCUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem));
        ks.resident[dev] = nsm * std::max(1, std::min(per, cap));
    }
    return ks.resident[dev];
}

template <int CIN, int COUT, int EPI>
void launch_conv(int n, int h, int w, const bf16* x, const bf16* wt, const bf16* mask, int relu, bf16* y,
                 float* y32, cudaStream_t st)
{
    constexpr int sm = conv_smem<CIN, COUT>();
    static KernelSlots ks;
    open_kernel(ks, k_conv3<CIN, COUT, EPI>, FWD_THREADS, sm, 1 << 20);
    const dim3 grid((w + CT_W - 1) / CT_W, (h + CT_H - 1) / CT_H, n);
    k_conv3<CIN, COUT, EPI><<<grid, FWD_THREADS, sm, st>>>(x, wt, mask, relu, h, w, y, y32);
    CCUDA(cudaGetLastError());
}

// try_wait polls of the tcgen05 kernel's accumulator waits (process-wide)
long long g_tc_wait_limit = TC_WAIT_LIMIT;

template <int CIN, int COUT, int EPI>
void launch_conv_tc(int n, int h, int w, const bf16* x, const bf16* wt, const bf16* mask, int relu, bf16* y,
                    float* y32, cudaStream_t st)
{
    constexpr int sm = TcLayout<CIN, COUT>::SMEM;
    static KernelSlots ks;
    // each resident CTA holds TC_TMEM_COLS TMEM columns of the SM's 512
    const int grid_cap = open_kernel(ks, k_conv3_tc<CIN, COUT, EPI>, TC_THREADS, sm, 512 / TC_TMEM_COLS);
    const long long tiles = (long long)n * ((h + TC_STRIP - 1) / TC_STRIP) * ((w + TC_PIX - 1) / TC_PIX);
    const int grid = (int)std::min<long long>(tiles, grid_cap);
    k_conv3_tc<CIN, COUT, EPI><<<grid, TC_THREADS, sm, st>>>(x, wt, mask, relu, n, h, w, y, y32, g_tc_wait_limit);
    CCUDA(cudaGetLastError());
}

template <int CIN, int COUT>
int wgrad_blocks(int n, int h, int w)
{
    static KernelSlots ks;
    const int resident = open_kernel(ks, k_conv3_wgrad<CIN, COUT>, WG_THREADS, wgrad_smem<CIN, COUT>(), 1 << 20);
    const long long tiles = (long long)((w + CT_W - 1) / CT_W) * ((h + CT_H - 1) / CT_H) * n;
    return (int)std::min<long long>(tiles, resident);
}

}  // namespace

namespace {
int g_conv_path = 0;   // 0: mma.sync kernel (measured faster on these channel counts), 1: tcgen05 kernel
}

void cnn_set_conv_path(int path)
{
    if (path != 0 && path != 1) throw Error(EIO_ERR_ARG, "convolution path must be 0 (mma.sync) or 1 (tcgen05)");
    g_conv_path = path;
}

int cnn_get_conv_path() { return g_conv_path; }

void cnn_set_wait_limit(long long polls) { g_tc_wait_limit = polls < 0 ? TC_WAIT_LIMIT : polls; }
long long cnn_get_wait_limit() { return g_tc_wait_limit; }

int cnn_status(int reset)
{
    int e = 0;
    CCUDA(cudaMemcpyFromSymbol(&e, g_cnn_err, sizeof(int)));
    if (reset) {
        const int z = 0;
        CCUDA(cudaMemcpyToSymbol(g_cnn_err, &z, sizeof(int)));
    }
    return e;
}

void cnn_conv3x3(int n, int h, int w, int cin, int cout, const void* x, const void* wt, const void* mask, int relu,
                 void* y, float* y32, void* stream)
{
    check_channels(cin, cout);
    check_dims(n, h, w);
    check_ptr(x, "input");
    check_ptr(wt, "weights");
    check_ptr(y, "output");
    if (mask) check_ptr(mask, "mask");
    if (y32) check_ptr(y32, "FP32 output");
    auto st = static_cast<cudaStream_t>(stream);
    auto X = static_cast<const bf16*>(x);
    auto Wt = static_cast<const bf16*>(wt);
    auto M = static_cast<const bf16*>(mask);
    auto Y = static_cast<bf16*>(y);
#define CONV_CASE(CI, CO)                                                                 \
    if (cin == CI && cout == CO) {                                                        \
        if (g_conv_path == 1) {                                                           \
            if (M) launch_conv_tc<CI, CO, 1>(n, h, w, X, Wt, M, 0, Y, y32, st);           \
            else launch_conv_tc<CI, CO, 0>(n, h, w, X, Wt, nullptr, relu, Y, y32, st);    \
        } else {                                                                          \
            if (M) launch_conv<CI, CO, 1>(n, h, w, X, Wt, M, 0, Y, y32, st);              \
            else launch_conv<CI, CO, 0>(n, h, w, X, Wt, nullptr, relu, Y, y32, st);       \
        }                                                                                 \
        return;                                                                           \
    }
    CONV_CASE(16, 16)
    CONV_CASE(16, 32)
    CONV_CASE(32, 16)
    CONV_CASE(32, 32)
#undef CONV_CASE
}

long long cnn_wgrad_scratch(int n, int h, int w, int cin, int cout)
{
    check_channels(cin, cout);
    check_dims(n, h, w);
    int nb = 0;
    if (cin == 16 && cout == 16) nb = wgrad_blocks<16, 16>(n, h, w);
    if (cin == 16 && cout == 32) nb = wgrad_blocks<16, 32>(n, h, w);
    if (cin == 32 && cout == 16) nb = wgrad_blocks<32, 16>(n, h, w);
    if (cin == 32 && cout == 32) nb = wgrad_blocks<32, 32>(n, h, w);
    return ((long long)nb + SUM_CHUNKS) * 9 * cin * cout;   // block partials, then the chunk sums
}

void cnn_conv3x3_wgrad(int n, int h, int w, int cin, int cout, const void* x, const void* dy, float* dw,
                       float* scratch, long long scratchFloats, void* stream)
{
    check_channels(cin, cout);
    check_dims(n, h, w);
    check_ptr(x, "input");
    check_ptr(dy, "output gradient");
    check_ptr(dw, "weight gradient");
    check_ptr(scratch, "scratch");
    const long long need = cnn_wgrad_scratch(n, h, w, cin, cout);
    if (scratchFloats < need)
        throw Error(EIO_ERR_ARG, "weight-gradient scratch holds " + std::to_string(scratchFloats) + " floats, needs " +
                                     std::to_string(need));
    const int nb = (int)(need / (9LL * cin * cout)) - SUM_CHUNKS;
    auto st = static_cast<cudaStream_t>(stream);
    auto X = static_cast<const bf16*>(x);
    auto D = static_cast<const bf16*>(dy);
#define WG_CASE(CI, CO)                                                                                     \
    if (cin == CI && cout == CO)                                                                            \
        k_conv3_wgrad<CI, CO><<<nb, WG_THREADS, wgrad_smem<CI, CO>(), st>>>(X, D, n, h, w, scratch);
    WG_CASE(16, 16)
    WG_CASE(16, 32)
    WG_CASE(32, 16)
    WG_CASE(32, 32)
#undef WG_CASE
    CCUDA(cudaGetLastError());
    const int len = 9 * cin * cout;
    float* mid = scratch + (size_t)nb * len;
    k_sum_partials<<<dim3((len + 255) / 256, SUM_CHUNKS), 256, 0, st>>>(scratch, nb, len, mid);
    CCUDA(cudaGetLastError());
    k_sum_chunks<<<(len + 255) / 256, 256, 0, st>>>(mid, len, dw);
    CCUDA(cudaGetLastError());
}

void cnn_flip(int cin, int cout, const void* w, void* wt, void* stream)
{
    check_channels(cin, cout);
    if (!w || !wt) throw Error(EIO_ERR_ARG, "null weights");
    const int len = 9 * cin * cout;
    k_flip<<<(len + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const bf16*>(w), cin,
                                                                             cout, static_cast<bf16*>(wt));
    CCUDA(cudaGetLastError());
}

void cnn_mse(long long npix, int c, int nc, const float* y32, const float* target, void* dz, double* part,
             double* loss, void* stream)
{
    constexpr int nPart = CNN_MSE_PARTIALS;   // fixed, so the summation order does not depend on the device
    if (npix < 1 || c < 1 || nc < 1 || nc > c) throw Error(EIO_ERR_ARG, "bad loss sizes");
    if (!y32 || !target || !dz || !part || !loss) throw Error(EIO_ERR_ARG, "null loss buffer");
    auto st = static_cast<cudaStream_t>(stream);
    const double cnt = (double)npix * nc;
    k_mse<<<nPart, MSE_THREADS, 0, st>>>(y32, target, npix, c, nc, (float)(1.0 / cnt), static_cast<bf16*>(dz), part);
    CCUDA(cudaGetLastError());
    k_sum_double<<<1, 32, 0, st>>>(part, nPart, 0.5 / cnt, loss);
    CCUDA(cudaGetLastError());
}

void cnn_adam(long long n, float* p, float* m, float* v, const float* g, float lr, float b1, float b2, float eps,
              int step, void* pb, void* stream)
{
    if (n < 1 || !p || !m || !v || !g || step < 1) throw Error(EIO_ERR_ARG, "bad Adam arguments");
    const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, step)));
    k_adam<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        p, m, v, g, n, lr, b1, b2, eps, c1, c2, static_cast<bf16*>(pb));
    CCUDA(cudaGetLastError());
}

}  // namespace eio
