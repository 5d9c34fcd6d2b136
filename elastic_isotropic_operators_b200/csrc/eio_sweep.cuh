// TMA-pipelined x-sweep version of the fused fine step (same semantics as
// k_step in eio_kernels.cuh, see there for the reference citations).
//
// Each CTA owns a z-strip of TZ interior rows and a contiguous range of
// CW-column chunks along x.  The current level (forward) or the current level
// plus the medium (adjoint) is brought into a ring of CW-column shared-memory
// units by cp.async.bulk.tensor (TMA) with an mbarrier per slot, so halo
// columns are read from HBM once per strip instead of once per tile; the old
// level and the medium of each chunk (no halo) come through a second
// double-buffered TMA stage.  While chunk k is computed, unit k+2 and the
// stage of chunk k+1 are in flight.  Every mbarrier wait is bounded: on
// timeout the CTA sets an error flag, waits (bounded) for its outstanding
// copies and returns; the host turns the flag into an error.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "eio_kernels.cuh"

namespace eio {

constexpr long long WAIT_LIMIT = 1LL << 20;   // default try_wait polls before a pipeline wait gives up
constexpr long long DRAIN_LIMIT = 1LL << 24;  // polls of a drain wait after a timeout (never shortened)
constexpr int SWEEP_MAXK = 64;                // chunks per CTA range (upper bound)

struct SweepArgs {
    CUtensorMap tc[5];    // current level, box (TZ+8) x CW
    CUtensorMap tp[5];    // medium: forward box TZ x CW, adjoint box (TZ+8) x CW
    CUtensorMap to[5];    // old level, box TZ x CW
    float* o[5];          // old level; overwritten with the new level
    const float* dampz;
    const float* dampx;
    int nz, nx;
    int nstrips;          // z strips
    int nchunks;          // CW-column chunks along x over the whole interior
    int cpr;              // chunks per CTA range
    int nranges;          // ranges per strip
    float cz[4], cx[4];
    SparseOp inj, ext;    // tile id = strip * nchunks + chunk
    float* W0; float* W1; long long wstride; int wt; float ww0, ww1;
    const float* ssL[5]; const float* ssR[5];
    float* eL[5]; float* eR[5];
    float sw0, sw1;
    int tmode; float tw_o, tw_c, tw_n;   // EPI_TRI, see StepArgs
    const float* c[5];                  // current level (adjoint EPI_TRI reads it directly)
    int* err;
    long long wait_limit;   // try_wait polls of a pipeline wait (the drain always gets DRAIN_LIMIT)
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// bounded wait on phase `parity` (at most `limit` polls); returns false on timeout
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, long long limit) {
    const unsigned a = smem_u32(bar);
    for (long long it = 0; it < limit; it++) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}

template <int TZ, int CW, int DIR>
struct SweepLayout {
    static constexpr int NZG = TZ / 4;
    static constexpr int NT = NZG * CW;
    static constexpr int HZ = TZ + 2 * FAT;
    static constexpr int RU = 3;                       // ring units
    static constexpr int UNIT = CW * HZ;               // floats per field per unit
    static constexpr int STG = CW * TZ;                // floats per field per interior stage
    static constexpr int NRAWF = DIR == 0 ? 5 : 10;    // fields per TMA unit
    static constexpr int NSTGF = DIR == 0 ? 10 : 5;    // fields per interior stage (o [+ medium])
    static constexpr int NRAWBUF = DIR == 0 ? RU : 2;  // TMA unit buffers
    // offsets in floats
    static constexpr int RAW = 0;
    static constexpr int PROD = RAW + NRAWBUF * NRAWF * UNIT;            // adjoint product ring
    static constexpr int STAGE = PROD + (DIR == 0 ? 0 : RU * 5 * UNIT);
    static constexpr int SPARSE = STAGE + 2 * NSTGF * STG;
    static constexpr int META = SPARSE + 5 * STG;                         // per-CTA metadata
    static constexpr int META_F = 2 * (SWEEP_MAXK + 1) + SWEEP_MAXK * CW;  // 2 bucket offset lists + taper
    static constexpr int BAR = META + ((META_F + 3) / 4) * 4;            // mbarriers (8 B each)
    static constexpr int NBAR = NRAWBUF + 2;
    static constexpr size_t BYTES = (size_t)BAR * 4 + NBAR * 8;
    static constexpr unsigned UNIT_TX = NRAWF * UNIT * 4;
    static constexpr unsigned STAGE_TX = NSTGF * STG * 4;
};

template <int DIR, int EPI, int TZ, int CW>
__global__ void __launch_bounds__(SweepLayout<TZ, CW, DIR>::NT) k_sweep(const __grid_constant__ SweepArgs a)
{
    using Ly = SweepLayout<TZ, CW, DIR>;
    constexpr int NZG = Ly::NZG, NT = Ly::NT, HZ = Ly::HZ, RU = Ly::RU, UNIT = Ly::UNIT, STG = Ly::STG;
    extern __shared__ __align__(128) float sm[];
    float* raw = sm + Ly::RAW;
    float* prod = (DIR == 0) ? raw : sm + Ly::PROD;   // ring the stencils read
    float* stage = sm + Ly::STAGE;
    float* sparse = sm + Ly::SPARSE;
    int* m_inj = reinterpret_cast<int*>(sm + Ly::META);          // [K+1] bucket offsets of my chunks
    int* m_ext = m_inj + (SWEEP_MAXK + 1);
    float* m_dx = sm + Ly::META + 2 * (SWEEP_MAXK + 1);          // [K*CW] taper along x
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm + Ly::BAR);
    unsigned long long* rbar = bar;                       // [NRAWBUF]
    unsigned long long* sbar = bar + Ly::NRAWBUF;         // [2]
    __shared__ int abort_flag;

    const int tid = threadIdx.x;
    const int strip = blockIdx.x / a.nranges;
    const int range = blockIdx.x % a.nranges;
    const int ck0 = range * a.cpr;                        // first chunk of this CTA
    const int K = min(a.cpr, a.nchunks - ck0);            // chunks of this CTA
    if (K <= 0) return;                                   // CTA-uniform
    const int z0 = FAT + strip * TZ;
    const int xb = FAT + ck0 * CW;                        // first interior column of the range
    const int nz = a.nz;

    if (tid == 0) {
        for (int i = 0; i < Ly::NBAR; i++) mbar_init(bar + i, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // per-CTA metadata, read once instead of once per chunk on the critical path
    {
        const int tile0 = strip * a.nchunks + ck0;
        for (int i = tid; i <= K; i += NT) {
            m_inj[i] = a.inj.tile_start ? __ldg(a.inj.tile_start + tile0 + i) : 0;
            m_ext[i] = a.ext.tile_start ? __ldg(a.ext.tile_start + tile0 + i) : 0;
        }
        for (int i = tid; i < K * CW; i += NT) m_dx[i] = __ldg(a.dampx + xb + i);
    }
    __syncthreads();

    // phases issued by thread 0 (used to drain after an aborted wait)
    int pend[Ly::NBAR];
    unsigned ppar[Ly::NBAR];
#pragma unroll
    for (int i = 0; i < Ly::NBAR; i++) { pend[i] = 0; ppar[i] = 0; }
    // unit u covers columns xb - FAT + u*CW ... + CW-1; chunk k needs units k and k+1
    auto issue_unit = [&](int u) {
        if (u > K) return;
        float* dst = raw + (u % Ly::NRAWBUF) * (Ly::NRAWF * UNIT);
        unsigned long long* b = rbar + (u % Ly::NRAWBUF);
        pend[u % Ly::NRAWBUF] = 1;
        ppar[u % Ly::NRAWBUF] = (u / Ly::NRAWBUF) & 1;
        mbar_expect_tx(b, Ly::UNIT_TX);
        const int x = xb - FAT + u * CW;
#pragma unroll
        for (int f = 0; f < 5; f++) tma_load_2d(dst + f * UNIT, &a.tc[f], z0 - FAT, x, b);
        if (DIR == 1) {
#pragma unroll
            for (int f = 0; f < 5; f++) tma_load_2d(dst + (5 + f) * UNIT, &a.tp[f], z0 - FAT, x, b);
        }
    };
    auto issue_stage = [&](int k) {
        if (k >= K) return;
        float* dst = stage + (k & 1) * (Ly::NSTGF * STG);
        unsigned long long* b = sbar + (k & 1);
        pend[Ly::NRAWBUF + (k & 1)] = 1;
        ppar[Ly::NRAWBUF + (k & 1)] = (k >> 1) & 1;
        mbar_expect_tx(b, Ly::STAGE_TX);
        const int x = xb + k * CW;
#pragma unroll
        for (int f = 0; f < 5; f++) tma_load_2d(dst + f * STG, &a.to[f], z0, x, b);
        if (DIR == 0) {
#pragma unroll
            for (int f = 0; f < 5; f++) tma_load_2d(dst + (5 + f) * STG, &a.tp[f], z0, x, b);
        }
    };
    // adjoint: scaled combinations of a landed raw unit into the product ring
    auto transform = [&](int u) {
        const float* r = raw + (u % Ly::NRAWBUF) * (Ly::NRAWF * UNIT);
        float* p = prod + (u % RU) * (5 * UNIT);
        for (int q = tid; q < UNIT / 4; q += NT) {
            const float4 vx = ld4(r + 0 * UNIT + 4 * q), vz = ld4(r + 1 * UNIT + 4 * q);
            const float4 sxx = ld4(r + 2 * UNIT + 4 * q), szz = ld4(r + 3 * UNIT + 4 * q);
            const float4 sxz = ld4(r + 4 * UNIT + 4 * q);
            const float4 rx = ld4(r + 5 * UNIT + 4 * q), rz = ld4(r + 6 * UNIT + 4 * q);
            const float4 l2m = ld4(r + 7 * UNIT + 4 * q), lam = ld4(r + 8 * UNIT + 4 * q);
            const float4 mu = ld4(r + 9 * UNIT + 4 * q);
            float4 A, B, M, P, Q;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                at(A, j) = at(l2m, j) * at(sxx, j) + at(lam, j) * at(szz, j);
                at(B, j) = at(lam, j) * at(sxx, j) + at(l2m, j) * at(szz, j);
                at(M, j) = at(mu, j) * at(sxz, j);
                at(P, j) = at(rx, j) * at(vx, j);
                at(Q, j) = at(rz, j) * at(vz, j);
            }
            st4(p + 0 * UNIT + 4 * q, A);
            st4(p + 1 * UNIT + 4 * q, B);
            st4(p + 2 * UNIT + 4 * q, M);
            st4(p + 3 * UNIT + 4 * q, P);
            st4(p + 4 * UNIT + 4 * q, Q);
        }
    };
    bool ok = true;
    auto fail = [&]() {
        if (a.err) atomicExch(a.err, 1);
        abort_flag = 1;
    };

    // ---- prologue
    if (tid == 0) {
        issue_unit(0);
        issue_unit(1);
        if (DIR == 0) issue_unit(2);
        issue_stage(0);
        issue_stage(1);
    }
    if (DIR == 1) {
        for (int u = 0; u < 2; u++) {
            if (!mbar_wait(rbar + (u % 2), (u / 2) & 1, a.wait_limit)) fail();
            transform(u);
            __syncthreads();
            if (abort_flag) break;
            if (tid == 0) issue_unit(u + 2);
        }
    } else {
        if (!mbar_wait(rbar, 0, a.wait_limit)) fail();
    }

    const int zg = tid % NZG, jc = tid / NZG;
    const int gz = z0 + 4 * zg;
    const bool valid = gz < nz - FAT;
    const int zrow = FAT + 4 * zg;                        // row of my float4 inside a unit
    float dz4[4];
#pragma unroll
    for (int j = 0; j < 4; j++) dz4[j] = valid ? __ldg(a.dampz + gz + j) : 1.f;

    for (int k = 0; k < K; k++) {
        __syncthreads();
        if (abort_flag) break;
        const int gx = xb + k * CW + jc;
        const long long gi = (long long)gx * nz + gz;
        // Born dense inputs: issue the loads before waiting on the pipeline
        float4 pre[10];
        if (EPI == EPI_INJ_SS && valid) {
            const bool right = a.sw1 != 0.f;
#pragma unroll
            for (int f = 0; f < 5; f++) {
                pre[f] = ldg4(a.ssL[f] + gi);
                pre[5 + f] = right ? ldg4(a.ssR[f] + gi) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
        if (EPI == EPI_EXT_SS && valid) {
#pragma unroll
            for (int f = 0; f < 5; f++) { pre[f] = ld4(a.eL[f] + gi); pre[5 + f] = ld4(a.eR[f] + gi); }
        }
        if (EPI == EPI_SAVE_W && valid) {
            const float* w0p = a.W0 + (long long)a.wt * a.wstride + gi;
            const float* w1p = a.W1 + (long long)a.wt * a.wstride + gi;
            pre[0] = ld4(w0p); pre[1] = ld4(w0p + a.wstride); pre[2] = ld4(w1p); pre[3] = ld4(w1p + a.wstride);
        }
        if (DIR == 0) {
            if (!mbar_wait(rbar + ((k + 1) % RU), ((k + 1) / RU) & 1, a.wait_limit)) fail();
        }
        if (!mbar_wait(sbar + (k & 1), (k >> 1) & 1, a.wait_limit)) fail();
        // (the adjoint product units k, k+1 were completed by earlier iterations / the prologue)
        const float* u0 = prod + (k % RU) * (5 * UNIT);
        const float* u1 = prod + ((k + 1) % RU) * (5 * UNIT);
        const float* stg = stage + (k & 1) * (Ly::NSTGF * STG) + jc * TZ + 4 * zg;
        // column m of my 9-wide window (absolute column gx - 4 + m) lives in unit k + (jc+m)/CW
        auto colp = [&](int f, int m) -> const float* {
            const int r = jc + m;
            const float* ub = (r < CW) ? u0 : u1;
            return ub + f * UNIT + (r % CW) * HZ;
        };
        float4 t[5];
        {
            const float* cz = a.cz;
            const float* cx = a.cx;
            float4 q[9];
            float w[12];
            auto xw = [&](int f) {
#pragma unroll
                for (int m = 0; m < 9; m++) q[m] = ld4(colp(f, m) + zrow);
            };
            auto zw = [&](int f) {
                const float* p = colp(f, 4) + zrow - FAT;
                float4 x0 = ld4(p), x1 = ld4(p + 4), x2 = ld4(p + 8);
                w[0] = x0.x; w[1] = x0.y; w[2] = x0.z; w[3] = x0.w;
                w[4] = x1.x; w[5] = x1.y; w[6] = x1.z; w[7] = x1.w;
                w[8] = x2.x; w[9] = x2.y; w[10] = x2.z; w[11] = x2.w;
            };
            if (DIR == 0) {
                // fields: 0 vx, 1 vz, 2 sxx, 3 szz, 4 sxz
                xw(2); const float4 dxsxx = dmx(q, 4, cx);
                xw(4); const float4 dxsxz = dpx(q, 4, cx);
                xw(0); const float4 dxvx = dpx(q, 4, cx);
                xw(1); const float4 dxvz = dmx(q, 4, cx);
                zw(4); const float4 dzsxz = dpz(w, cz);
                zw(3); const float4 dzszz = dmz(w, cz);
                zw(0); const float4 dzvx = dmz(w, cz);
                zw(1); const float4 dzvz = dpz(w, cz);
                const float4 rx = ld4(stg + 5 * STG), rz = ld4(stg + 6 * STG), l2m = ld4(stg + 7 * STG),
                             lam = ld4(stg + 8 * STG), mu = ld4(stg + 9 * STG);
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    at(t[0], j) = at(rx, j) * (at(dxsxx, j) + at(dzsxz, j));
                    at(t[1], j) = at(rz, j) * (at(dzszz, j) + at(dxsxz, j));
                    at(t[2], j) = at(l2m, j) * at(dxvx, j) + at(lam, j) * at(dzvz, j);
                    at(t[3], j) = at(lam, j) * at(dxvx, j) + at(l2m, j) * at(dzvz, j);
                    at(t[4], j) = at(mu, j) * (at(dzvx, j) + at(dxvz, j));
                }
            } else {
                // products: 0 A, 1 B, 2 M, 3 P, 4 Q
                xw(0); const float4 dxA = dmx(q, 4, cx);
                xw(2); const float4 dxM = dpx(q, 4, cx);
                xw(3); const float4 dxP = dpx(q, 4, cx);
                xw(4); const float4 dxQ = dmx(q, 4, cx);
                zw(2); const float4 dzM = dpz(w, cz);
                zw(1); const float4 dzB = dmz(w, cz);
                zw(3); const float4 dzP = dmz(w, cz);
                zw(4); const float4 dzQ = dpz(w, cz);
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    at(t[0], j) = -(at(dxA, j) + at(dzM, j));
                    at(t[1], j) = -(at(dzB, j) + at(dxM, j));
                    at(t[2], j) = -at(dxP, j);
                    at(t[3], j) = -at(dzQ, j);
                    at(t[4], j) = -(at(dzP, j) + at(dxQ, j));
                }
            }
        }
        // deferred taper of the old level + leapfrog sum (+ scattered-field source)
        const float dxc = m_dx[k * CW + jc];
        float dd[4];
#pragma unroll
        for (int j = 0; j < 4; j++) dd[j] = fminf(dz4[j], dxc);
        float4 osave[5];
        float4 csave[2];
        if (EPI == EPI_TRI && DIR == 0) {
            csave[0] = ld4(colp(0, 4) + zrow);
            csave[1] = ld4(colp(1, 4) + zrow);
        }
#pragma unroll
        for (int f = 0; f < 5; f++) {
            const float4 o = ld4(stg + f * STG);
            if (EPI == EPI_TRI) osave[f] = o;
#pragma unroll
            for (int j = 0; j < 4; j++) at(t[f], j) = dd[j] * at(o, j) + at(t[f], j);
        }
        if (EPI == EPI_INJ_SS && valid) {
#pragma unroll
            for (int f = 0; f < 5; f++)
#pragma unroll
                for (int j = 0; j < 4; j++) at(t[f], j) += at(pre[f], j) * a.sw0 + at(pre[5 + f], j) * a.sw1;
        }
        // sparse injection before the final taper
        {
            const int e0 = m_inj[k], e1 = m_inj[k + 1];
            if (e1 > e0) {
                for (int i = tid; i < 5 * STG; i += NT) sparse[i] = 0.f;
                __syncthreads();
                for (int e = e0 + tid; e < e1; e += NT) {
                    const PointEntry pe = a.inj.ent[e];
                    const int f = pe.key >> 16, lx = (pe.key >> 8) & 0xff, lzz = pe.key & 0xff;
                    const float* sg = a.inj.sig[f];
                    const int ld = a.inj.ld[f];
                    const float v = sg[(long long)a.inj.t0 * ld + pe.col] * a.inj.w0 +
                                    sg[(long long)(a.inj.t0 + 1) * ld + pe.col] * a.inj.w1;
                    atomicAdd(sparse + (f * CW + lx) * TZ + lzz, v);
                }
                __syncthreads();
#pragma unroll
                for (int f = 0; f < 5; f++) {
                    const float4 v = ld4(sparse + (f * CW + jc) * TZ + 4 * zg);
#pragma unroll
                    for (int j = 0; j < 4; j++) at(t[f], j) += at(v, j);
                }
            }
        }
        // final taper, store, dense epilogues
#pragma unroll
        for (int f = 0; f < 5; f++)
#pragma unroll
            for (int j = 0; j < 4; j++) at(t[f], j) *= dd[j];
        if (valid) {
#pragma unroll
            for (int f = 0; f < 5; f++) st4(a.o[f] + gi, t[f]);
            if (EPI == EPI_SAVE_W) {
                float* w0p = a.W0 + (long long)a.wt * a.wstride + gi;
                float* w1p = a.W1 + (long long)a.wt * a.wstride + gi;
                float4 p0 = pre[0], p1 = pre[1], q0 = pre[2], q1 = pre[3];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    at(p0, j) += at(t[0], j) * a.ww0; at(p1, j) += at(t[0], j) * a.ww1;
                    at(q0, j) += at(t[1], j) * a.ww0; at(q1, j) += at(t[1], j) * a.ww1;
                }
                st4(w0p, p0); st4(w0p + a.wstride, p1); st4(w1p, q0); st4(w1p + a.wstride, q1);
            }
            if (EPI == EPI_EXT_SS) {
#pragma unroll
                for (int f = 0; f < 5; f++) {
                    float4 l = pre[f], r = pre[5 + f];
#pragma unroll
                    for (int j = 0; j < 4; j++) { at(l, j) += at(t[f], j) * a.sw0; at(r, j) += at(t[f], j) * a.sw1; }
                    st4(a.eL[f] + gi, l); st4(a.eR[f] + gi, r);
                }
            }
            if (EPI == EPI_TRI && a.tmode) {
                if (DIR == 0) {
                    st4(a.W0 + (long long)a.wt * a.wstride + gi,
                        tri_sample(a.tmode, osave[0], csave[0], t[0], a.tw_o, a.tw_c, a.tw_n));
                    st4(a.W1 + (long long)a.wt * a.wstride + gi,
                        tri_sample(a.tmode, osave[1], csave[1], t[1], a.tw_o, a.tw_c, a.tw_n));
                } else {
#pragma unroll
                    for (int f = 0; f < 5; f++)
                        st4(a.eL[f] + gi,
                            tri_sample(a.tmode, osave[f], ldg4(a.c[f] + gi), t[f], a.tw_o, a.tw_c, a.tw_n));
                }
            }
        }
        // sparse extraction after the final taper
        {
            const int e0 = m_ext[k], e1 = m_ext[k + 1];
            if (e1 > e0) {
                __syncthreads();
#pragma unroll
                for (int f = 0; f < 5; f++) st4(sparse + (f * CW + jc) * TZ + 4 * zg, t[f]);
                __syncthreads();
                for (int e = e0 + tid; e < e1; e += NT) {
                    const PointEntry pe = a.ext.ent[e];
                    const int f = pe.key >> 16, lx = (pe.key >> 8) & 0xff, lzz = pe.key & 0xff;
                    const float v = sparse[(f * CW + lx) * TZ + lzz];
                    float* sg = a.ext.sig[f];
                    const int ld = a.ext.ld[f];
                    sg[(long long)a.ext.t0 * ld + pe.col] += v * a.ext.w0;
                    sg[(long long)(a.ext.t0 + 1) * ld + pe.col] += v * a.ext.w1;
                }
            }
        }
        // refill: every thread is done with ring unit k and stage k&1
        __syncthreads();
        if (abort_flag) break;
        if (DIR == 0) {
            if (tid == 0) { issue_unit(k + RU); issue_stage(k + 2); }
        } else {
            if (tid == 0) issue_stage(k + 2);
            // product unit k+2 replaces unit k-1; its raw copy was issued two iterations ago
            if (k + 2 <= K) {
                if (!mbar_wait(rbar + (k % 2), ((k + 2) / 2) & 1, a.wait_limit)) fail();
                transform(k + 2);
                __syncthreads();
                if (tid == 0 && !abort_flag) issue_unit(k + 4);
            }
        }
    }
    (void)ok;
    if (abort_flag && tid == 0) {
        // drain: wait (bounded) for the last phase issued on every barrier
        for (int i = 0; i < Ly::NBAR; i++) {
            if (!pend[i]) continue;
            mbar_wait(bar + i, ppar[i], DRAIN_LIMIT);
        }
    }
}

}  // namespace eio
