// Two fused fine steps per launch (temporal blocking of the step kernel).
//
// A CTA owns the same 64x16 tile as k_step.  It stages the current level
// (forward) or its scaled combinations (adjoint) with an 8-cell halo, computes
// step A (level t+1) on the tile widened by 4 cells on every side, keeps that
// level in shared memory and computes step B (level t+2) on the tile from it.
// The old level, the current level and the medium are read once for two
// steps and both new levels are written once: 100 B per cell for two updates
// instead of 2 x 80 B.  The ring of step-A cells outside the tile is computed
// again by the neighbouring CTA (the same operations on the same inputs, so
// the same values); only the tile's own cells are stored.
//
// Because neighbours read the old and current levels around their tiles
// while this CTA writes, the two new levels go to two other buffers (four
// level buffers in all); the leapfrog aliasing n = o of the single-step
// kernel does not apply here.
//
// Step A applies, in the order of the single-step kernel: the old level with
// the deferred taper, the scattered-field source (Born), the sparse sources
// (through per-tile lists of every point of the widened tile), the final
// taper; cells outside the updated interior stay zero.  Step B is the
// single-step tail (step_tail) with its own time weights.
#pragma once
#include "eio_kernels.cuh"

namespace eio {

constexpr int PH = 2 * FAT;                  // halo of the staged current level
constexpr int CZ = TZ + 2 * PH;              // 80
constexpr int CX = TX + 2 * PH;              // 32
constexpr int CFIELD = CZ * CX;
constexpr int EZ4 = SZ / 4;                  // float4 rows of the widened tile (18)
constexpr int NHALO = EZ4 * SX - NTZ * NTX;  // widened-tile units outside the tile (176)
constexpr int PAIR_SMEM = (5 * CFIELD + 5 * SMEM_FIELD) * (int)sizeof(float);
static_assert(NHALO <= NT, "one halo unit per thread");

struct PairArgs {
    // s[0], step A: o = level t-1, c = level t, inj = the widened-tile lists.
    // s[1], step B: o = the buffer that receives level t+2, c = level t+1.
    StepArgs s[2];
    float* n1[5];    // the buffer that receives level t+1 (= s[1].c)
};

// current level (forward) or its scaled combinations (adjoint) of the tile
// with an 8-cell halo into smc [5][CX][CZ]; zero outside the grid
template <int DIR>
__device__ __forceinline__ void pair_stage(const StepArgs& a, float* smc, int z0, int x0, int tid)
{
    const int nz = a.nz, nx = a.nx;
    constexpr int nq = CZ / 4;
    for (int q = tid; q < nq * CX; q += NT) {
        const int lx = q / nq, lz4 = (q % nq) * 4;
        const int gz = z0 - PH + lz4, gx = x0 - PH + lx;
        float4 v[5];
        if (gz >= 0 && gz < nz && gx >= 0 && gx < nx) {
            const long long gi = (long long)gx * nz + gz;
            if (DIR == 0) {
#pragma unroll
                for (int f = 0; f < 5; f++) v[f] = ldg4(a.c[f] + gi);
            } else {
                adj_products(ldg4(a.c[0] + gi), ldg4(a.c[1] + gi), ldg4(a.c[2] + gi), ldg4(a.c[3] + gi),
                             ldg4(a.c[4] + gi), ldg4(a.par[0] + gi), ldg4(a.par[1] + gi), ldg4(a.par[2] + gi),
                             ldg4(a.par[3] + gi), ldg4(a.par[4] + gi), v);
            }
        } else {
#pragma unroll
            for (int f = 0; f < 5; f++) v[f] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int f = 0; f < 5; f++) st4(smc + f * CFIELD + lx * CZ + lz4, v[f]);
    }
}

template <int DIR, int EPI>
__global__ void __launch_bounds__(NT, 2) k_pair(PairArgs p)
{
    extern __shared__ __align__(16) float psm[];
    float* smc = psm;                    // [5][CX][CZ]  level t (or its combinations), 8-cell halo
    float* smn = psm + 5 * CFIELD;       // [5][SX][SZ]  level t+1 on the widened tile
    const StepArgs& A = p.s[0];
    const StepArgs& B = p.s[1];

    const int tid = threadIdx.x;
    const int tile = blockIdx.x;
    const int bz = tile % A.ntz, bx = tile / A.ntz;
    const int z0 = FAT + bz * TZ, x0 = FAT + bx * TX;
    const int nz = A.nz, nx = A.nx;
    const int tzi = tid % NTZ, txi = tid / NTZ;
    const int gz = z0 + 4 * tzi, gx = x0 + txi;
    const bool valid = gz < nz - FAT;
    const long long gi = (long long)gx * nz + gz;

    pdl_begin(A, gi, valid);
    pair_stage<DIR>(A, smc, z0, x0, tid);
    __syncthreads();

    // ---------------------------------------------------------------- step A
    const bool injA = A.inj.tile_start && A.inj.tile_start[tile + 1] > A.inj.tile_start[tile];   // CTA-uniform
    float tri_max[2] = {0.f, 0.f};

    // my units of the widened tile (float4 row hz, column hx): the tile unit
    // of k_step's thread layout, and one unit of the surrounding ring
    int hz = 0, hx = 0;
    if (tid < 2 * TX) {
        hx = FAT + tid % TX;
        hz = tid < TX ? 0 : EZ4 - 1;
    } else if (tid < NHALO) {
        const int u = tid - 2 * TX, col = u / EZ4;
        hx = col < FAT ? col : TX + col;
        hz = u % EZ4;
    }

    // final taper, store, coarse sample of one step-A unit
    auto finishA = [&](float4 (&t)[5], const float4 (&osave)[5], const float (&dd)[4], long long ui, float* sn,
                       int lxc, int lzc, bool tileu) {
#pragma unroll
        for (int f = 0; f < 5; f++) {
#pragma unroll
            for (int j = 0; j < 4; j++) at(t[f], j) *= dd[j];
            st4(sn + f * SMEM_FIELD, t[f]);
        }
        if (tileu) {
#pragma unroll
            for (int f = 0; f < 5; f++) st4(p.n1[f] + ui, t[f]);
            if (EPI == EPI_TRI && A.tmode) {
                if (DIR == 0) {
                    const float4 c0 = ld4(smc + lxc * CZ + lzc), c1 = ld4(smc + CFIELD + lxc * CZ + lzc);
                    const float4 s0 = tri_sample(A.tmode, osave[0], c0, t[0], A.tw_o, A.tw_c, A.tw_n);
                    const float4 s1 = tri_sample(A.tmode, osave[1], c1, t[1], A.tw_o, A.tw_c, A.tw_n);
                    st4(A.W0 + (long long)A.wt * A.wstride + ui, s0);
                    st4(A.W1 + (long long)A.wt * A.wstride + ui, s1);
                    tri_max[0] = fmaxf(fmaxf(fabsf(s0.x), fabsf(s0.y)), fmaxf(fabsf(s0.z), fabsf(s0.w)));
                    tri_max[1] = fmaxf(fmaxf(fabsf(s1.x), fabsf(s1.y)), fmaxf(fabsf(s1.z), fabsf(s1.w)));
                } else {
#pragma unroll
                    for (int f = 0; f < 5; f++)
                        st4(A.eL[f] + ui, tri_sample(A.tmode, osave[f], ldg4(A.c[f] + ui), t[f], A.tw_o, A.tw_c, A.tw_n));
                }
            }
        }
    };

    // one unit of step A; with sparse sources in the widened tile the value
    // before the final taper is parked in smn and finished after the injection
    auto unitA = [&](int uz4, int ux4, bool tileu) {
        const int uz = z0 - FAT + 4 * uz4, ux = x0 - FAT + ux4;
        float* sn = smn + ux4 * SZ + 4 * uz4;
        const bool in = uz >= FAT && uz < nz - FAT && ux >= FAT && ux < nx - FAT;
        if (!in) {
#pragma unroll
            for (int f = 0; f < 5; f++) st4(sn + f * SMEM_FIELD, make_float4(0.f, 0.f, 0.f, 0.f));
            return;
        }
        const long long ui = (long long)ux * nz + uz;
        const int lxc = ux4 + FAT, lzc = 4 * uz4 + FAT;    // position in smc
        float4 t[5];
        auto par = [&](int k) { return ldg4(A.par[k] + ui); };
        stencil_fields<DIR, 0, 5, decltype(par), CZ, CFIELD>(smc, lxc, lzc, A.cz, A.cx, true, par, t);
        float dd[4];
        {
            const float dxc = __ldg(A.dampx + ux);
#pragma unroll
            for (int j = 0; j < 4; j++) dd[j] = fminf(__ldg(A.dampz + uz + j), dxc);
        }
        float4 osave[5];
#pragma unroll
        for (int f = 0; f < 5; f++) {
            const float4 o = ld4(A.o[f] + ui);
            osave[f] = o;
#pragma unroll
            for (int j = 0; j < 4; j++) at(t[f], j) = dd[j] * at(o, j) + at(t[f], j);
        }
        if (EPI == EPI_INJ_SS) {
            const bool right = A.sw1 != 0.f;
#pragma unroll
            for (int f = 0; f < 5; f++) {
                const float4 l = ldg4(A.ssL[f] + ui);
                const float4 r = right ? ldg4(A.ssR[f] + ui) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int j = 0; j < 4; j++) at(t[f], j) += at(l, j) * A.sw0 + at(r, j) * A.sw1;
            }
        }
        if (injA) {
#pragma unroll
            for (int f = 0; f < 5; f++) st4(sn + f * SMEM_FIELD, t[f]);
        } else {
            finishA(t, osave, dd, ui, sn, lxc, lzc, tileu);
        }
    };

    unitA(tzi + 1, txi + FAT, true);
    if (tid < NHALO) unitA(hz, hx, false);

    if (injA) {
        // sparse sources of the widened tile (keys relative to its corner)
        __syncthreads();
        const int e0 = A.inj.tile_start[tile], e1 = A.inj.tile_start[tile + 1];
        for (int e = e0 + tid; e < e1; e += NT) {
            const PointEntry pe = A.inj.ent[e];
            const int f = pe.key >> 16, lx = (pe.key >> 8) & 0xff, lzz = pe.key & 0xff;
            const float* sg = A.inj.sig[f];
            const int ld = A.inj.ld[f];
            const float v = sg[(long long)A.inj.t0 * ld + pe.col] * A.inj.w0 +
                            sg[(long long)(A.inj.t0 + 1) * ld + pe.col] * A.inj.w1;
            atomicAdd(smn + f * SMEM_FIELD + lx * SZ + lzz, v);
        }
        __syncthreads();
        auto finish_parked = [&](int uz4, int ux4, bool tileu) {
            const int uz = z0 - FAT + 4 * uz4, ux = x0 - FAT + ux4;
            if (!(uz >= FAT && uz < nz - FAT && ux >= FAT && ux < nx - FAT)) return;
            const long long ui = (long long)ux * nz + uz;
            float* sn = smn + ux4 * SZ + 4 * uz4;
            float4 t[5], osave[5];
            float dd[4];
            const float dxc = __ldg(A.dampx + ux);
#pragma unroll
            for (int j = 0; j < 4; j++) dd[j] = fminf(__ldg(A.dampz + uz + j), dxc);
#pragma unroll
            for (int f = 0; f < 5; f++) {
                t[f] = ld4(sn + f * SMEM_FIELD);
                osave[f] = (EPI == EPI_TRI && tileu) ? ld4(A.o[f] + ui) : t[f];
            }
            finishA(t, osave, dd, ui, sn, ux4 + FAT, 4 * uz4 + FAT, tileu);
        };
        finish_parked(tzi + 1, txi + FAT, true);
        if (tid < NHALO) finish_parked(hz, hx, false);
    }

    if (EPI == EPI_TRI && DIR == 0 && A.tmode && A.pmax) {   // uniform over the CTA
#pragma unroll
        for (int f = 0; f < 2; f++) {
            float m = tri_max[f];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if ((tid & 31) == 0) A.pmax[((long long)tile * 16 + (tid >> 5)) * 2 + f] = m;
        }
    }
    __syncthreads();

    // sparse extraction of step A (the tile's own points) from level t+1
    bool extA = false;
    if (A.ext.tile_start) {
        const int e0 = A.ext.tile_start[tile], e1 = A.ext.tile_start[tile + 1];
        extA = e1 > e0;
        for (int e = e0 + tid; e < e1; e += NT) {
            const PointEntry pe = A.ext.ent[e];
            const int f = pe.key >> 16, lx = (pe.key >> 8) & 0xff, lzz = pe.key & 0xff;
            const float v = smn[f * SMEM_FIELD + (lx + FAT) * SZ + lzz + FAT];
            float* sg = A.ext.sig[f];
            const int ld = A.ext.ld[f];
            sg[(long long)A.ext.t0 * ld + pe.col] += v * A.ext.w0;
            sg[(long long)(A.ext.t0 + 1) * ld + pe.col] += v * A.ext.w1;
        }
    }

    if (DIR == 1) {
        // the adjoint stencils act on the scaled combinations of level t+1
        if (extA) __syncthreads();
        auto combine = [&](int uz4, int ux4) {
            const int uz = z0 - FAT + 4 * uz4, ux = x0 - FAT + ux4;
            if (!(uz >= FAT && uz < nz - FAT && ux >= FAT && ux < nx - FAT)) return;   // stays zero
            const long long ui = (long long)ux * nz + uz;
            float* sn = smn + ux4 * SZ + 4 * uz4;
            float4 v[5];
            adj_products(ld4(sn), ld4(sn + SMEM_FIELD), ld4(sn + 2 * SMEM_FIELD), ld4(sn + 3 * SMEM_FIELD),
                         ld4(sn + 4 * SMEM_FIELD), ldg4(A.par[0] + ui), ldg4(A.par[1] + ui), ldg4(A.par[2] + ui),
                         ldg4(A.par[3] + ui), ldg4(A.par[4] + ui), v);
#pragma unroll
            for (int f = 0; f < 5; f++) st4(sn + f * SMEM_FIELD, v[f]);
        };
        combine(tzi + 1, txi + FAT);
        if (tid < NHALO) combine(hz, hx);
        __syncthreads();
    }

    // ---------------------------------------------------------------- step B
    float4 t[5];
    stencil_core<DIR>(smn, FAT + txi, FAT + 4 * tzi, B.cz, B.cx, valid, [&](int k) { return ldg4(B.par[k] + gi); }, t);
    float4 csave[2];
    if (EPI == EPI_TRI && DIR == 0) {
        csave[0] = ld4(smn + (FAT + txi) * SZ + FAT + 4 * tzi);
        csave[1] = ld4(smn + SMEM_FIELD + (FAT + txi) * SZ + FAT + 4 * tzi);
    }
    // old level of step B = level t: raw values in smc (forward), global (adjoint)
    auto old = [&](int f) {
        if (DIR == 0) return ld4(smc + f * CFIELD + (PH + txi) * CZ + PH + 4 * tzi);
        return ld4(A.c[f] + gi);
    };
    step_tail<DIR, EPI, 0, 5, NT, decltype(old), false>(B, smc, tile, tid, tzi, txi, gz, gx, valid, gi, t, old, csave);
}

}  // namespace eio
