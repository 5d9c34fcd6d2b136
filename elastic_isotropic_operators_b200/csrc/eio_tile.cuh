// Persistent TMA-pipelined version of the fused fine step (same semantics and
// 64x16-cell tiles as k_step in eio_kernels.cuh, see there for the reference
// citations).
//
// One CTA per SM walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...
// Every input of a tile arrives in shared memory by cp.async.bulk.tensor
// (TMA) on one mbarrier, into one of two stages:
//   forward: current level with its 4-cell halo (5 boxes 72x24), old level
//            and medium at the tile cells (10 boxes 64x16)     = 75.5 KB
//   adjoint: current level and medium with halo (10 boxes 72x24), old level
//            (5 boxes 64x16); the scaled combinations are formed in place = 87.5 KB
// At the top of iteration i thread 0 issues the copies of tile i+1 into the
// other stage (freed by the barrier that closed iteration i-1), so HBM reads
// of the next tile overlap the stencils of this one.  Every mbarrier wait is
// bounded: on timeout the CTA sets the error flag, waits (bounded) for its
// copies in flight and returns.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "eio_sweep.cuh"

namespace eio {

struct TileArgs {
    CUtensorMap tc[5];    // current level, box SZ x SX
    CUtensorMap to[5];    // old level, box TZ x TX
    CUtensorMap tp[5];    // medium: forward box TZ x TX, adjoint box SZ x SX
    StepArgs s;           // everything else, as for k_step
    int ntiles;
    int* err;
    long long wait_limit;   // try_wait polls of a pipeline wait (the drain always gets DRAIN_LIMIT)
};

template <int DIR>
struct TileLayout {
    static constexpr int FI = TX * TZ;                            // floats per interior box
    static constexpr int C = 0;                                   // [5][SX][SZ]
    static constexpr int P = C + 5 * SMEM_FIELD;                  // medium
    static constexpr int O = P + (DIR == 0 ? 5 * FI : 5 * SMEM_FIELD);   // old level [5][TX][TZ]
    static constexpr int STAGE = O + 5 * FI;                      // floats per stage
    static constexpr int SCRATCH = 2 * STAGE;                     // sparse staging [5][TX][TZ]
    static constexpr int BAR = SCRATCH + 5 * FI;                  // 2 mbarriers
    static constexpr size_t BYTES = (size_t)BAR * 4 + 16;
    static constexpr unsigned TXB = (DIR == 0 ? 5 * SMEM_FIELD + 10 * FI : 10 * SMEM_FIELD + 5 * FI) * 4;
};

// bounded, CTA-uniform wait; false after a timeout (error flag set)
__device__ __forceinline__ bool tile_wait(unsigned long long* bar, unsigned parity, int* err, long long limit)
{
    const bool ok = mbar_wait(bar, parity, limit);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0 && err) atomicExch(err, 1);
        return false;
    }
    return true;
}

template <int DIR>
__device__ __forceinline__ void tile_issue(const TileArgs& ta, float* st, unsigned long long* bar, int tile)
{
    using Ly = TileLayout<DIR>;
    const int ntz = ta.s.ntz;
    const int z0 = FAT + (tile % ntz) * TZ, x0 = FAT + (tile / ntz) * TX;
    // generic-proxy reads of this stage (previous tile) are ordered before the async-proxy writes
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, Ly::TXB);
    // z coordinates z0 - FAT = 64*bz and z0 = 4 + 64*bz are multiples of 4 floats (16 B)
#pragma unroll
    for (int f = 0; f < 5; f++) tma_load_2d(st + Ly::C + f * SMEM_FIELD, &ta.tc[f], z0 - FAT, x0 - FAT, bar);
    if (DIR == 0) {
#pragma unroll
        for (int f = 0; f < 5; f++) tma_load_2d(st + Ly::P + f * Ly::FI, &ta.tp[f], z0, x0, bar);
    } else {
#pragma unroll
        for (int f = 0; f < 5; f++) tma_load_2d(st + Ly::P + f * SMEM_FIELD, &ta.tp[f], z0 - FAT, x0 - FAT, bar);
    }
#pragma unroll
    for (int f = 0; f < 5; f++) tma_load_2d(st + Ly::O + f * Ly::FI, &ta.to[f], z0, x0, bar);
}

template <int DIR, int EPI>
__global__ void __launch_bounds__(NT, 1) k_tile(const __grid_constant__ TileArgs ta)
{
    using Ly = TileLayout<DIR>;
    extern __shared__ __align__(128) float sm[];
    const StepArgs& a = ta.s;
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm + Ly::BAR);
    float* scratch = sm + Ly::SCRATCH;
    const int tid = threadIdx.x;
    const int nz = a.nz;
    const int tzi = tid % NTZ, txi = tid / NTZ;
    const int lz = FAT + 4 * tzi;
    const int lx = FAT + txi;
    const int li = txi * TZ + 4 * tzi;         // my float4 in an interior box

    if (blockIdx.x >= ta.ntiles) return;       // CTA-uniform
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        tile_issue<DIR>(ta, sm, bar, blockIdx.x);
    }
    __syncthreads();

    int i = 0;
    for (int tile = blockIdx.x; tile < ta.ntiles; tile += gridDim.x, i++) {
        const int s = i & 1;
        float* st = sm + s * Ly::STAGE;
        const int next = tile + gridDim.x;
        if (tid == 0 && next < ta.ntiles) tile_issue<DIR>(ta, sm + (s ^ 1) * Ly::STAGE, bar + (s ^ 1), next);
        if (!tile_wait(bar + s, (i >> 1) & 1, ta.err, ta.wait_limit)) {
            // drain: this stage and, if issued, the next one
            mbar_wait(bar + s, (i >> 1) & 1, DRAIN_LIMIT);
            if (next < ta.ntiles) mbar_wait(bar + (s ^ 1), ((i + 1) >> 1) & 1, DRAIN_LIMIT);
            return;
        }
        const int z0 = FAT + (tile % a.ntz) * TZ, x0 = FAT + (tile / a.ntz) * TX;
        const int gz = z0 + 4 * tzi;
        const int gx = x0 + txi;
        const bool valid = gz < nz - FAT;
        const long long gi = (long long)gx * nz + gz;

        if (DIR == 1) {
            // scaled combinations in place (cells beyond the grid were filled with zeros)
            const int nq = SZ / 4;
            for (int q = tid; q < nq * SX; q += NT) {
                const int off = (q / nq) * SZ + (q % nq) * 4;
                const float* c = st + Ly::C + off;
                const float* p = st + Ly::P + off;
                float4 v[5];
                adj_products(ld4(c), ld4(c + SMEM_FIELD), ld4(c + 2 * SMEM_FIELD), ld4(c + 3 * SMEM_FIELD),
                             ld4(c + 4 * SMEM_FIELD), ld4(p), ld4(p + SMEM_FIELD), ld4(p + 2 * SMEM_FIELD),
                             ld4(p + 3 * SMEM_FIELD), ld4(p + 4 * SMEM_FIELD), v);
#pragma unroll
                for (int f = 0; f < 5; f++) st4(st + Ly::C + f * SMEM_FIELD + off, v[f]);
            }
            __syncthreads();
        }

        float4 t[5];
        stencil_core<DIR>(st + Ly::C, lx, lz, a.cz, a.cx, valid,
                          [&](int k) { return ld4(st + Ly::P + k * Ly::FI + li); }, t);
        float4 csave[2];
        if (EPI == EPI_TRI && DIR == 0) {
            csave[0] = ld4(st + Ly::C + lx * SZ + lz);
            csave[1] = ld4(st + Ly::C + SMEM_FIELD + lx * SZ + lz);
        }
        step_tail<DIR, EPI, 0, 5, NT>(a, scratch, tile, tid, tzi, txi, gz, gx, valid, gi, t,
                            [&](int f) { return ld4(st + Ly::O + f * Ly::FI + li); }, csave);
        __syncthreads();    // stage s and the scratch are free again
    }
}

}  // namespace eio
