// Persistent time loop: every fine step of a propagation phase (of one shot
// or a group of shots in lockstep) in ONE launch.
//
// The per-step launches of the time loops (eio_engine.cu) pay, at every fine
// step, the launch, the ramp-up of a fresh grid and the drain of its last
// wave, with every CTA of a wave loading, then computing, then storing in step
// with the others.  Here a cooperative grid of resident CTAs walks the steps
// itself: CTA b owns the units (shot, tile) u = b, b + G, ... (shots of a tile
// next to each other, as k_step_shots orders them) and, for step s, works on
// each of its units once the tile's eight neighbours have finished step s-1:
//   * a tile reads its neighbours' level s (the stencil halo) and
//   * overwrites its own level s-1, which its neighbours read as their halo
//     at step s-1,
// so "every neighbour has finished step s-1" is the one condition a unit
// waits for (true dependency and anti-dependency; the diagonal neighbours are
// included because the staged halo box reaches into their corners).  A
// per-unit counter holds the steps finished: the CTA publishes it after a
// barrier and a fence; eight threads of a waiting CTA poll one neighbour each
// and fence before the barrier that releases the CTA.  Wavefield reads go through L2 (step_body_sm with COH).  CTAs
// drift apart instead of meeting at a grid-wide barrier every step, so one
// CTA's loads overlap another's stencils and no step pays a ramp or a tail.
//
// No deadlock: every CTA finishes all its units of step s before any of step
// s+1, so the units of the lowest step in progress always find their
// neighbours done; all CTAs are resident (cooperative launch).  Waits are
// bounded: a unit whose neighbours do not arrive within the poll limit sets
// the error flag and its CTA returns; the others then run out of polls too.
//
// The per-step arguments are the StepArgs the per-launch loops build (a
// device array [nsteps][nb]); the epilogue of each step is a runtime choice.
// The Born forward's secondary sources of coarse sample k are computed by the
// owning CTA for its own tile just before the first step that needs them
// (imaging_body_sm into a two-slot ring), so that phase needs no second stream.
#pragma once
#include "eio_kernels.cuh"

namespace eio {

// per-step flag: the forward scattered phase first computes the secondary
// sources of coarse sample ss_k (imaging_body_sm)
constexpr int WAVE_SS = 8;

struct WaveArgs {
    const StepArgs* plan;          // [nsteps][nb]
    const int* mode;               // [nsteps]: WAVE_SS or 0
    const int* ss_k;               // [nsteps]: coarse sample of the secondary sources (WAVE_SS)
    ImagingArgs img[STEP_BATCH];   // per shot: history, perturbation (ss and its set per use)
    float* ss[STEP_BATCH][2][5];   // per shot: the two ring slots (sample k in slot k % 2)
    int* done;                     // [nb * max_tiles]: steps finished per unit (zeroed before the launch)
    int* err;
    long long wait_limit;          // polls of one neighbour wait
    int nsteps, nb, max_tiles;
};

__device__ __forceinline__ int ld_relaxed(const int* p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(int* p, int v)
{
    asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Threads 0..7 each wait for one of the eight neighbours of tile (bz, bx) of
// shot `shot` to have finished `need` steps (a neighbour outside the tile grid
// counts as done); relaxed polls, then a fence, so that the barrier after
// this orders every thread's later reads after the neighbours' writes.
// Returns false on a thread whose neighbour did not arrive within the limit.
__device__ __forceinline__ bool wave_wait(const WaveArgs& w, int shot, int bz, int bx, int ntz, int ntx, int need)
{
    const int t = threadIdx.x;
    if (t >= 8) return true;
    const int k = t < 4 ? t : t + 1;           // skip the centre of the 3 x 3 block
    const int z = bz + k % 3 - 1, x = bx + k / 3 - 1;
    if (z < 0 || z >= ntz || x < 0 || x >= ntx) return true;
    const int* f = w.done + (size_t)shot * w.max_tiles + x * ntz + z;
    long long polls = 0;
    while (ld_relaxed(f) < need) {
        if (++polls > w.wait_limit) return false;
        __nanosleep(20);
    }
    __threadfence();
    return true;
}

// One epilogue for every step of a phase: EPI_TRI (source wavefield; the
// steps without a coarse sample have tmode 0, which makes them plain steps),
// EPI_INJ_SS (scattered field), EPI_TRI_IMG (adjoint; tmode 0 the same way),
// EPI_NONE (nonlinear operators).
template <int DIR, int EPI, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_wave(const __grid_constant__ WaveArgs w)
{
    __shared__ __align__(16) float sm[5 * SMEM_FIELD];
    const int units = w.nb * w.max_tiles;
    for (int s = 0; s < w.nsteps; s++) {
        const int mode = __ldg(w.mode + s);
        for (int u = blockIdx.x; u < units; u += gridDim.x) {
            const int shot = u % w.nb, tile = u / w.nb;
            const StepArgs& a = w.plan[(size_t)s * w.nb + shot];
            const int ntz = a.ntz, ntx = (a.nx - 2 * FAT) / TX;
            if (tile >= ntz * ntx) continue;   // CTA-uniform: a shot with fewer tiles
            if (s > 0) {
                const bool ok = wave_wait(w, shot, tile % ntz, tile / ntz, ntz, ntx, s);
                if (!ok) atomicExch(w.err, 1);
                if (!__syncthreads_and(ok)) return;   // CTA-uniform
            }
            if constexpr (EPI == EPI_INJ_SS) {
                if (mode & WAVE_SS) {
                    const int k = __ldg(w.ss_k + s);
                    imaging_body_sm<0, 0>(w.img[shot], tile, sm, k, w.ss[shot][k & 1]);
                    __syncthreads();           // the snapshot stage is free again
                }
            }
            step_body_sm<DIR, EPI, MINB, false, true>(a, tile, sm);
            __syncthreads();                   // every store of this unit's step issued
            if (threadIdx.x == 0) {
                __threadfence();               // ... and visible at gpu scope before the count
                st_relaxed(w.done + (size_t)shot * w.max_tiles + tile, s + 1);
            }
        }
    }
}

}  // namespace eio
