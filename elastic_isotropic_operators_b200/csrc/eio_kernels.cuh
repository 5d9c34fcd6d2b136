// sm_100a kernels for the 2-D isotropic elastic velocity-stress staggered-grid
// engine: one fused kernel per fine time step (leapfrog update of all five
// fields + cosine taper + sparse source/receiver injection/extraction +
// Born dense epilogues), plus the Born secondary-source / imaging kernels.
//
// Reference semantics restated here (paths relative to the reference project,
// F/ = elastic_iso_lib/elastic_iso_float/prop, K = F/src/kernelsGpuElastic.cu):
//   ker_step_fwd K:234-377, ker_step_adj K:380-529, dampCosineEdge K:1192-1221,
//   ker_inject_interp_source_* K:172-189, ker_inject_source_* K:121-168,
//   ker_interp_inject_data_* K:191-229, ker_record_interp_* K:7-60,100-116,
//   interpWavefieldSingleComp K:1337-1346, injectSecondarySource K:1363-1367,
//   extractInterpAdjointWavefield K:1369-1376, imagingElaFwdGpu K:1381-1459,
//   imagingElaAdjGpu K:1538-1613.
//
// Fusion of the taper.  The reference runs  n = o + D(c); n += src;
// damp(n); damp(c); swap  with o and n aliased.  The copy of c damped at step
// k is only consumed as "o" at step k+1, so the second damping of each array
// is deferred to its next use:  n = d * (d * o + D(c) + src).  Every array is
// therefore multiplied by the same taper coefficients in the same order as in
// the reference, without a separate full-grid launch.
//
// Layout: every field is [nx][nz] with z fastest (i = ix*nz + iz), exactly
// the reference layout.  The interior (FAT..n-FAT) is updated; the 4-cell FAT
// frame is never written and stays zero.  nz % 4 == 0 always holds because the
// reference requires (nz - 2*FAT) % 16 == 0, so every column is 16-byte
// aligned and the z axis is processed with float4 vectors.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace eio {

constexpr int FAT = 4;
constexpr int TZ = 64;             // tile cells along z
constexpr int TX = 16;             // tile cells along x
constexpr int NTZ = TZ / 4;        // threads along z (one float4 each)
constexpr int NTX = TX;            // threads along x (one column each)
constexpr int NT = NTZ * NTX;      // 256 threads per CTA
constexpr int SZ = TZ + 2 * FAT;   // shared tile extent along z (72)
constexpr int SX = TX + 2 * FAT;   // shared tile extent along x (24)
constexpr int SMEM_FIELD = SX * SZ;

// sparse point entry: packed local cell + field, and the column of the
// time-major signal matrix of that field
struct PointEntry {
    int key;   // field << 16 | lx << 8 | lz   (lx < TX, lz < TZ)
    int col;
};

struct SparseOp {
    const int* tile_start;    // [ntiles+1] CSR over tiles, or nullptr
    const PointEntry* ent;
    float* sig[5];            // time-major [nt][ld[f]] per field
    int ld[5];
    int t0;                   // coarse (or fine) time row
    float w0, w1;             // time-interpolation weights for rows t0, t0+1
};

// source-wavefield history (coarse Vx / Vz snapshots)
struct WHist {
    const void* Wvx; const void* Wvz;     // float, or 16-bit codes for Q = 1 (BF16) / 2 (FP16)
    const float* wscale;                  // Q > 0: [nts][2] scale of every snapshot (vx, vz)
    long long wstride;
    int nts;
};

struct StepArgs {
    float* o[5];              // old level, overwritten with the new level
    const float* c[5];        // current level
    const float* par[5];      // rhoxDtw, rhozDtw, lamb2MuDtw, lambDtw, muxzDtw
    const float* dampz;       // [nz] taper along z (1 outside the pad band)
    const float* dampx;       // [nx]
    int nz, nx;
    int ntz;                  // number of tiles along z
    float cz[4], cx[4];
    SparseOp inj;             // added before the final taper (sources / data)
    SparseOp ext;             // read after the final taper (receivers / sources)
    // Born dense epilogues
    float* W0; float* W1;     // source history vx / vz, [nts][nx*nz]
    long long wstride;        // nx*nz
    int wt;                   // coarse row
    float ww0, ww1;
    const float* ssL[5]; const float* ssR[5];   // scattered-field injection
    float* eL[5]; float* eR[5];                 // adjoint extraction
    float sw0, sw1;
    // EPI_TRI (two fine steps per coarse sample): one coarse sample written at
    // once from the old (o), current (c) and new (n) levels of this step,
    //   tmode 1: fma(n, tw_n, fma(c, tw_c, o * tw_o));  tmode 2: fma(n, tw_n, c * tw_c)
    // forward: vx, vz into row wt of W0 / W1;  adjoint: all five fields into eL[f]
    int tmode;
    float tw_o, tw_c, tw_n;
    // 16-bit checkpoints: forward EPI_TRI also leaves, per tile and warp, the
    // largest |sample| of vx and vz in pmax[(tile * 16 + warp) * 2 + {0, 1}]
    float* pmax;
    // free surface at z = 2*FAT (surfaceCondition = 1, k_step only): fsc[ix] is
    // the sigmaxx coefficient on the surface row
    int fs;
    const float* fsc;
    // EPI_TRI_IMG (adjoint, k_step only): the coarse adjoint sample of this step
    // goes straight into the imaging condition of coarse sample img_its against
    // the history wh, accumulated into img[5]; no sample buffer is written
    WHist wh;
    int img_its;
    float dts_inv;
    float* img[5];
};

constexpr int SURF = 2 * FAT;   // free-surface row

enum { EPI_NONE = 0, EPI_SAVE_W = 1, EPI_INJ_SS = 2, EPI_EXT_SS = 3, EPI_TRI = 4, EPI_TRI_IMG = 5 };
// EPI_TRI_IMG + Q: the history holds FP32 (Q = 0), BF16 (1) or FP16 (2) snapshots

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
// L2-coherent load (bypasses L1 and the read-only path): for data that other
// CTAs of the same launch write (the persistent time loop, eio_wave.cuh)
__device__ __forceinline__ float4 ldcg4(const float* p) { return __ldcg(reinterpret_cast<const float4*>(p)); }
// a wavefield value another CTA of this launch may have written (COH), or one
// that is constant for the launch
template <bool COH>
__device__ __forceinline__ float4 ldw4(const float* p) { return COH ? ldcg4(p) : ldg4(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float& at(float4& v, int j) { return reinterpret_cast<float*>(&v)[j]; }
__device__ __forceinline__ float at(const float4& v, int j) { return reinterpret_cast<const float*>(&v)[j]; }

// coarse sample of EPI_TRI, same operation order as the reference's running sums
__device__ __forceinline__ float4 tri_sample(int mode, float4 o, float4 c, float4 n, float wo, float wc, float wn)
{
    float4 r;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float a = (mode == 1) ? fmaf(at(c, j), wc, at(o, j) * wo) : at(c, j) * wc;
        at(r, j) = fmaf(at(n, j), wn, a);
    }
    return r;
}


// z-derivatives of 4 consecutive cells from a 12-value window v[-4..7]
// (w = v shifted by +4).  Dminus: sum c_k (f[z+k] - f[z-1-k]); Dplus: sum c_k (f[z+1+k] - f[z-k]).
__device__ __forceinline__ float4 dmz(const float* w, const float* c)
{
    float4 r;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float* v = w + 4 + j;
        at(r, j) = c[0] * (v[0] - v[-1]) + c[1] * (v[1] - v[-2]) + c[2] * (v[2] - v[-3]) + c[3] * (v[3] - v[-4]);
    }
    return r;
}
__device__ __forceinline__ float4 dpz(const float* w, const float* c)
{
    float4 r;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float* v = w + 4 + j;
        at(r, j) = c[0] * (v[1] - v[0]) + c[1] * (v[2] - v[-1]) + c[2] * (v[3] - v[-2]) + c[3] * (v[4] - v[-3]);
    }
    return r;
}
// x-derivatives at column index m of a window of float4 columns q[] (q[m] = column x)
__device__ __forceinline__ float4 dmx(const float4* q, int m, const float* c)
{
    float4 r;
#pragma unroll
    for (int j = 0; j < 4; j++)
        at(r, j) = c[0] * (at(q[m], j) - at(q[m - 1], j)) + c[1] * (at(q[m + 1], j) - at(q[m - 2], j)) +
                   c[2] * (at(q[m + 2], j) - at(q[m - 3], j)) + c[3] * (at(q[m + 3], j) - at(q[m - 4], j));
    return r;
}
__device__ __forceinline__ float4 dpx(const float4* q, int m, const float* c)
{
    float4 r;
#pragma unroll
    for (int j = 0; j < 4; j++)
        at(r, j) = c[0] * (at(q[m + 1], j) - at(q[m], j)) + c[1] * (at(q[m + 2], j) - at(q[m - 1], j)) +
                   c[2] * (at(q[m + 3], j) - at(q[m - 2], j)) + c[3] * (at(q[m + 4], j) - at(q[m - 3], j));
    return r;
}

// Load the 12-value z window for local column lx starting at local z lz (multiple of 4)
// of a staged field with RZ floats per column
template <int RZ = SZ>
__device__ __forceinline__ void zwin(const float* s, int lx, int lz, float* w)
{
    const float* p = s + lx * RZ + lz - FAT;
    float4 a = ld4(p), b = ld4(p + 4), c = ld4(p + 8);
    w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
    w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
    w[8] = c.x; w[9] = c.y; w[10] = c.z; w[11] = c.w;
}
// Load the 10 float4 columns lx0-4 .. lx0+5 at local z lz
__device__ __forceinline__ void xwin(const float* s, int lx0, int lz, float4* q)
{
#pragma unroll
    for (int m = 0; m < 10; m++) q[m] = ld4(s + (lx0 - FAT + m) * SZ + lz);
}

// Stencil part of one fused fine step for the float4 at local (lx, lz) of a
// staged tile (5 fields [..][RZ] at stride FSTR, by default [SX][SZ] at
// SMEM_FIELD): forward, the current level and the medium at the cell from
// par(k); adjoint, the staged scaled combinations.  t[f] receives the update
// of fields F0 <= f < F1 before the old level is added; the field groups
// {vx, vz} and {sxx, szz, sxz} need four derivatives each.
template <int DIR, int F0, int F1, class Par, int RZ = SZ, int FSTR = SMEM_FIELD>
__device__ __forceinline__ void stencil_fields(const float* sm, int lx, int lz, const float* cz, const float* cx,
                                               bool valid, Par par, float4 (&t)[5])
{
    static_assert((F0 == 0 && F1 == 5) || (F0 == 0 && F1 == 2) || (F0 == 2 && F1 == 5), "field group");
    const float* s0 = sm;
    const float* s1 = sm + FSTR;
    const float* s2 = sm + 2 * FSTR;
    const float* s3 = sm + 3 * FSTR;
    const float* s4 = sm + 4 * FSTR;
    float4 q[9];
    float w[12];
    auto xw = [&](const float* sf) {
#pragma unroll
        for (int m = 0; m < 9; m++) q[m] = ld4(sf + (lx - FAT + m) * RZ + lz);
    };
    if (DIR == 0) {
        // s0 vx, s1 vz, s2 sxx, s3 szz, s4 sxz; one output field at a time keeps few registers live
        if (F0 == 0) {
            xw(s2); float4 dx = dmx(q, 4, cx);
            zwin<RZ>(s4, lx, lz, w); float4 dz = dpz(w, cz);
            if (valid) {
                const float4 rx = par(0);
#pragma unroll
                for (int j = 0; j < 4; j++) at(t[0], j) = at(rx, j) * (at(dx, j) + at(dz, j));
            }
            zwin<RZ>(s3, lx, lz, w); dz = dmz(w, cz);
            xw(s4); dx = dpx(q, 4, cx);
            if (valid) {
                const float4 rz = par(1);
#pragma unroll
                for (int j = 0; j < 4; j++) at(t[1], j) = at(rz, j) * (at(dz, j) + at(dx, j));
            }
        }
        if (F1 == 5) {
            xw(s0); float4 dx = dpx(q, 4, cx);
            zwin<RZ>(s1, lx, lz, w); float4 dz = dpz(w, cz);
            if (valid) {
                const float4 l2m = par(2), lam = par(3);
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    at(t[2], j) = at(l2m, j) * at(dx, j) + at(lam, j) * at(dz, j);
                    at(t[3], j) = at(lam, j) * at(dx, j) + at(l2m, j) * at(dz, j);
                }
            }
            zwin<RZ>(s0, lx, lz, w); dz = dmz(w, cz);
            xw(s1); dx = dmx(q, 4, cx);
            if (valid) {
                const float4 mu = par(4);
#pragma unroll
                for (int j = 0; j < 4; j++) at(t[4], j) = at(mu, j) * (at(dz, j) + at(dx, j));
            }
        }
    } else {
        // s0 A=l2m*sxx+lam*szz, s1 B=lam*sxx+l2m*szz, s2 M=mu*sxz, s3 P=rhox*vx, s4 Q=rhoz*vz
        if (F0 == 0) {
            xw(s0); float4 dx = dmx(q, 4, cx);
            zwin<RZ>(s2, lx, lz, w); float4 dz = dpz(w, cz);
#pragma unroll
            for (int j = 0; j < 4; j++) at(t[0], j) = -(at(dx, j) + at(dz, j));
            zwin<RZ>(s1, lx, lz, w); dz = dmz(w, cz);
            xw(s2); dx = dpx(q, 4, cx);
#pragma unroll
            for (int j = 0; j < 4; j++) at(t[1], j) = -(at(dz, j) + at(dx, j));
        }
        if (F1 == 5) {
            xw(s3); float4 dx = dpx(q, 4, cx);
#pragma unroll
            for (int j = 0; j < 4; j++) at(t[2], j) = -at(dx, j);
            zwin<RZ>(s4, lx, lz, w); float4 dz = dpz(w, cz);
#pragma unroll
            for (int j = 0; j < 4; j++) at(t[3], j) = -at(dz, j);
            zwin<RZ>(s3, lx, lz, w); dz = dmz(w, cz);
            xw(s4); dx = dmx(q, 4, cx);
#pragma unroll
            for (int j = 0; j < 4; j++) at(t[4], j) = -(at(dz, j) + at(dx, j));
        }
    }
}

template <int DIR, class Par>
__device__ __forceinline__ void stencil_core(const float* sm, int lx, int lz, const float* cz, const float* cx,
                                             bool valid, Par par, float4 (&t)[5])
{
    stencil_fields<DIR, 0, 5>(sm, lx, lz, cz, cx, valid, par, t);
}

// adjoint staging: the scaled combinations the transposed stencils act on
__device__ __forceinline__ void adj_products(float4 vx, float4 vz, float4 sxx, float4 szz, float4 sxz, float4 rx,
                                             float4 rz, float4 l2m, float4 lam, float4 mu, float4 (&v)[5])
{
#pragma unroll
    for (int j = 0; j < 4; j++) {
        at(v[0], j) = at(l2m, j) * at(sxx, j) + at(lam, j) * at(szz, j);  // -> d/dx-  (vx)
        at(v[1], j) = at(lam, j) * at(sxx, j) + at(l2m, j) * at(szz, j);  // -> d/dz-  (vz)
        at(v[2], j) = at(mu, j) * at(sxz, j);                             // -> vx, vz
        at(v[3], j) = at(rx, j) * at(vx, j);                              // -> sxx, sxz
        at(v[4], j) = at(rz, j) * at(vz, j);                              // -> szz, sxz
    }
}

// Four consecutive history values of snapshot `its` at cell index i (float4
// aligned) of field f (0 vx, 1 vz): FP32, or 16-bit codes times the snapshot scale.
template <int Q>
__device__ __forceinline__ float4 ldw(const WHist& a, int f, int its, long long i)
{
    const long long k = (long long)its * a.wstride + i;
    const void* base = f ? a.Wvz : a.Wvx;
    if (Q == 0) return ldg4(static_cast<const float*>(base) + k);
    const uint2 u = __ldg(reinterpret_cast<const uint2*>(static_cast<const unsigned short*>(base) + k));
    const float s = __ldg(a.wscale + 2 * its + f);
    const unsigned h[4] = {u.x & 0xffffu, u.x >> 16, u.y & 0xffffu, u.y >> 16};
    float4 r;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float v;
        if (Q == 1) v = __uint_as_float(h[j] << 16);                       // BF16: upper half of a float
        else v = __half2float(__ushort_as_half((unsigned short)h[j]));     // FP16
        at(r, j) = v * s;
    }
    return r;
}

// snapshot `its` (vx, vz) of tile (z0, x0) with its 4-cell halo into sm [2][SX][SZ]; NT threads
template <int Q>
__device__ __forceinline__ void stage_snapshot(const WHist& h, int its, int nz, float* sm, int z0, int x0, int tid)
{
    const int nq = SZ / 4;
    for (int q = tid; q < nq * SX; q += NT) {
        const int lx = q / nq, lz4 = (q % nq) * 4;
        const int gz = z0 - FAT + lz4, gx = x0 - FAT + lx;
        float4 u = make_float4(0.f, 0.f, 0.f, 0.f), v = u;
        if (gz < nz) {
            const long long gi = (long long)gx * nz + gz;
            u = ldw<Q>(h, 0, its, gi);
            v = ldw<Q>(h, 1, its, gi);
        }
        st4(sm + lx * SZ + lz4, u);
        st4(sm + SMEM_FIELD + lx * SZ + lz4, v);
    }
}

// The source-wavefield terms of both imaging kernels at the float4 (lx, lz) of a
// staged snapshot: staggered derivatives of Vx, Vz and their time difference
// W[its-1] - W[its+1] (one-sided at the ends like the reference).
struct ImgTerms {
    float4 dvx_dx, dvx_dz, dvz_dx, dvz_dz, tx, tz;
};
template <int Q>
__device__ __forceinline__ ImgTerms imaging_terms(const WHist& h, const float* sm, int lx, int lz, long long gi,
                                                  int its, const float* cz, const float* cx)
{
    ImgTerms r;
    const float* svx = sm;
    const float* svz = sm + SMEM_FIELD;
    float4 q[9];
    float w[12];
#pragma unroll
    for (int m = 0; m < 9; m++) q[m] = ld4(svx + (lx - FAT + m) * SZ + lz);
    r.dvx_dx = dpx(q, 4, cx);
    zwin(svx, lx, lz, w);
    r.dvx_dz = dmz(w, cz);
#pragma unroll
    for (int m = 0; m < 9; m++) q[m] = ld4(svz + (lx - FAT + m) * SZ + lz);
    r.dvz_dx = dmx(q, 4, cx);
    zwin(svz, lx, lz, w);
    r.dvz_dz = dpz(w, cz);
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 xo = its > 0 ? ldw<Q>(h, 0, its - 1, gi) : zero;
    const float4 zo = its > 0 ? ldw<Q>(h, 1, its - 1, gi) : zero;
    const float4 xn = its < h.nts - 1 ? ldw<Q>(h, 0, its + 1, gi) : zero;
    const float4 zn = its < h.nts - 1 ? ldw<Q>(h, 1, its + 1, gi) : zero;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        // one-sided at the ends like the reference: -W[its+1] at its = 0, W[its-1] at nts-1
        at(r.tx, j) = (its == 0) ? -at(xn, j) : (its == h.nts - 1) ? at(xo, j) : at(xo, j) - at(xn, j);
        at(r.tz, j) = (its == 0) ? -at(zn, j) : (its == h.nts - 1) ? at(zo, j) : at(zo, j) - at(zn, j);
    }
    return r;
}

// imaging condition (imagingElaAdjGpu, K:1538-1613): the images at gi += the
// adjoint sample s[5] against the source-wavefield terms
template <bool COH = false>
__device__ __forceinline__ void imaging_accumulate(float* const dm[5], long long gi, const float4 (&s)[5],
                                                   const ImgTerms& t, float dts_inv)
{
    auto ld = [&](const float* p) { return COH ? ldcg4(p) : ld4(p); };
    float4 d0 = ld(dm[0] + gi), d1 = ld(dm[1] + gi), d2 = ld(dm[2] + gi), d3 = ld(dm[3] + gi),
           d4 = ld(dm[4] + gi);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float dvx = at(t.dvx_dx, j), dvz = at(t.dvz_dz, j);
        at(d0, j) += at(s[0], j) * at(t.tx, j) * dts_inv;
        at(d1, j) += at(s[1], j) * at(t.tz, j) * dts_inv;
        at(d2, j) += (at(s[2], j) + at(s[3], j)) * (dvx + dvz);
        at(d3, j) += 2.0f * (dvx * at(s[2], j) + dvz * at(s[3], j));
        at(d4, j) += at(s[4], j) * (at(t.dvx_dz, j) + at(t.dvz_dx, j));
    }
    st4(dm[0] + gi, d0); st4(dm[1] + gi, d1); st4(dm[2] + gi, d2);
    st4(dm[3] + gi, d3); st4(dm[4] + gi, d4);
}

// Everything of one fused fine step after the stencils, for the float4 of
// thread (tzi, txi) of tile `tile` and the fields F0 <= f < F1: deferred taper
// of the old level (o(f) returns it), leapfrog sum, scattered-field source,
// sparse injection, final taper, store of the new level, dense Born
// epilogues, sparse extraction.  NTHR threads of the CTA take part (every one
// reaches the same barriers); scratch: >= 5*TX*TZ floats of shared memory that
// the stencils no longer need.
template <int DIR, int EPI, int F0, int F1, int NTHR, class Old, bool FS = false, bool COH = false>
__device__ __forceinline__ void step_tail(const StepArgs& a, float* scratch, int tile, int tid, int tzi, int txi,
                                          int gz, int gx, bool valid, long long gi, float4 (&t)[5], Old oload,
                                          const float4 (&csave)[2])
{
    constexpr bool IMG = EPI >= EPI_TRI_IMG;                 // sample straight into the imaging condition
    constexpr bool TRI = EPI == EPI_TRI || IMG;
    static_assert(!IMG || (DIR == 1 && NTHR == NT && F0 == 0 && F1 == 5), "fused imaging: adjoint k_step only");
    float4 osave[5];      // old level (EPI_TRI)
    float4 smp[5];        // coarse adjoint samples (EPI_TRI_IMG)
    float tri_max[2] = {0.f, 0.f};   // |max| of this thread's coarse samples (16-bit checkpoints)
    float dd[4];
    {
        const float dxc = __ldg(a.dampx + gx);
#pragma unroll
        for (int j = 0; j < 4; j++) dd[j] = valid ? fminf(__ldg(a.dampz + gz + j), dxc) : 1.f;
    }
    if (valid) {
#pragma unroll
        for (int f = F0; f < F1; f++) {
            const float4 o = oload(f);
            if (TRI) osave[f] = o;
#pragma unroll
            for (int j = 0; j < 4; j++) at(t[f], j) = dd[j] * at(o, j) + at(t[f], j);
        }
        if (EPI == EPI_INJ_SS) {
            // with two fine steps per coarse sample every other step has sw1 == 0:
            // the right slice is then not read (ssR * 0 adds nothing)
            const bool right = a.sw1 != 0.f;
#pragma unroll
            for (int f = F0; f < F1; f++) {
                const float4 l = ldw4<COH>(a.ssL[f] + gi);
                const float4 r = right ? ldw4<COH>(a.ssR[f] + gi) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int j = 0; j < 4; j++) at(t[f], j) += at(l, j) * a.sw0 + at(r, j) * a.sw1;
            }
        }
    }

    // ---- free surface, adjoint: transpose of the top pass on the column
    // (the mirrored stress rows return to their sources below the surface,
    // the rows the top pass overwrites get nothing)
    if (FS && DIR == 1 && a.fs && tile % a.ntz == 0) {   // CTA-uniform
        __shared__ float fsv[2][5][TX];            // sigmazz, sigmaxz on rows SURF-4 .. SURF
        if (valid && F0 <= 3 && F1 >= 5) {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int row = gz + j;
                if (row >= SURF - 4 && row <= SURF) {
                    fsv[0][row - (SURF - 4)][txi] = at(t[3], j);
                    fsv[1][row - (SURF - 4)][txi] = at(t[4], j);
                }
            }
        }
        __syncthreads();
        if (valid) {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int row = gz + j;
                if (F0 <= 3 && F1 >= 5) {
                    if (row > SURF && row <= SURF + 4) {
                        at(t[3], j) -= fsv[0][(2 * SURF - row) - (SURF - 4)][txi];     // szz[S+k] -= szz[S-k]
                        at(t[4], j) -= fsv[1][(2 * SURF + 1 - row) - (SURF - 4)][txi]; // sxz[S+1+k] -= sxz[S-k]
                    }
                    if (row >= SURF - 4 && row <= SURF) at(t[3], j) = 0.f;
                    if (row >= SURF - 3 && row <= SURF) at(t[4], j) = 0.f;
                }
                if (F0 == 0) {
                    if (row >= SURF - 4 && row < SURF) at(t[0], j) = 0.f;
                    if (row >= SURF - 4 && row <= SURF) at(t[1], j) = 0.f;
                }
            }
        }
    }

    // ---- sparse injection (sources / adjoint data), before the final taper
    if (a.inj.tile_start) {
        const int e0 = a.inj.tile_start[tile], e1 = a.inj.tile_start[tile + 1];
        if (e1 > e0) {   // CTA-uniform
            float* acc = scratch;                 // [5][TX][TZ]
            __syncthreads();
            for (int i = tid; i < 5 * TX * TZ; i += NTHR) acc[i] = 0.f;
            __syncthreads();
            for (int e = e0 + tid; e < e1; e += NTHR) {
                const PointEntry pe = a.inj.ent[e];
                const int f = pe.key >> 16, lx = (pe.key >> 8) & 0xff, lzz = pe.key & 0xff;
                const float* sg = a.inj.sig[f];
                const int ld = a.inj.ld[f];
                const float v = sg[(long long)a.inj.t0 * ld + pe.col] * a.inj.w0 +
                                sg[(long long)(a.inj.t0 + 1) * ld + pe.col] * a.inj.w1;
                atomicAdd(acc + (f * TX + lx) * TZ + lzz, v);
            }
            __syncthreads();
            if (valid) {
#pragma unroll
                for (int f = F0; f < F1; f++) {
                    const float4 v = ld4(acc + (f * TX + txi) * TZ + 4 * tzi);
#pragma unroll
                    for (int j = 0; j < 4; j++) at(t[f], j) += at(v, j);
                }
            }
        }
    }

    // ---- final taper, store, dense epilogues
    if (valid) {
#pragma unroll
        for (int f = F0; f < F1; f++) {
#pragma unroll
            for (int j = 0; j < 4; j++) at(t[f], j) *= dd[j];
            st4(a.o[f] + gi, t[f]);
        }
        if (EPI == EPI_SAVE_W && F0 == 0) {
            float* w0p = a.W0 + (long long)a.wt * a.wstride + gi;
            float* w1p = a.W1 + (long long)a.wt * a.wstride + gi;
            float4 u0 = ld4(w0p), u1 = ld4(w0p + a.wstride), v0 = ld4(w1p), v1 = ld4(w1p + a.wstride);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                at(u0, j) += at(t[0], j) * a.ww0; at(u1, j) += at(t[0], j) * a.ww1;
                at(v0, j) += at(t[1], j) * a.ww0; at(v1, j) += at(t[1], j) * a.ww1;
            }
            st4(w0p, u0); st4(w0p + a.wstride, u1); st4(w1p, v0); st4(w1p + a.wstride, v1);
        }
        if (EPI == EPI_EXT_SS) {
#pragma unroll
            for (int f = F0; f < F1; f++) {
                float4 l = ld4(a.eL[f] + gi), r = ld4(a.eR[f] + gi);
#pragma unroll
                for (int j = 0; j < 4; j++) { at(l, j) += at(t[f], j) * a.sw0; at(r, j) += at(t[f], j) * a.sw1; }
                st4(a.eL[f] + gi, l); st4(a.eR[f] + gi, r);
            }
        }
        if (TRI && a.tmode) {
            if (DIR == 0) {
                if (F0 == 0) {
                    const float4 s0 = tri_sample(a.tmode, osave[0], csave[0], t[0], a.tw_o, a.tw_c, a.tw_n);
                    const float4 s1 = tri_sample(a.tmode, osave[1], csave[1], t[1], a.tw_o, a.tw_c, a.tw_n);
                    st4(a.W0 + (long long)a.wt * a.wstride + gi, s0);
                    st4(a.W1 + (long long)a.wt * a.wstride + gi, s1);
                    tri_max[0] = fmaxf(fmaxf(fabsf(s0.x), fabsf(s0.y)), fmaxf(fabsf(s0.z), fabsf(s0.w)));
                    tri_max[1] = fmaxf(fmaxf(fabsf(s1.x), fabsf(s1.y)), fmaxf(fabsf(s1.z), fabsf(s1.w)));
                }
            } else {
#pragma unroll
                for (int f = F0; f < F1; f++) {
                    smp[f] = tri_sample(a.tmode, osave[f], COH ? ldcg4(a.c[f] + gi) : ld4(a.c[f] + gi), t[f],
                                        a.tw_o, a.tw_c, a.tw_n);
                    if (!IMG) st4(a.eL[f] + gi, smp[f]);
                }
            }
        }
    }

    if (EPI == EPI_TRI && DIR == 0 && F0 == 0) {
        if (a.pmax && a.tmode) {              // uniform over the CTA
#pragma unroll
            for (int f = 0; f < 2; f++) {
                float m = tri_max[f];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
                if ((tid & 31) == 0) a.pmax[((long long)tile * 16 + (tid >> 5)) * 2 + f] = m;
            }
        }
    }

    // ---- sparse extraction (receivers / adjoint sources), after the final taper
    if (a.ext.tile_start) {
        const int e0 = a.ext.tile_start[tile], e1 = a.ext.tile_start[tile + 1];
        if (e1 > e0) {
            float* stg = scratch;                 // [5][TX][TZ]
            __syncthreads();
            if (valid) {
#pragma unroll
                for (int f = F0; f < F1; f++) st4(stg + (f * TX + txi) * TZ + 4 * tzi, t[f]);
            }
            __syncthreads();
            for (int e = e0 + tid; e < e1; e += NTHR) {
                const PointEntry pe = a.ext.ent[e];
                const int f = pe.key >> 16, lx = (pe.key >> 8) & 0xff, lzz = pe.key & 0xff;
                const float v = stg[(f * TX + lx) * TZ + lzz];
                float* sg = a.ext.sig[f];
                const int ld = a.ext.ld[f];
                sg[(long long)a.ext.t0 * ld + pe.col] += v * a.ext.w0;
                sg[(long long)(a.ext.t0 + 1) * ld + pe.col] += v * a.ext.w1;
            }
        }
    }

    // ---- imaging condition of coarse sample img_its (EPI_TRI_IMG): the snapshot
    // with its halo in the scratch, then the same terms as k_imaging<1>
    if (IMG && a.tmode) {   // uniform over the CTA
        constexpr int Q = EPI - EPI_TRI_IMG;
        __syncthreads();   // the scratch is free
        stage_snapshot<Q>(a.wh, a.img_its, a.nz, scratch, gz - 4 * tzi, gx - txi, tid);
        __syncthreads();
        if (valid) {
            const ImgTerms it = imaging_terms<Q>(a.wh, scratch, FAT + txi, FAT + 4 * tzi, gi, a.img_its, a.cz, a.cx);
            imaging_accumulate<COH>(a.img, gi, smp, it, a.dts_inv);
        }
    }
}

// Free surface, top pass on the current level before each forward step
// (ker_step_fwd_surface_top, K:543-587): sigmazz = 0 on the surface, sigmazz
// and sigmaxz mirrored with opposite sign above it, vx and vz zero above it
// (vz also on it).  One thread per interior column.
__global__ void __launch_bounds__(128) k_fs_top(float* vx, float* vz, float* szz, float* sxz, int nz, int nx)
{
    const int ix = FAT + blockIdx.x * blockDim.x + threadIdx.x;
    if (ix >= nx - FAT) return;
    const long long b = (long long)ix * nz + SURF;
    szz[b] = 0.f;
#pragma unroll
    for (int k = 1; k <= 4; k++) szz[b - k] = -szz[b + k];
#pragma unroll
    for (int k = 0; k < 4; k++) sxz[b - k] = -sxz[b + 1 + k];
#pragma unroll
    for (int k = 1; k <= 4; k++) vx[b - k] = 0.f;
#pragma unroll
    for (int k = 0; k <= 4; k++) vz[b - k] = 0.f;
}

// Free surface, forward update of the rows gz..gz+3 of a thread in the top
// tile row (ker_step_fwd_surface_body, K:589-776): nothing above the surface;
// on it only vx and sigmaxx, the latter with the reduced coefficient fsc.
__device__ __forceinline__ void fs_forward_rows(const StepArgs& a, const float* sm, int lx, int lz, int gz, int gx,
                                                float4 (&t)[5])
{
    if (gz > SURF) return;
    float4 q[9];
#pragma unroll
    for (int m = 0; m < 9; m++) q[m] = ld4(sm + (lx - FAT + m) * SZ + lz);   // staged vx
    const float4 dvx = dpx(q, 4, a.cx);
    const float fc = __ldg(a.fsc + gx);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int row = gz + j;
        if (row < SURF) {
#pragma unroll
            for (int f = 0; f < 5; f++) at(t[f], j) = 0.f;
        } else if (row == SURF) {
            at(t[1], j) = 0.f; at(t[3], j) = 0.f; at(t[4], j) = 0.f;
            at(t[2], j) = fc * at(dvx, j);
        }
    }
}

// Programmatic dependent launch: a step kernel launched with the
// programmatic-serialization attribute may start while the previous kernel of
// the stream drains.  Before griddepcontrol.wait it touches only data no kernel
// writes (the medium, prefetched to L2); every read of the wavefields comes
// after the wait, which returns once the previous grid has completed and its
// writes are visible.  Launched without the attribute, the wait returns at once.
__device__ __forceinline__ void pdl_begin(const StepArgs& a, long long gi, bool valid)
{
    if (valid) {
#pragma unroll
        for (int k = 0; k < 5; k++) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.par[k] + gi));
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Stage the current level (forward) or its scaled combinations (adjoint) of
// tile (z0, x0) with its 4-cell halo into sm [5][SX][SZ]; NTHR threads.
template <int DIR, int NTHR, bool FS = false, bool COH = false>
__device__ __forceinline__ void stage_tile(const StepArgs& a, float* sm, int z0, int x0, int tid)
{
    const int nz = a.nz;
    const int nq = SZ / 4;                        // float4 per shared column
    if constexpr (DIR == 0 && !FS && NTHR == NT) {
        // forward: every load of the thread in flight before the first store
        constexpr int NU = (SZ / 4) * SX;
        constexpr int R = (NU + NT - 1) / NT;
        float4 v[R][5];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int q = tid + r * NT;
            const int lx = q / nq, lz4 = (q % nq) * 4;
            const int gz = z0 - FAT + lz4, gx = x0 - FAT + lx;
            if (q < NU && gz < nz) {
                const long long gi = (long long)gx * nz + gz;
#pragma unroll
                for (int f = 0; f < 5; f++) v[r][f] = ldw4<COH>(a.c[f] + gi);
            } else {
#pragma unroll
                for (int f = 0; f < 5; f++) v[r][f] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int q = tid + r * NT;
            if (q < NU) {
                const int lx = q / nq, lz4 = (q % nq) * 4;
#pragma unroll
                for (int f = 0; f < 5; f++) st4(sm + f * SMEM_FIELD + lx * SZ + lz4, v[r][f]);
            }
        }
    } else {
    for (int q = tid; q < nq * SX; q += NTHR) {
        const int lx = q / nq, lz4 = (q % nq) * 4;
        const int gz = z0 - FAT + lz4, gx = x0 - FAT + lx;
        float4 v[5];
        if (gz < nz) {
            const long long gi = (long long)gx * nz + gz;
            if (DIR == 0) {
#pragma unroll
                for (int f = 0; f < 5; f++) v[f] = ldw4<COH>(a.c[f] + gi);
            } else {
                const float4 sxx = ldw4<COH>(a.c[2] + gi);
                adj_products(ldw4<COH>(a.c[0] + gi), ldw4<COH>(a.c[1] + gi), sxx, ldw4<COH>(a.c[3] + gi),
                             ldw4<COH>(a.c[4] + gi), ldg4(a.par[0] + gi), ldg4(a.par[1] + gi), ldg4(a.par[2] + gi),
                             ldg4(a.par[3] + gi), ldg4(a.par[4] + gi), v);
                if (FS && a.fs && gz <= SURF) {
                    // free surface: only what the forward update uses (see fs_forward_rows)
                    const float fc = __ldg(a.fsc + gx);
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const int row = gz + j;
                        if (row < SURF) {
#pragma unroll
                            for (int f = 0; f < 5; f++) at(v[f], j) = 0.f;
                        } else if (row == SURF) {
                            at(v[0], j) = fc * at(sxx, j);
                            at(v[1], j) = 0.f; at(v[2], j) = 0.f; at(v[4], j) = 0.f;
                        }
                    }
                }
            }
        } else {
#pragma unroll
            for (int f = 0; f < 5; f++) v[f] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int f = 0; f < 5; f++) st4(sm + f * SMEM_FIELD + lx * SZ + lz4, v[f]);
    }
    }
}

// One fused fine step.  DIR 0 = forward (ker_step_fwd), 1 = adjoint (ker_step_adj).
// The current level (forward) or its scaled combinations (adjoint) are staged
// with plain loads; the old level and the medium are read from global memory.
// MINB CTAs per SM (3: <= 80 registers, 4: <= 64).
// COH: the persistent time loop (eio_wave.cuh), where other CTAs of the same
// launch write the wavefields: no programmatic-dependent-launch handshake, and
// every wavefield read goes through L2 (ldcg4).
template <int DIR, int EPI, int MINB, bool FS, bool COH = false>
__device__ __forceinline__ void step_body_sm(const StepArgs& a, int tile, float* sm)
{
    const int tid = threadIdx.x;
    const int bz = tile % a.ntz, bx = tile / a.ntz;
    const int z0 = FAT + bz * TZ, x0 = FAT + bx * TX;
    const int nz = a.nz;
    const int tzi = tid % NTZ, txi = tid / NTZ;
    const int lz = FAT + 4 * tzi;              // local z of my float4
    const int lx = FAT + txi;                  // my local column
    const int gz = z0 + 4 * tzi;
    const int gx = x0 + txi;
    const bool valid = gz < nz - FAT;
    const long long gi = (long long)gx * nz + gz;

    if (!COH) pdl_begin(a, gi, valid);
    stage_tile<DIR, NT, FS, COH>(a, sm, z0, x0, tid);
    // with 3 CTAs per SM the old level is loaded here, its latency hidden
    // behind the barrier and the stencils
    constexpr bool HOIST = MINB == 3 && !FS;
    auto ldo = [&](int f) { return COH ? ldcg4(a.o[f] + gi) : ld4(a.o[f] + gi); };
    float4 oreg[5];
    if (HOIST) {
#pragma unroll
        for (int f = 0; f < 5; f++) oreg[f] = valid ? ldo(f) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();

    float4 t[5];                               // new values before the final taper

    stencil_core<DIR>(sm, lx, lz, a.cz, a.cx, valid, [&](int k) { return ldg4(a.par[k] + gi); }, t);
    if (FS && DIR == 0 && a.fs && bz == 0) fs_forward_rows(a, sm, lx, lz, gz, gx, t);

    float4 csave[2];      // current vx, vz (forward EPI_TRI; shared memory is reused below)
    if (EPI == EPI_TRI && DIR == 0) {
        csave[0] = ld4(sm + lx * SZ + lz);
        csave[1] = ld4(sm + SMEM_FIELD + lx * SZ + lz);
    }
    auto old = [&](int f) { return HOIST ? oreg[f] : ldo(f); };
    step_tail<DIR, EPI, 0, 5, NT, decltype(old), FS, COH>(a, sm, tile, tid, tzi, txi, gz, gx, valid, gi, t, old,
                                                          csave);
}

template <int DIR, int EPI, int MINB, bool FS>
__device__ __forceinline__ void step_body(const StepArgs& a, int tile)
{
    __shared__ __align__(16) float sm[5 * SMEM_FIELD];
    step_body_sm<DIR, EPI, MINB, FS>(a, tile, sm);
}

template <int DIR, int EPI, int MINB = 3, bool FS = false>
__global__ void __launch_bounds__(NT, MINB) k_step(StepArgs a)
{
    step_body<DIR, EPI, MINB, FS>(a, blockIdx.x);
}

// Argument block of the step launches that cover several shots (k_step_shots).
struct StepBatch {
    StepArgs a[STEP_BATCH];
};

// The same step for nb <= STEP_BATCH shots in one launch, with the shots of a
// tile next to each other in the launch order: CTA b runs tile b / nb of shot
// b % nb.  The CTAs of one tile are then resident at the same time; shots that
// share the medium arrays (and the Born perturbation) read a tile of them from
// HBM once, the other shots' reads hit in L2.  Each shot keeps its own
// wavefields, window, taper, point lists and epilogue buffers in its StepArgs;
// a shot's tiles beyond its own count leave before touching memory.
template <int DIR, int EPI, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_step_shots(const __grid_constant__ StepBatch b, int nb)
{
    const int shot = blockIdx.x % nb, tile = blockIdx.x / nb;
    const StepArgs& a = b.a[shot];
    if (tile >= a.ntz * ((a.nx - 2 * FAT) / TX)) return;   // CTA-uniform
    step_body<DIR, EPI, MINB, false>(a, tile);
}

// Same step with two threads per float4: warps 0-7 update vx and vz, warps
// 8-15 sxx, szz and sxz (four derivatives per thread either way), which halves
// the dependent work on a thread's critical path.  2 CTAs per SM, <= 64 registers.
constexpr int NT2 = 2 * NT;

template <int DIR, int EPI>
__global__ void __launch_bounds__(NT2, 2) k_split(StepArgs a)
{
    __shared__ __align__(16) float sm[5 * SMEM_FIELD];

    const int tid = threadIdx.x;
    const int tile = blockIdx.x;
    const int bz = tile % a.ntz, bx = tile / a.ntz;
    const int z0 = FAT + bz * TZ, x0 = FAT + bx * TX;
    const int nz = a.nz;
    const int lt = tid & (NT - 1);
    const int tzi = lt % NTZ, txi = lt / NTZ;
    const int lz = FAT + 4 * tzi;
    const int lx = FAT + txi;
    const int gz = z0 + 4 * tzi;
    const int gx = x0 + txi;
    const bool valid = gz < nz - FAT;
    const long long gi = (long long)gx * nz + gz;

    pdl_begin(a, gi, valid && tid < NT);
    stage_tile<DIR, NT2>(a, sm, z0, x0, tid);
    __syncthreads();
    float4 t[5];
    float4 csave[2];
    auto par = [&](int k) { return ldg4(a.par[k] + gi); };
    auto old = [&](int f) { return ld4(a.o[f] + gi); };
    if (tid < NT) {                            // warp-uniform
        stencil_fields<DIR, 0, 2>(sm, lx, lz, a.cz, a.cx, valid, par, t);
        if (EPI == EPI_TRI && DIR == 0) {
            csave[0] = ld4(sm + lx * SZ + lz);
            csave[1] = ld4(sm + SMEM_FIELD + lx * SZ + lz);
        }
        step_tail<DIR, EPI, 0, 2, NT2>(a, sm, tile, tid, tzi, txi, gz, gx, valid, gi, t, old, csave);
    } else {
        stencil_fields<DIR, 2, 5>(sm, lx, lz, a.cz, a.cx, valid, par, t);
        step_tail<DIR, EPI, 2, 5, NT2>(a, sm, tile, tid, tzi, txi, gz, gx, valid, gi, t, old, csave);
    }
}

// ---------------------------------------------------------------------------
// Born secondary source (imagingElaFwdGpu) and imaging condition (imagingElaAdjGpu)
// One thread per interior cell; W holds coarse Vx/Vz snapshots [nts][nx*nz].
// ---------------------------------------------------------------------------
struct ImagingArgs {
    WHist h;
    int nz, nx, its;
    float cz[4], cx[4];
    float dts_inv;
    float* dm[5];   // fwd: read; adj: accumulated
    float* ss[5];   // fwd: written; adj: read
};

// Born secondary sources (ADJ=0, imagingElaFwdGpu, prop/src/kernelsGpuElastic.cu:1381)
// and imaging condition (ADJ=1, imagingElaAdjGpu, kernelsGpuElastic.cu:1538) at
// coarse sample its.  64x16-cell tiles, 256 threads (one float4 of z x one column
// each); the snapshot at its is staged with its 4-cell halo in shared memory for
// the staggered derivatives, the neighbouring snapshots give the time difference.
// sm: >= 2 * SMEM_FIELD floats of shared memory.  Every thread returns
// through the end (no barrier after the early exit of the threads past the grid).
template <int ADJ, int Q>
__device__ __forceinline__ void imaging_body_sm(const ImagingArgs& a, int tile, float* sm, int its,
                                                float* const* ss)
{
    const int tid = threadIdx.x;
    const int ntz = (a.nz - 2 * FAT + TZ - 1) / TZ;
    const int bz = tile % ntz, bx = tile / ntz;
    const int z0 = FAT + bz * TZ, x0 = FAT + bx * TX;
    const long long nz = a.nz;
    stage_snapshot<Q>(a.h, its, a.nz, sm, z0, x0, tid);
    __syncthreads();
    const int tzi = tid % NTZ, txi = tid / NTZ;
    const int lz = FAT + 4 * tzi, lx = FAT + txi;
    const int gz = z0 + 4 * tzi;
    if (gz >= a.nz - FAT) return;
    const long long gi = (long long)(x0 + txi) * nz + gz;
    const ImgTerms t = imaging_terms<Q>(a.h, sm, lx, lz, gi, its, a.cz, a.cx);
    if (!ADJ) {
        const float4 d0 = ldg4(a.dm[0] + gi), d1 = ldg4(a.dm[1] + gi), dl = ldg4(a.dm[2] + gi),
                     du = ldg4(a.dm[3] + gi), d4 = ldg4(a.dm[4] + gi);
        float4 s0, s1, s2, s3, s4;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            at(s0, j) = at(d0, j) * at(t.tx, j) * a.dts_inv;
            at(s1, j) = at(d1, j) * at(t.tz, j) * a.dts_inv;
            const float dvx = at(t.dvx_dx, j), dvz = at(t.dvz_dz, j);
            at(s2, j) = at(dl, j) * (dvx + dvz) + 2.0f * at(du, j) * dvx;
            at(s3, j) = at(dl, j) * (dvx + dvz) + 2.0f * at(du, j) * dvz;
            at(s4, j) = at(d4, j) * (at(t.dvx_dz, j) + at(t.dvz_dx, j));
        }
        st4(ss[0] + gi, s0); st4(ss[1] + gi, s1); st4(ss[2] + gi, s2);
        st4(ss[3] + gi, s3); st4(ss[4] + gi, s4);
    } else {
        const float4 s[5] = {ldg4(ss[0] + gi), ldg4(ss[1] + gi), ldg4(ss[2] + gi), ldg4(ss[3] + gi),
                             ldg4(ss[4] + gi)};
        imaging_accumulate(a.dm, gi, s, t, a.dts_inv);
    }
}

template <int ADJ, int Q>
__device__ __forceinline__ void imaging_body(const ImagingArgs& a, int tile)
{
    __shared__ __align__(16) float sm[2 * SMEM_FIELD];
    imaging_body_sm<ADJ, Q>(a, tile, sm, a.its, a.ss);
}

template <int ADJ, int Q>
__global__ void __launch_bounds__(NT) k_imaging(ImagingArgs a)
{
    imaging_body<ADJ, Q>(a, blockIdx.x);
}

// k_imaging for nb <= STEP_BATCH shots, the shots of a tile next to each other
// in the launch order (CTA b: tile b / nb of shot b % nb), so that the Born
// perturbation the forward kernels of all shots read comes from HBM once.
struct ImagingBatch {
    ImagingArgs a[STEP_BATCH];
};

template <int ADJ, int Q>
__global__ void __launch_bounds__(NT) k_imaging_shots(const __grid_constant__ ImagingBatch b, int nb)
{
    const int shot = blockIdx.x % nb, tile = blockIdx.x / nb;
    const ImagingArgs& a = b.a[shot];
    if (tile >= ((a.nz - 2 * FAT + TZ - 1) / TZ) * ((a.nx - 2 * FAT) / TX)) return;   // CTA-uniform
    imaging_body<ADJ, Q>(a, tile);
}

// Coarse-time sample of all five fields of the new level (interpWavefield,
// K:1258-1291): W[its][f] += p[f] * w0 and W[its+1][f] += p[f] * w1 at every
// interior cell, W laid out [nts][5][nx][nz].  One float4 of z per thread.
struct SaveArgs {
    const float* p[5];
    float* W;
    long long n;              // nx * nz
    int nz, nx, its;
    float w0, w1;
};

__global__ void __launch_bounds__(128) k_save_wavefield(SaveArgs a)
{
    const int gz = FAT + 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int gx = FAT + blockIdx.y;
    if (gz >= a.nz - FAT) return;
    const long long gi = (long long)gx * a.nz + gz;
#pragma unroll
    for (int f = 0; f < 5; f++) {
        const float4 v = ld4(a.p[f] + gi);
        float* r0 = a.W + ((long long)a.its * 5 + f) * a.n + gi;
        float* r1 = r0 + 5 * a.n;
        float4 u0 = ld4(r0), u1 = ld4(r1);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            at(u0, j) = fmaf(at(v, j), a.w0, at(u0, j));
            at(u1, j) = fmaf(at(v, j), a.w1, at(u1, j));
        }
        st4(r0, u0);
        st4(r1, u1);
    }
}

// 16-bit source-wavefield checkpoints: one coarse snapshot (vx, vz) from the
// FP32 staging rows into codes with a scale per snapshot and field.  Every CTA
// first reduces the per-(tile, warp) maxima the EPI_TRI step left in pmax
// (npart entries of 2); the scale is max (BF16) or max / 2^15 (FP16, so the
// codes use the normal range), 0 for an all-zero snapshot.  The CTAs also
// clear pmax_next, the slots the next snapshot's step fills.
struct QuantArgs {
    const float* stage[2];        // FP32 snapshot of vx, vz, [nx][nz]
    unsigned short* row[2];       // destination codes, [nx][nz]
    float* scale;                 // 2 floats: this snapshot's vx, vz scale
    const float* pmax;
    float* pmax_next;
    int npart;
    int nz, nx;
};

template <int Q>
__global__ void __launch_bounds__(256) k_quantize(QuantArgs a)
{
    __shared__ float red[2][8];
    const int tid = threadIdx.x;
    float m0 = 0.f, m1 = 0.f;
    for (int i = tid; i < a.npart; i += blockDim.x) {
        m0 = fmaxf(m0, a.pmax[2 * i]);
        m1 = fmaxf(m1, a.pmax[2 * i + 1]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m0 = fmaxf(m0, __shfl_xor_sync(0xffffffffu, m0, o));
        m1 = fmaxf(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    }
    if ((tid & 31) == 0) { red[0][tid >> 5] = m0; red[1][tid >> 5] = m1; }
    __syncthreads();
    float amax[2] = {0.f, 0.f};
#pragma unroll
    for (int w = 0; w < 8; w++) { amax[0] = fmaxf(amax[0], red[0][w]); amax[1] = fmaxf(amax[1], red[1][w]); }
    float sc[2], inv[2];
#pragma unroll
    for (int f = 0; f < 2; f++) {
        sc[f] = (Q == 1) ? amax[f] : amax[f] * (1.0f / 32768.0f);
        inv[f] = sc[f] > 0.f ? 1.0f / sc[f] : 0.f;
    }
    if (blockIdx.x == 0 && tid == 0) { a.scale[0] = sc[0]; a.scale[1] = sc[1]; }
    const long long gtid = (long long)blockIdx.x * blockDim.x + tid;
    const long long gstride = (long long)gridDim.x * blockDim.x;
    for (long long i = gtid; i < 2LL * a.npart; i += gstride) a.pmax_next[i] = 0.f;
    const int nq = (a.nz - 2 * FAT) / 4;
    const long long total = (long long)nq * (a.nx - 2 * FAT);
    for (long long q = gtid; q < total; q += gstride) {
        const long long gi = (long long)(FAT + q / nq) * a.nz + FAT + 4 * (q % nq);
#pragma unroll
        for (int f = 0; f < 2; f++) {
            const float4 v = ld4(a.stage[f] + gi);
            unsigned h[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float x = at(v, j) * inv[f];
                if (Q == 1) h[j] = __bfloat16_as_ushort(__float2bfloat16_rn(x));
                else h[j] = __half_as_ushort(__float2half_rn(x));
            }
            *reinterpret_cast<uint2*>(a.row[f] + gi) = make_uint2(h[0] | (h[1] << 16), h[2] | (h[3] << 16));
        }
    }
}

// Spatial interpolation of receiver traces on the device (spaceInterpGpu
// forward / adjoint, F/src/spaceInterpGpu.cpp:288-361), trace-major [n][nt].
// Forward gathers irreg[d][t] = sum_k w[d,k] * reg[slot[d,k]][t]; the adjoint
// gathers reg[s][t] = sum of w * irreg[d][t] over the (d, k) that use slot s
// (inverse CSR in ascending (d, k)), the order the host loops accumulate in,
// with unfused multiply and add so the sums equal the host's bit for bit.
__global__ void __launch_bounds__(256) k_interp_fwd(const float* reg, float* irreg, const int* slot, const float* w,
                                                    int nIrreg, int nft, int nt)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nIrreg * nt) return;
    const int d = (int)(i / nt), t = (int)(i % nt);
    float acc = 0.f;
    for (int k = 0; k < nft; k++) {
        const int e = d * nft + k;
        acc = __fadd_rn(acc, __fmul_rn(__ldg(w + e), __ldg(reg + (long long)__ldg(slot + e) * nt + t)));
    }
    irreg[i] = acc;
}

__global__ void __launch_bounds__(256) k_interp_adj(const float* irreg, float* reg, const int* start, const int* ent,
                                                    const float* w, int nReg, int nft, int nt)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nReg * nt) return;
    const int s = (int)(i / nt), t = (int)(i % nt);
    float acc = 0.f;
    for (int j = __ldg(start + s); j < __ldg(start + s + 1); j++) {
        const int e = __ldg(ent + j);
        acc = __fadd_rn(acc, __fmul_rn(__ldg(w + e), __ldg(irreg + (long long)(e / nft) * nt + t)));
    }
    reg[i] = acc;
}

// time-major <-> trace-major transposes for the sparse signal matrices
__global__ void k_transpose(const float* __restrict__ in, float* __restrict__ out, int rows, int cols)
{
    __shared__ float tileb[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = by + k, c = bx + threadIdx.x;
        if (r < rows && c < cols) tileb[k][threadIdx.x] = in[(long long)r * cols + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = bx + k, c = by + threadIdx.x;   // out is [cols][rows]
        if (r < cols && c < rows) out[(long long)r * rows + c] = tileb[threadIdx.x][k];
    }
}

}  // namespace eio
