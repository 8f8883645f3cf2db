// bp_tma.cuh -- persistent, TMA-fed voxel-driven backprojection for sm_100a.
//
// Same geometry contract, MIRROR view layout and bounds rule as bp_fast.cuh (circular orbit,
// slab pair, element (u, v) = (P[u][v], P[u][nv-1-v])).  What changes is how views reach
// shared memory and how the gather is indexed:
//
//  * Persistent CTAs walk the (16 x 16 column) x (R slices) tiles, x fastest, so the tiles in
//    flight at any moment sit in the same z band and share detector rows in L2.
//  * Warp 8 is the producer.  For each chunk of NV views of the current tile it computes the
//    detector footprint of the tile's voxels (8 corners; a linear-fractional map takes its
//    extremes there), and one lane issues a 3-D TMA tile load (cp.async.bulk.tensor) of a
//    BW x BH element box per view into a ring of S stages, completing on an mbarrier
//    (expect_tx).  Consumers release a stage through a second mbarrier.  No CTA-wide barrier
//    is on the hot path, and no consumer instruction is spent on staging.
//  * Warps 0-7 consume.  Lanes are an 8 x 4 block of voxel columns: their detector samples
//    fall on about ten box rows at nearly the same v, and a row pitch of 68 words (34 elements
//    of 8 bytes, 4 mod 32) spreads them over the banks (ncu: 10% extra shared wavefronts,
//    against 2.9 wavefronts per gather for 16 x 2 lanes with pitch 24).
//  * FP16 path: v is carried in fixed point, t = (v - v_lo) * 1024 + 1.5 * 2^23, one FFMA per
//    voxel, with the per-view constants of that form folded into the stage metadata by the
//    producer (fold_lerp_meta).  The integer part of t's bits indexes the box; the low 10 bits
//    are the fraction, which as the mantissa of an FP16 subnormal is fv 2^-14 directly.  The
//    v-lerp is one HFMA2 over the (voxel, mirror) pair of the interpolation layout (HalfLerp),
//    the two u-lerps use weights (1-fu) w and fu w folded in, and the result is added to FP32
//    accumulators with the sm_100 mixed-precision add (add.rn.f32.f16).
//
// Every wait is bounded (kWaitLimit polls); a timeout sets the device error word, the CTA
// drains the copies it issued (bounded) and returns.
#pragma once
#include <cuda.h>
#include <cuda_fp16.h>

#include <cstddef>
#include <type_traits>

#include "common.h"
#include "tma_common.cuh"

namespace fdk {

template <typename E>
struct TmaCfg;
// Tile and pipeline shapes (macros for tuning sweeps).  Measured on the 2048^3 / 4096-view
// workload with the first MIXED form of this kernel (FP16 mirror pairs gathered straight from
// 36 x 40 boxes, 8 views per stage; replaced by the interpolation layout below), 128 views per
// launch: mixed R 12 -> 16 and 4 -> 8 views per stage 1985 -> 2215 GUPS (more stages changed
// nothing; R >= 20 spills); FP32 R 8 -> 12: 1007 -> 1051 GUPS.  Unrolling the view loop (1641
// GUPS) and pairing two views per slice with an FP16 pre-add (2115 GUPS) were slower: both raise
// register pressure past the 2-CTA budget.  Three CTAs per SM (72 registers;
// FDK_TMA_MIN_BLOCKS=3) were slower too: R 12 with 4 or 6 views per stage 2003 / 1960 GUPS, R 8
// with 4 views 1830 GUPS -- the per-column setup amortised over fewer slices costs more than the
// extra warps gain.  Again with the current MIXED kernel (folded per-view constants, scaled
// interpolation layout; compact boxes of 4 views, 3 views in the 34 x 40 boxes, so that both
// kernels hold three CTAs per SM): R 12 2648 and R 8 2130 against 3152 GUPS for R 16 at two.  Prefetching a tile's volume runs a few view chunks before its end (a branch
// inside the view loop) instead of at its start measured 11% slower (2168 against 2421 GUPS at
// 512-view batches), though the loop's registers did not change.  A layout with two detector
// columns per 8-byte element (read by 64-bit loads) measured slower than that FP16 gather: 2133
// against 2257 GUPS (its doubled boxes halved the views per stage and the kernel spilled).
#ifndef FDK_TMA_MIXED_R
#define FDK_TMA_MIXED_R 16
#endif
#ifndef FDK_TMA_FP32_R
#define FDK_TMA_FP32_R 12
#endif
#ifndef FDK_TMA_FP32_S
#define FDK_TMA_FP32_S 2
#endif
template <>
struct TmaCfg<float2> {
    static constexpr int R = FDK_TMA_FP32_R;
    static constexpr int BW = 34;  // 272 B rows
    static constexpr int BH = 40;
    static constexpr int NV = 4;
    static constexpr int S = FDK_TMA_FP32_S;
};

// MIXED views in the interpolation layout: element (u, v) holds e = E(v) 2^-k and d = (E(v+1) -
// E(v)) 2^(14-k), E(v) the FP16 mirror pair of the MIRROR layout and 2^k just above the batch's
// largest |E| (d = 0 at v = nv-1, which no sample reads; to_lerp_kernel).  A sample at v = vi + fv
// is then (e + (fv 2^-14) d) 2^k: one HFMA2 whose fv 2^-14 is the FP16 subnormal with the
// fixed-point fraction as its mantissa, and one 8-byte load per detector column; the launch's
// accumulator scale carries the 2^k.  The earlier form a = E(v) - d with 1 + fv from the fraction
// bits under FP16's exponent of 1.0 rounded a, up to 3 |E| on uncorrelated data: on white-noise
// views 1.06e-3 rel-L2 against the reference arithmetic, 8.4e-4 in this form, and 3096 -> 3195
// GUPS at 2048^3 (512-view batches, one B200, both builds twice).
struct __align__(8) HalfLerp {
    __half2 e, d;
};
// Measured on the 2048^3 / 4096-view workload, 512-view batches, conversion included: 2644
// against 2339 GUPS for the FP16 gather it replaced, on one box.  5 views per stage: 2528 against
// 2502 GUPS at 1024^3 (C4), but 1868 against 1961 for the drop-in's 32-view calls, whose last
// stage is then partial; 4 kept.
#ifndef FDK_TMA_LERP_NV
#define FDK_TMA_LERP_NV 4
#endif
#ifndef FDK_TMA_LERP_BW
#define FDK_TMA_LERP_BW 34
#endif
#ifndef FDK_TMA_LERP_BH
#define FDK_TMA_LERP_BH 40
#endif
#ifndef FDK_TMA_LERP_S
#define FDK_TMA_LERP_S 2
#endif
template <>
struct TmaCfg<HalfLerp> {
    static constexpr int R = FDK_TMA_MIXED_R;  // top-slab slices per thread
    static constexpr int BW = FDK_TMA_LERP_BW;  // 34: 272 B rows, 68 words, an 8-row bank period for 8-byte loads
    static constexpr int BH = FDK_TMA_LERP_BH;
    static constexpr int NV = FDK_TMA_LERP_NV;
    static constexpr int S = FDK_TMA_LERP_S;
};
// The same layout read through shorter boxes with more views per stage, for geometries where
// every tile's footprint fits them (chosen on the host: lerp_compact_fits).  On one B200, 5 views
// per stage: 2768 against 2718 GUPS at 2048^3, but 1077 against 2499 at 1024^3 from 1536 x 1024
// views, where half the footprints do not fit and are gathered from global memory.  Views per
// stage at 2048^3 / 512^3: 4 2727 / 2651, 5 2774 / 2696, 6 2792 / 2721 (7 would not leave room
// for two CTAs per SM); with the current kernel at 2048^3, 5 views 3159 against 3171 GUPS for 6.
struct __align__(8) HalfLerpCompact : HalfLerp {};
#ifndef FDK_TMA_COMPACT_NV
#define FDK_TMA_COMPACT_NV 6
#endif
template <>
struct TmaCfg<HalfLerpCompact> {
    static constexpr int R = FDK_TMA_MIXED_R;
    static constexpr int BW = 34;
    static constexpr int BH = 32;
    static constexpr int NV = FDK_TMA_COMPACT_NV;
    static constexpr int S = 2;
};
template <typename E>
constexpr bool is_lerp_v = std::is_same<E, HalfLerp>::value || std::is_same<E, HalfLerpCompact>::value;
// Whether a kernel gathers the views of a tile whose footprint exceeds its box from global
// memory.  The compact-box kernel runs only where the host found that every footprint fits
// (lerp_compact_fits, with slack for rounding), so it has no such path: it skips such a view and
// sets the device error word (kErrFootprint), never silently, and keeps the registers the path
// would take.
template <typename E>
constexpr bool has_global_fallback_v = !std::is_same<E, HalfLerpCompact>::value;

struct __align__(16) TmaMeta {
    float m[12];
    int u_lo, v_lo, staged;
    int interior;  // every detector row v of the tile's voxels lies inside (0, nv-1): no per-slice checks
};
static_assert(sizeof(TmaMeta) == 64 && offsetof(TmaMeta, u_lo) == 48, "load_meta reads TmaMeta as 4 x 16 B");

// In the lerp kernels the producer rewrites m[] for the tile once per view (fold_lerp_meta), so
// a consumer's per-column setup shrinks to the arithmetic that depends on its column:
//   m[0..2]  (m0, m1, m3) s           U = (m[0] x + m[1] y + m[2]) rw
//   m[3..5]  (m8, m9, m11) s          rw = 1 / (m[3] x + m[4] y + m[5]); weight rw^2
//   m[6..8]  (m4, m5, m6 z0 + m7) 1024 s   with z0 the tile's first slice
//   m[9]     m6 1024 s                fixed-point v step per slice: m[9] rw
//   m[10]    1.5 2^23 - 1024 v_lo     fixed point of the first slice: (m[6] x + m[7] y + m[8]) rw + m[10]
//   m[11]    (bits) shared address of the view's box, less u_lo rows and the fixed-point offset
// s = wscale^-1/2 is a power of two (weight_scale), so the scaled rows give U, v and rw^2 wscale
// bit for bit as the unscaled ones give U, v and rw^2 times wscale.  Against the consumer-side
// setup (I2F, FADD and FMULs per column and view for the fixed point, the weight and the box row):
// register spill 16 -> 4 bytes (compact boxes), 2945 -> 3079 GUPS at 2048^3 in 512-view batches,
// both builds measured twice on one B200.

struct BpTmaArgs {
    float *vol;
    float *comp;
    const void *proj;    // MIRROR layout (global gathers of views that do not fit the box)
    const float *mats;   // 12 floats per view (device)
    const float *scale;  // accumulator scale (device scalar) or null
    unsigned int *err;   // device error word
    int n_proj, nu, nv;
    int x0, y0, z0, nxs, nys, nzz;
    long long D;
    float wscale;  // a power of four (weight_scale)
    float wsinv;   // wscale^-1/2, a power of two
    int tiles_x, tiles_y, tiles_z;
    int tz0;  // first z tile of this launch (a launch may cover a band of z tiles)
    unsigned long long wait_ns;  // limit of every mbarrier wait (FDK_BP_WAIT_NS, default 10 s)
    int withhold;  // test switch (FDK_BP_TEST_WITHHOLD): CTA 0 never fills its first stage
    // views taken from a views buffer in any order (device arrays of n_proj entries): the slot of
    // each (the TMA z coordinate) and its view index (its matrix); null: views 0..n_proj-1 in
    // slots 0..n_proj-1
    const int *list_slot;
    const int *list_view;
};

// Host record of one launch's view list, uploaded to a device copy that the kernel reads (a
// list passed by value would make the kernel parameters exceed 4 KB).
constexpr int kMaxListViews = 512;
struct ViewList {
    int n;
    int slot[kMaxListViews];
    int view[kMaxListViews];
};

template <typename E>
__host__ __device__ constexpr int tma_box_bytes() {
    return ((TmaCfg<E>::BW * TmaCfg<E>::BH * (int)sizeof(E)) + 127) / 128 * 128;
}
template <typename E>
__host__ __device__ constexpr int tma_smem_bytes() {
    return TmaCfg<E>::S * TmaCfg<E>::NV * (tma_box_bytes<E>() + (int)sizeof(TmaMeta)) + 2 * TmaCfg<E>::S * 8;
}

__device__ __forceinline__ float2 lds64f(unsigned addr) {
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
    return v;
}
// (An ordinary C++ load through __cvta_shared_to_generic, which the compiler may schedule, measured
// the same: 3131 against 3132 GUPS at 2048^3.)
__device__ __forceinline__ uint2 lds64u(unsigned addr) {
    uint2 v;
    asm volatile("ld.shared.v2.b32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(addr));
    return v;
}
__device__ __forceinline__ __half2 u2h(unsigned u) { return *reinterpret_cast<__half2 *>(&u); }
__device__ __forceinline__ void acc_add_f16x2(float &lo_acc, float &hi_acc, __half2 r) {
    // sm_100 mixed-precision add (measured faster than converting the pair and adding in FP32)
    const unsigned u = *reinterpret_cast<unsigned *>(&r);
    asm("{\n .reg .f16 lo, hi;\n mov.b32 {lo, hi}, %2;\n add.rn.f32.f16 %0, lo, %0;\n add.rn.f32.f16 %1, hi, %1;\n}"
        : "+f"(lo_acc), "+f"(hi_acc)
        : "r"(u));
}

// A view's metadata in registers, read from shared memory with four 128-bit loads (the struct is
// 16-byte aligned: m[0..3], m[4..7], m[8..11], then u_lo, v_lo, staged, interior) instead of up
// to sixteen scalar ones per column and view.
#ifndef FDK_META_SCALAR
#define FDK_META_SCALAR 0
#endif
struct MetaRegs {
    float m[12];
    int u_lo, v_lo, staged, interior;
};
__device__ __forceinline__ MetaRegs load_meta(const TmaMeta &md) {
#if FDK_META_SCALAR  // tuning comparison: field by field
    MetaRegs r;
    for (int i = 0; i < 12; i++) r.m[i] = md.m[i];
    r.u_lo = md.u_lo;
    r.v_lo = md.v_lo;
    r.staged = md.staged;
    r.interior = md.interior;
    return r;
#endif
    const float4 a = *reinterpret_cast<const float4 *>(&md.m[0]);
    const float4 b = *reinterpret_cast<const float4 *>(&md.m[4]);
    const float4 c = *reinterpret_cast<const float4 *>(&md.m[8]);
    const int4 d = *reinterpret_cast<const int4 *>(&md.u_lo);
    return MetaRegs{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w}, d.x, d.y, d.z, d.w};
}

// Footprint box of a tile in one view; fills meta (matrix copied by the caller).
template <typename E>
__device__ __forceinline__ void tile_box(const float *m, float xa, float xb, float ya, float yb, float za, float zb,
                                         int nu, int nv, TmaMeta &md) {
    using C = TmaCfg<E>;
    float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float x = (c & 1) ? xb : xa, y = (c & 2) ? yb : ya;
        const float rw = 1.0f / fmaf(m[8], x, fmaf(m[9], y, m[11]));
        const float U = fmaf(m[0], x, fmaf(m[1], y, m[3])) * rw;
        const float vw = fmaf(m[4], x, fmaf(m[5], y, m[7]));
        const float va = fmaf(m[6], za, vw) * rw, vb = fmaf(m[6], zb, vw) * rw;
        umin = fminf(umin, U);
        umax = fmaxf(umax, U);
        vmin = fminf(vmin, fminf(va, vb));
        vmax = fmaxf(vmax, fmaxf(va, vb));
    }
    // one element of margin absorbs FP32 differences between corners and per-column math
    const float ulo = fmaxf(floorf(umin) - 1.f, -1.f), uhi = fminf(floorf(umax) + 2.f, (float)nu);
    const float vlo = fmaxf(floorf(vmin) - 1.f, -8.f), vhi = fminf(floorf(vmax) + 2.f, (float)nv + 4.f);
    const int u_lo = (int)ulo;
    const int v_lo = ((int)vlo) & ~3;  // 16-byte aligned TMA x coordinate (floor for negatives)
    md.u_lo = u_lo;
    md.v_lo = v_lo;
    md.staged = ((int)uhi - u_lo + 1 <= C::BH && (int)vhi - v_lo + 1 <= C::BW) ? 1 : 0;
    // u needs no tile-level flag: each column checks its own U before its slices
    md.interior = (vmin > 1e-3f && vmax < (float)(nv - 1) - 1e-3f) ? 1 : 0;
}

// The lerp kernels' form of a view's metadata (layout above TmaMeta): m is the view's matrix in
// registers, za the tile's first slice, box the shared address of the view's box, s = wscale^-1/2.
template <typename E>
__device__ __forceinline__ void fold_lerp_meta(const float (&m)[12], float za, unsigned box, float s, TmaMeta &md) {
    constexpr unsigned RB = TmaCfg<E>::BW * 8;  // box row bytes
    const float s10 = s * 1024.f;
    const float f[12] = {m[0] * s,   m[1] * s,   m[3] * s,   m[8] * s,  m[9] * s, m[11] * s, m[4] * s10, m[5] * s10,
                         fmaf(m[6], za, m[7]) * s10, m[6] * s10, 12582912.f - 1024.f * (float)md.v_lo,
                         __uint_as_float(box - (unsigned)md.u_lo * RB - (0x4B400000u >> 10) * 8u)};
#pragma unroll
    for (int q = 0; q < 12; q++) md.m[q] = f[q];
}

// One view's contribution to a thread's column: R voxel pairs.
template <typename E>
__device__ __forceinline__ void column_view(const TmaMeta &md_s, unsigned box, const E *gview, float x, float y,
                                            float zf0, int nu, int nv, float wscale, float (&am)[TmaCfg<E>::R],
                                            float (&ar)[TmaCfg<E>::R]) {
    using C = TmaCfg<E>;
    constexpr int R = C::R;
    const MetaRegs md = load_meta(md_s);
    const float *m = md.m;
    if constexpr (is_lerp_v<E>) {
        // metadata folded by the producer (fold_lerp_meta)
        constexpr unsigned RB = C::BW * 8;  // box row bytes
        const float rw = __fdividef(1.0f, fmaf(m[3], x, fmaf(m[4], y, m[5])));
        const float U = fmaf(m[0], x, fmaf(m[1], y, m[2])) * rw;
        if (!(U >= 0.f && U < (float)(nu - 1))) return;  // every sample of this column is zero
        const float fuf = floorf(U);
        const float fu = U - fuf;
        const int u0 = (int)fuf;
        const float wt = rw * rw;
        const float bwf = fu * wt;
        const __half2 aw = __float2half2_rn(wt - bwf), bw = __float2half2_rn(bwf);
        const float nv1024 = fmaf(m[6], x, fmaf(m[7], y, m[8]));  // 1024 (v at the run's first slice) / rw
        if (md.staged) {
            // fixed point: bits = 0x4B400000 + round(1024 (v - v_lo)); the box row of u0 is m[11] + u0 rows
            const float C0 = fmaf(nv1024, rw, m[10]);
            const float B1 = m[9] * rw;
            const unsigned rowp = __float_as_uint(m[11]) + (unsigned)u0 * RB;
            if (md.interior) {
#pragma unroll
                for (int k = 0; k < R; k++) {
                    const unsigned bits = __float_as_uint(fmaf((float)k, B1, C0));
                    const unsigned a = rowp + (bits >> 10) * 8u;
                    const __half2 g = __low2half2(u2h(bits & 0x3FFu));  // fv 2^-14 (FP16 subnormal)
                    const uint2 p0 = lds64u(a), p1 = lds64u(a + RB);
                    const __half2 l0 = __hfma2(g, u2h(p0.y), u2h(p0.x));
                    const __half2 l1 = __hfma2(g, u2h(p1.y), u2h(p1.x));
                    acc_add_f16x2(am[k], ar[k], __hfma2(l1, bw, __hmul2(l0, aw)));
                }
            } else {
                const float A = nv1024 * rw * (1.0f / 1024.f), B = B1 * (1.0f / 1024.f);  // v in pixels
#pragma unroll
                for (int k = 0; k < R; k++) {
                    const float v = fmaf(B, (float)k, A);
                    const float vr = (float)(nv - 1) - v;
                    const bool mv = v >= 0.f && v < (float)(nv - 1);
                    const bool rv = vr >= 0.f && vr < (float)(nv - 1);
                    if (!(mv || rv)) continue;
                    const unsigned bits = __float_as_uint(fmaf((float)k, B1, C0));
                    const unsigned a = rowp + (bits >> 10) * 8u;
                    const __half2 g = __low2half2(u2h(bits & 0x3FFu));
                    const uint2 p0 = lds64u(a), p1 = lds64u(a + RB);
                    const __half2 l0 = __hfma2(g, u2h(p0.y), u2h(p0.x));
                    const __half2 l1 = __hfma2(g, u2h(p1.y), u2h(p1.x));
                    const float2 rf = __half22float2(__hfma2(l1, bw, __hmul2(l0, aw)));
                    if (mv) am[k] += rf.x;
                    if (rv) ar[k] += rf.y;
                }
            }
            return;
        }
        if constexpr (!has_global_fallback_v<E>) return;  // reported by the producer
        // a tile whose footprint does not fit the box: the column's two detector rows from global
        // memory (row pointer formed once; rare, and kept lean so the hot loops above keep their
        // registers)
        const float A = nv1024 * rw * (1.0f / 1024.f), B = m[9] * rw * (1.0f / 1024.f);
        const uint2 *grow = reinterpret_cast<const uint2 *>(gview) + (long long)u0 * nv;
#pragma unroll
        for (int k = 0; k < R; k++) {
            const float v = fmaf(B, (float)k, A);
            const float vr = (float)(nv - 1) - v;
            const bool mv = v >= 0.f && v < (float)(nv - 1);
            const bool rv = vr >= 0.f && vr < (float)(nv - 1);
            if (!(mv || rv)) continue;
            const float vf = fminf(floorf(v), (float)(nv - 2));
            const __half2 g = __float2half2_rn((v - vf) * 6.103515625e-05f);  // fv 2^-14
            const int vi = (int)vf;
            const uint2 p0 = __ldg(grow + vi), p1 = __ldg(grow + nv + vi);
            const __half2 l0 = __hfma2(g, u2h(p0.y), u2h(p0.x));
            const __half2 l1 = __hfma2(g, u2h(p1.y), u2h(p1.x));
            const float2 rf = __half22float2(__hfma2(l1, bw, __hmul2(l0, aw)));
            if (mv) am[k] += rf.x;
            if (rv) ar[k] += rf.y;
        }
        return;
    }
    const float w = fmaf(m[8], x, fmaf(m[9], y, m[11]));
    const float rw = __fdividef(1.0f, w);
    const float U = fmaf(m[0], x, fmaf(m[1], y, m[3])) * rw;
    const float A = fmaf(m[4], x, fmaf(m[5], y, fmaf(m[6], zf0, m[7]))) * rw;  // v at the run's first slice
    const float B = m[6] * rw;                                                  // dv per slice
    const float wt = rw * rw * wscale;
    if (!(U >= 0.f && U < (float)(nu - 1))) return;  // every sample of this column is zero
    const float fuf = floorf(U);
    const float fu = U - fuf;
    const int u0 = (int)fuf;
    const float wa = (1.f - fu) * wt, wb = fu * wt;
#pragma unroll
    for (int k = 0; k < R; k++) {
        const float v = fmaf(B, (float)k, A);
        bool mv = true, rv = true;
        float vf;
        if (!(md.staged && md.interior)) {
            const float vr = (float)(nv - 1) - v;
            mv = v >= 0.f && v < (float)(nv - 1);
            rv = vr >= 0.f && vr < (float)(nv - 1);
            if (!(mv || rv)) continue;
            vf = fminf(floorf(v), (float)(nv - 2));
        } else {
            vf = floorf(v);
        }
        const int vi = (int)vf;
        const float fv = v - vf;
        float2 e0, e1, e2, e3;
        if (md.staged) {
            const unsigned a = box + (unsigned)(((u0 - md.u_lo) * C::BW + (vi - md.v_lo)) * 8);
            e0 = lds64f(a);
            e1 = lds64f(a + 8);
            e2 = lds64f(a + C::BW * 8);
            e3 = lds64f(a + C::BW * 8 + 8);
        } else {
            const float2 *g0 = reinterpret_cast<const float2 *>(gview) + (long long)u0 * nv + vi;
            e0 = __ldg(g0);
            e1 = __ldg(g0 + 1);
            e2 = __ldg(g0 + nv);
            e3 = __ldg(g0 + nv + 1);
        }
        const float c0x = fmaf(e2.x, wb, e0.x * wa), c0y = fmaf(e2.y, wb, e0.y * wa);
        const float c1x = fmaf(e3.x, wb, e1.x * wa), c1y = fmaf(e3.y, wb, e1.y * wa);
        if (mv) am[k] += fmaf(fv, c1x - c0x, c0x);
        if (rv) ar[k] += fmaf(fv, c1y - c0y, c0y);
    }
}

__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Prefetch a thread's two volume segments (top run and mirror run, and their compensation
// terms) into L2 at the start of a tile, so the write-back at its end does not wait on DRAM.
template <int R>
__device__ __forceinline__ void prefetch_column(const float *vol, const float *comp, long long base, long long D,
                                                int zt) {
    const long long t0 = base + zt, b0 = base + D - zt - R;
    prefetch_l2(vol + t0);
    prefetch_l2(vol + t0 + R - 1);
    prefetch_l2(vol + b0);
    prefetch_l2(vol + b0 + R - 1);
    if (comp) {
        prefetch_l2(comp + t0);
        prefetch_l2(comp + t0 + R - 1);
        prefetch_l2(comp + b0);
        prefetch_l2(comp + b0 + R - 1);
    }
}

// Add a thread's accumulators to its column: top slices zt..zt+nrun-1 and their mirrors
// D-1-zt-k.  Loads are issued before any store (restrict pointers), as 128-bit accesses when
// the runs are 16-byte aligned; with comp, a compensated (Kahan) sum across launches.
template <int R>
__device__ __forceinline__ void write_back(float *__restrict__ vol, float *__restrict__ comp, long long base,
                                           long long D, int zt, int nrun, float sc, const float (&am)[R],
                                           const float (&ar)[R]) {
    float *vt = vol + base + zt;           // top run, ascending in k
    float *vb = vol + base + D - zt - R;   // mirror run: element j holds k = R-1-j
    float *ct = comp ? comp + base + zt : nullptr;
    float *cb = comp ? comp + base + D - zt - R : nullptr;
    if (nrun == R && (R % 4) == 0 && (D % 4) == 0 && (zt % 4) == 0 && ((base & 3) == 0)) {
        // top run, then mirror run (keeps at most 2R extra values live)
#pragma unroll
        for (int half = 0; half < 2; half++) {
            float *v = half ? vb : vt;
            float *c = half ? cb : ct;
            float t[R], tc[R];
#pragma unroll
            for (int q = 0; q < R / 4; q++) {
                *reinterpret_cast<float4 *>(&t[4 * q]) = reinterpret_cast<const float4 *>(v)[q];
                if (comp) *reinterpret_cast<float4 *>(&tc[4 * q]) = reinterpret_cast<const float4 *>(c)[q];
            }
#pragma unroll
            for (int k = 0; k < R; k++) {
                const float d = (half ? ar[R - 1 - k] : am[k]) * sc;  // mirror element k is voxel R-1-k
                if (comp) {
                    const float y = d - tc[k], s = t[k] + y;
                    tc[k] = (s - t[k]) - y;
                    t[k] = s;
                } else {
                    t[k] += d;
                }
            }
#pragma unroll
            for (int q = 0; q < R / 4; q++) {
                reinterpret_cast<float4 *>(v)[q] = *reinterpret_cast<const float4 *>(&t[4 * q]);
                if (comp) reinterpret_cast<float4 *>(c)[q] = *reinterpret_cast<const float4 *>(&tc[4 * q]);
            }
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < R; k++) {  // static indices keep the accumulators in registers
        if (k >= nrun) break;
        const long long i1 = base + zt + k, i2 = base + D - 1 - zt - k;
        const float dm = am[k] * sc, dr = ar[k] * sc;
        if (comp) {
            const float o1 = vol[i1], c1 = comp[i1], o2 = vol[i2], c2 = comp[i2];
            const float y1 = dm - c1, s1 = o1 + y1;
            const float y2 = dr - c2, s2 = o2 + y2;
            comp[i1] = (s1 - o1) - y1;
            vol[i1] = s1;
            comp[i2] = (s2 - o2) - y2;
            vol[i2] = s2;
        } else {
            vol[i1] += dm;
            vol[i2] += dr;
        }
    }
}

template <typename E>
#ifndef FDK_TMA_MIN_BLOCKS
#define FDK_TMA_MIN_BLOCKS 2
#endif
__global__ void __launch_bounds__(288, FDK_TMA_MIN_BLOCKS)
    bp_tma_kernel(const __grid_constant__ CUtensorMap tmap, BpTmaArgs a) {
    using C = TmaCfg<E>;
    constexpr int R = C::R, NV = C::NV, S = C::S;
    constexpr int BOX = tma_box_bytes<E>();
    constexpr unsigned BOX_TX = C::BW * C::BH * sizeof(E);
    extern __shared__ __align__(128) unsigned char smem[];
    TmaMeta *meta = reinterpret_cast<TmaMeta *>(smem + S * NV * BOX);
    uint64_t *bars = reinterpret_cast<uint64_t *>(meta + S * NV);
    const unsigned boxes = smem_u32(smem);
    const unsigned full0 = smem_u32(bars), empty0 = smem_u32(bars + S);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 8);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int n_chunks = (a.n_proj + NV - 1) / NV;
    const int n_tiles = a.tiles_x * a.tiles_y * a.tiles_z;
    const long long frame = (long long)a.nu * a.nv;

    if (warp == 8) {
        // ---------------- producer
        int it = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
            const int tx = tile % a.tiles_x, ty = (tile / a.tiles_x) % a.tiles_y;
            const int tz = a.tz0 + tile / (a.tiles_x * a.tiles_y);
            const float xa = (float)(a.x0 + tx * 16), xb = (float)(a.x0 + min(tx * 16 + 16, a.nxs) - 1);
            const float ya = (float)(a.y0 + ty * 16), yb = (float)(a.y0 + min(ty * 16 + 16, a.nys) - 1);
            const float za = (float)(a.z0 + tz * R), zb = za + (float)(R - 1);
            for (int c = 0; c < n_chunks; c++, it++) {
                const int s = it % S;
                const unsigned ph = (unsigned)(it / S) & 1u;
                if (it >= S && !mbar_wait_backoff(empty0 + 8 * s, ph ^ 1u, a.wait_ns, FDK_PRODUCER_SLEEP_NS)) {
                    ok = false;
                    break;
                }
                if (a.withhold && blockIdx.x == 0 && it == 0) continue;  // the consumers' wait runs out
                const int view = c * NV + lane;
                if (lane < NV) {
                    TmaMeta &md = meta[s * NV + lane];
                    if (view < a.n_proj) {
                        const float *mg = a.mats + 12 * (long long)(a.list_view ? __ldg(a.list_view + view) : view);
                        float mr[12];
#pragma unroll
                        for (int q = 0; q < 12; q++) mr[q] = __ldg(mg + q);
                        tile_box<E>(mr, xa, xb, ya, yb, za, zb, a.nu, a.nv, md);
                        if constexpr (is_lerp_v<E>) {
                            fold_lerp_meta<E>(mr, za, boxes + (s * NV + lane) * BOX, a.wsinv, md);
                        } else {
#pragma unroll
                            for (int q = 0; q < 12; q++) md.m[q] = mr[q];
                        }
                    } else {
                        md.staged = 0;
                        md.interior = 0;
                    }
                }
                __syncwarp();
                if (lane == 0) {
                    unsigned n_staged = 0, n_views = 0;
                    for (int l = 0; l < NV; l++)
                        if (c * NV + l < a.n_proj) {
                            n_views++;
                            if (meta[s * NV + l].staged) n_staged++;
                        }
                    if (!has_global_fallback_v<E> && n_staged != n_views) atomicOr(a.err, kErrFootprint);
                    mbar_arrive_tx(full0 + 8 * s, n_staged * BOX_TX);
                    for (int l = 0; l < NV; l++) {
                        const TmaMeta &md = meta[s * NV + l];
                        if (c * NV + l < a.n_proj && md.staged)
                            tma_load_3d(boxes + (s * NV + l) * BOX, &tmap, md.v_lo, md.u_lo,
                                        a.list_slot ? __ldg(a.list_slot + c * NV + l) : c * NV + l, full0 + 8 * s);
                    }
                }
                __syncwarp();
            }
        }
        if (!ok && lane == 0) atomicOr(a.err, kErrTimeout);
        // drain (always): wait, bounded, for the copies of the last stages to land before the CTA
        // may exit -- consumers that gave up on a wait have left already.  Immediate when the
        // consumers have waited for these stages themselves.
        if (lane == 0)
            for (int k = (it > S ? it - S : 0); k < it; k++)
                mbar_wait(full0 + 8 * (k % S), (unsigned)(k / S) & 1u, a.wait_ns);
        return;
    }

    // ---------------- consumers: warps 0..7, lanes = 8 x 4 columns
    const int wx = warp & 1, wy = warp >> 1;
    const int lx = lane & 7, ly = lane >> 3;
    const E *proj = reinterpret_cast<const E *>(a.proj);
    int it = 0;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int tx = tile % a.tiles_x, ty = (tile / a.tiles_x) % a.tiles_y;
        const int tz = a.tz0 + tile / (a.tiles_x * a.tiles_y);
        const int xi = tx * 16 + wx * 8 + lx, yi = ty * 16 + wy * 4 + ly;
        const bool col_ok = xi < a.nxs && yi < a.nys;
        const float x = (float)(a.x0 + xi), y = (float)(a.y0 + yi);
        const int zt = tz * R;
        const float zf0 = (float)(a.z0 + zt);
        if (col_ok) prefetch_column<R>(a.vol, a.comp, ((long long)xi * a.nys + yi) * a.D, a.D, zt);
        float am[R], ar[R];
#pragma unroll
        for (int k = 0; k < R; k++) am[k] = ar[k] = 0.f;
        for (int c = 0; c < n_chunks; c++, it++) {
            const int s = it % S;
            const unsigned ph = (unsigned)(it / S) & 1u;
            if (!mbar_wait(full0 + 8 * s, ph, a.wait_ns)) {
                if (lane == 0) atomicOr(a.err, kErrTimeout);
                return;
            }
            if (col_ok) {
                for (int l = 0; l < NV; l++) {
                    const int view = c * NV + l;
                    if (view >= a.n_proj) break;
                    const long long slot = a.list_slot ? __ldg(a.list_slot + view) : view;
                    column_view<E>(meta[s * NV + l], boxes + (s * NV + l) * BOX, proj + slot * frame, x, y, zf0, a.nu,
                                   a.nv, a.wscale, am, ar);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty0 + 8 * s);
        }
        if (col_ok) {
            const float sc = (a.scale ? *a.scale : 1.0f) / a.wscale;
            write_back<R>(a.vol, a.comp, ((long long)xi * a.nys + yi) * a.D, a.D, zt, min(R, a.nzz - zt), sc, am,
                          ar);
        }
    }
}

}  // namespace fdk

// ---------------------------------------------------------------------------------------
// host side
namespace fdk {

// 3-D map over MIRROR views [n][nu][nv] of esz-byte elements, box BW x BH x 1, zero fill.
template <typename E>
inline int encode_views_map(CUtensorMap *map, const void *base, int nu, int nv, int n) {
    EncodeTiledFn enc = tensor_map_encoder();
    if (!enc) return fail(FDK_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t dims[3] = {(cuuint64_t)nv, (cuuint64_t)nu, (cuuint64_t)n};
    const cuuint64_t strides[2] = {(cuuint64_t)nv * sizeof(E), (cuuint64_t)nu * nv * sizeof(E)};
    const cuuint32_t box[3] = {(cuuint32_t)TmaCfg<E>::BW, (cuuint32_t)TmaCfg<E>::BH, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapDataType dt = sizeof(E) == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    CUresult r = enc(map, dt, 3, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(FDK_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return FDK_OK;
}

template <typename E>
inline int tma_prepare(int &ctas, int device) {
    const int smem = tma_smem_bytes<E>();
    FDK_CUDA(cudaFuncSetAttribute(bp_tma_kernel<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0, sms = 0;
    FDK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_tma_kernel<E>, 288, smem));
    FDK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    ctas = sms * (per_sm > 0 ? per_sm : 1);
    return FDK_OK;
}

// Limit of the kernel's mbarrier waits: FDK_BP_WAIT_NS nanoseconds, default 10 s.
inline unsigned long long bp_wait_ns() {
    const char *e = getenv("FDK_BP_WAIT_NS");
    const long long v = e ? atoll(e) : 0;
    return v > 0 ? (unsigned long long)v : kWaitNs;
}
// Test switch FDK_BP_TEST_WITHHOLD=1: CTA 0's producer never fills the first pipeline stage,
// so its consumers' bounded wait runs out and the launch reports FDK_ERR_DEVICE_CHECK (the
// timeout path, exercised without a GPU fault).  Off unless the environment sets it.
inline int bp_test_withhold() {
    const char *e = getenv("FDK_BP_TEST_WITHHOLD");
    return (e && atoi(e) == 1) ? 1 : 0;
}

// Square of the source distance of the volume centre in view 0, rounded to a power of four
// (within a factor of two of it): keeps f^2 * wscale near 1, and its square root is a power of
// two, so scaling by it is exact (fold_lerp_meta folds wscale^-1/2 into the matrix rows).
inline float weight_scale(const float *host_mats, float xc, float yc) {
    const float w = host_mats[8] * xc + host_mats[9] * yc + host_mats[11];
    if (!(w > 0.f)) return 1.0f;
    return ldexpf(1.0f, 2 * (int)lrintf(log2f(w)));
}

// Backproject n views into the z tiles [tz_begin, tz_end) of R top slices each (with their
// mirror slices); tz_end < 0 means through the last tile.
// list (optional): the n views as slots of a buffer of n_slots views and their view indices
// (matrices d_mats + 12 * view), checked here; d_list: its device copy, which the kernel reads
// (uploaded on st before this launch).  Without a list, views and slots 0..n-1.
template <typename E>
inline int bp_tma_launch(const BpFastPlan &p, float *vol, float *comp, const void *proj, const float *d_mats,
                         const float *host_mats, int n, cudaStream_t st, const float *scale, int tz_begin = 0,
                         int tz_end = -1, const ViewList *list = nullptr, const ViewList *d_list = nullptr,
                         int n_slots = 0) {
    using C = TmaCfg<E>;
    FDK_CHECK_ARG(((uintptr_t)proj & 15) == 0, "TMA views must start on a 16-byte boundary");
    FDK_CHECK_ARG(!list == !d_list, "a view list needs its device copy");
    if (list) {
        FDK_CHECK_ARG(list->n == n && n <= kMaxListViews, "view list of %d entries for %d views", list->n, n);
        for (int i = 0; i < n; i++)
            FDK_CHECK_ARG(list->slot[i] >= 0 && list->slot[i] < n_slots, "list entry %d: slot outside the buffer", i);
    }
    CUtensorMap map;
    FDK_TRY(encode_views_map<E>(&map, proj, p.nu, p.nv, list ? n_slots : n));
    BpTmaArgs a;
    a.vol = vol;
    a.comp = comp;
    a.proj = proj;
    a.mats = d_mats;
    a.scale = scale;
    a.err = p.d_err;
    a.n_proj = n;
    a.nu = p.nu;
    a.nv = p.nv;
    a.x0 = p.x0;
    a.y0 = p.y0;
    a.z0 = p.z0;
    a.nxs = p.nxs;
    a.nys = p.nys;
    a.nzz = p.nzz;
    a.D = p.D;
    a.wscale = weight_scale(host_mats + (list ? 12 * (long long)list->view[0] : 0), p.x0 + 0.5f * (p.nxs - 1),
                            p.y0 + 0.5f * (p.nys - 1));
    a.wsinv = ldexpf(1.0f, -ilogbf(a.wscale) / 2);  // exact: wscale is a power of four
    a.tiles_x = (int)ceil_div(p.nxs, 16);
    a.tiles_y = (int)ceil_div(p.nys, 16);
    const int tz_all = (int)ceil_div(p.nzz, C::R);
    if (tz_end < 0 || tz_end > tz_all) tz_end = tz_all;
    FDK_CHECK_ARG(tz_begin >= 0 && tz_begin < tz_end, "z tiles [%d, %d) outside 0..%d", tz_begin, tz_end, tz_all);
    a.tz0 = tz_begin;
    a.tiles_z = tz_end - tz_begin;
    a.wait_ns = bp_wait_ns();
    a.withhold = bp_test_withhold();
    // addresses inside the device copy (no host access to it)
    const char *dl = reinterpret_cast<const char *>(d_list);
    a.list_slot = d_list ? reinterpret_cast<const int *>(dl + offsetof(ViewList, slot)) : nullptr;
    a.list_view = d_list ? reinterpret_cast<const int *>(dl + offsetof(ViewList, view)) : nullptr;
    const long long n_tiles = (long long)a.tiles_x * a.tiles_y * a.tiles_z;
    FDK_CHECK_ARG(n_tiles < (1ll << 31), "too many tiles");
    const int grid = (int)std::min<long long>(n_tiles, p.tma_ctas);
    bp_tma_kernel<E><<<grid, 288, tma_smem_bytes<E>(), st>>>(map, a);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
}

}  // namespace fdk
