// bp_sym.cuh -- backprojection of view quadruples related by the circular orbit's quarter-turn
// symmetry, for sm_100a.
//
// For a circular orbit of N views (N % 4 == 0) about the axis of a square, centred voxel grid,
// view b + jN/4 sees column T^j(x, y) exactly where view b sees column (x, y): T is a quarter
// turn of the grid, T(x, y) = (y, n-1-x) or (n-1-y, x) according to the orbit's direction (the
// host checks which one the matrices follow, and that they do).  So one detector position, one
// set of bilinear weights and one shared-memory address -- those of base view b at base column
// c -- serve four (column, view) pairs, (T^j(c), b + jN/4), and through the MIRROR element pairs
// (rows v and nv-1-v) also the mirror voxel nz-1-z of each: eight voxel updates per index
// computation instead of two.  With every view of an orbit once as the base, every view reaches
// every column of the grid.  This is the reference's own mirror
// shortcut (backprojectionFDK.cu:90-126) extended by the orbit's in-plane symmetry.
//
//  * Persistent CTAs walk tiles of one quadrant of the grid (16 x 16 base columns x R top-slab
//    slices); each consumer thread owns a base column and the three columns the quarter turns
//    map it to, 2 x 4 x R FP32 accumulators (top and mirror slices of the four columns).
//  * Warp 8 is the producer: per quadruple it computes the base view's footprint box of the
//    tile (8 corners) and issues four plain 3-D TMA tile loads of that box into its own CTA, one from
//    each member view's slot in the views buffer, into a ring of S stages completed by
//    mbarrier expect_tx; consumers release a stage through a second mbarrier.
//  * MIXED reads the views in the interpolation layout (HalfLerp, bp_tma.cuh): v in fixed point
//    (t = (v - v_lo) * 1024 + 1.5 * 2^23, one FFMA per slice gives the box index and fv 2^-14),
//    and per member two 8-byte loads and e + (fv 2^-14) d per detector column, then the u-lerp;
//    the FP16 pair is added to the FP32 accumulators by the sm_100 mixed-precision add.
//  * FP32: FP32 mirror pairs, the four bilinear weights formed once per slice, FFMA.
//  * The host admits a launch only when every tile's footprint fits the box in every base view
//    (sym_footprints_fit); a quadruple whose box would not fit is skipped and reported through
//    the device error word (kErrFootprint) rather than gathered from global memory, which would
//    cost the whole kernel registers.
//  * Every wait is bounded (a.wait_ns); a timeout sets the device error word; the producer
//    always drains its last stages before the CTA exits.
#pragma once
#include <cuda.h>
#include <cuda_fp16.h>

#include <type_traits>

#include "bp_tma.cuh"

namespace fdk {

#ifndef FDK_SYM_MIXED_R
#define FDK_SYM_MIXED_R 6
#endif
#ifndef FDK_SYM_FP32_R
#define FDK_SYM_FP32_R 6
#endif
#ifndef FDK_SYM_FP32_BW
#define FDK_SYM_FP32_BW 26
#endif
#ifndef FDK_SYM_FP32_BH
#define FDK_SYM_FP32_BH 32
#endif
#ifndef FDK_SYM_FP32_NQ
#define FDK_SYM_FP32_NQ 2
#endif
#ifndef FDK_SYM_FP32_S
#define FDK_SYM_FP32_S 2
#endif

// Tile and pipeline shapes (macros for tuning sweeps), measured on one B200 (GUPS of the kernel,
// 512-view batches in the bench's quarter read order; staged = bp_tma_kernel on the same views):
//   FP32:  C2 1227 staged -> 1777 (R 6, 34 x 40 boxes, 1 quad x 2 stages) -> 1908 (18 x 32 boxes,
//          2 quads x 3 stages); C3 1257 staged -> 1749.  R 4 at 64 registers (3 CTAs per SM):
//          1895 at C2 but 1426 at C3 (short volume runs).
//   MIXED, FP16 mirror pairs (this kernel's first MIXED form, since removed): C2 2320 staged
//          against 2090-2229 for every shape tried (R 4-6, 20-28 x 32-40 boxes, 2-4 quads, 2-4
//          stages, 2 or 3 CTAs per SM, FP16 or mixed-FMA interpolation); C3 2358 staged against
//          2084 -- near 57% of its shared-memory wavefront bound, issue 39%, latency-bound at 4
//          consumer warps per scheduler and 96 registers.
//   MIXED, interpolation layout (the FP32 shape): C2 2649 staged -> 2150, C3 2719 -> 1887.
//   The reconstructor therefore pairs views for FP32 only unless FDK_BP_SYM=1.
// At 112 registers (one CTA per SM: 9 warps) both ran at 1440-1630.
template <typename E>
struct SymCfg;
template <>
struct SymCfg<float2> {
    static constexpr int R = FDK_SYM_FP32_R;
    // 2 BW words a row: 52 words (= 20 mod 32) repeats every 8 rows, as 36 (= 4); 26 elements
    // also leave room for the volume's top and bottom tiles (footprint check)
    static constexpr int BW = FDK_SYM_FP32_BW;
    static constexpr int BH = FDK_SYM_FP32_BH;
    static constexpr int NQ = FDK_SYM_FP32_NQ;
    static constexpr int S = FDK_SYM_FP32_S;
};
// MIXED views in the interpolation layout (HalfLerp, 8-byte elements): the FP32 kernel's box and
// stage shape (the same element size); R = 6 keeps the 4 x 2 x R accumulators in 96 registers.
#ifndef FDK_SYM_LERP_NQ
#define FDK_SYM_LERP_NQ 2
#endif
template <>
struct SymCfg<HalfLerp> {
    static constexpr int R = FDK_SYM_MIXED_R;
    static constexpr int BW = FDK_SYM_FP32_BW;
    static constexpr int BH = FDK_SYM_FP32_BH;
    static constexpr int NQ = FDK_SYM_LERP_NQ;
    static constexpr int S = FDK_SYM_FP32_S;
};

constexpr int kSymMaxQuads = 512;

// Quadruples of one launch (a host record, uploaded to a device copy that the kernel reads): the slots (views-buffer index, the TMA z
// coordinate) of the four members b, b + N/4, b + N/2, b + 3N/4 (mod N), and the base view b
// whose matrix the four share.  A batch with whole orbits lists each view once as the base, so
// every view reaches every column: base columns c through itself, T^j(c) through the quadruple
// based j quarters earlier.
struct SymQuads {
    int4 slot[kSymMaxQuads];
    int view[kSymMaxQuads];
};

struct BpSymArgs {
    float *vol;
    float *comp;
    const void *proj;    // MIRROR layout views buffer
    const float *mats;   // 12 floats per view (device), indexed by view
    const float *scale;  // accumulator scale (device scalar) or null
    unsigned int *err;   // device error word
    int n_quads, nu, nv;
    int n;               // nx == ny: the grid's side
    int z0, nzz;
    long long D;
    float wscale;
    int tiles_q;         // tiles per side of the quadrant (ceil(n/2 / 16))
    int tiles_z, tz0;    // z tiles of this launch
    int rot;             // quarter turn: > 0 T(x, y) = (y, n-1-x), < 0 T(x, y) = (n-1-y, x)
    unsigned long long wait_ns;
    int withhold;        // test switch (FDK_BP_TEST_WITHHOLD): CTA 0 never fills its first stage
    const int4 *q_slot;  // device copy of the launch's quadruples: n_quads slots and base views
    const int *q_view;
};

// Volume offset ([x][y][zs]) of column T^j(x, y), T the launch's quarter turn.
__device__ __forceinline__ long long sym_column_base(int x, int y, int j, const BpSymArgs &a) {
    const int nm1 = a.n - 1;
#pragma unroll
    for (int t = 0; t < j; t++) {
        const int nx_ = a.rot > 0 ? y : nm1 - y, ny_ = a.rot > 0 ? nm1 - x : x;
        x = nx_;
        y = ny_;
    }
    return ((long long)x * a.n + y) * a.D;
}

template <typename E>
__host__ __device__ constexpr int sym_box_bytes() {
    return ((SymCfg<E>::BW * SymCfg<E>::BH * (int)sizeof(E)) + 127) / 128 * 128;
}
template <typename E>
__host__ __device__ constexpr int sym_smem_bytes() {
    return SymCfg<E>::S * SymCfg<E>::NQ * (4 * sym_box_bytes<E>() + (int)sizeof(TmaMeta)) + 2 * SymCfg<E>::S * 8;
}

// Footprint box of a tile of base columns in the base view (as tile_box, with this kernel's box).
template <typename E>
__device__ __forceinline__ void sym_tile_box(const float *m, float xa, float xb, float ya, float yb, float za,
                                             float zb, int nu, int nv, TmaMeta &md) {
    using C = SymCfg<E>;
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
    const float ulo = fmaxf(floorf(umin) - 1.f, -1.f), uhi = fminf(floorf(umax) + 2.f, (float)nu);
    const float vlo = fmaxf(floorf(vmin) - 1.f, -8.f), vhi = fminf(floorf(vmax) + 2.f, (float)nv + 4.f);
    const int u_lo = (int)ulo;
    const int v_lo = ((int)vlo) & ~3;  // 16-byte aligned TMA x coordinate (floor for negatives)
    md.u_lo = u_lo;
    md.v_lo = v_lo;
    md.staged = ((int)uhi - u_lo + 1 <= C::BH && (int)vhi - v_lo + 1 <= C::BW) ? 1 : 0;
    md.interior = (vmin > 1e-3f && vmax < (float)(nv - 1) - 1e-3f) ? 1 : 0;
}

// One quadruple's contribution to a thread's four columns: 4 x R voxel pairs.  box: the four
// member boxes (staged footprints), BOX bytes apart.
template <typename E>
__device__ __forceinline__ void column_quad(const TmaMeta &md, unsigned box, float x, float y, float zf0, int nu,
                                            int nv, float wscale, float (&am)[4][SymCfg<E>::R],
                                            float (&ar)[4][SymCfg<E>::R]) {
    using C = SymCfg<E>;
    constexpr int R = C::R;
    constexpr unsigned BOX = sym_box_bytes<E>();
    const MetaRegs mr = load_meta(md);  // md lives in shared memory: four 128-bit loads
    const float *m = mr.m;
    const bool interior = mr.interior;
    const int u_lo = mr.u_lo, v_lo = mr.v_lo;
    const float w = fmaf(m[8], x, fmaf(m[9], y, m[11]));
    const float rw = __fdividef(1.0f, w);
    const float U = fmaf(m[0], x, fmaf(m[1], y, m[3])) * rw;
    const float A = fmaf(m[4], x, fmaf(m[5], y, fmaf(m[6], zf0, m[7]))) * rw;  // v at the run's first slice
    const float B = m[6] * rw;                                                  // dv per slice
    const float wt = rw * rw * wscale;
    if (!(U >= 0.f && U < (float)(nu - 1))) return;  // every sample of these columns is zero
    const float fuf = floorf(U);
    const float fu = U - fuf;
    const int u0 = (int)fuf;

    if constexpr (std::is_same<E, HalfLerp>::value) {
        // one address, fraction and u-weight set per slice serves the four members: per member
        // two 8-byte loads (the sample's two detector columns) and e + (fv 2^-14) d per column
        constexpr unsigned RB = C::BW * 8;
        const __half2 aw = __float2half2_rn((1.f - fu) * wt), bw = __float2half2_rn(fu * wt);
        const float C0 = fmaf(A - (float)v_lo, 1024.f, 12582912.f);
        const float B1 = B * 1024.f;
        const unsigned rowp = box + (unsigned)(u0 - u_lo) * RB - (0x4B400000u >> 10) * 8u;
#pragma unroll
        for (int k = 0; k < R; k++) {
            bool mv = true, rv = true;
            if (!interior) {
                const float v = fmaf(B, (float)k, A);
                const float vr = (float)(nv - 1) - v;
                mv = v >= 0.f && v < (float)(nv - 1);
                rv = vr >= 0.f && vr < (float)(nv - 1);
                if (!(mv || rv)) continue;
            }
            const unsigned bits = __float_as_uint(fmaf((float)k, B1, C0));
            const unsigned a = rowp + (bits >> 10) * 8u;
            const __half2 g = __low2half2(u2h(bits & 0x3FFu));  // fv 2^-14 (FP16 subnormal)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint2 p0 = lds64u(a + j * BOX), p1 = lds64u(a + j * BOX + RB);
                const __half2 l0 = __hfma2(g, u2h(p0.y), u2h(p0.x));
                const __half2 l1 = __hfma2(g, u2h(p1.y), u2h(p1.x));
                const __half2 r = __hfma2(l1, bw, __hmul2(l0, aw));
                if (interior) {
                    acc_add_f16x2(am[j][k], ar[j][k], r);
                } else {
                    const float2 rf = __half22float2(r);
                    if (mv) am[j][k] += rf.x;
                    if (rv) ar[j][k] += rf.y;
                }
            }
        }
    } else {
        const float wa = (1.f - fu) * wt, wb = fu * wt;
        constexpr unsigned RB = C::BW * 8;
#pragma unroll
        for (int k = 0; k < R; k++) {
            const float v = fmaf(B, (float)k, A);
            bool mv = true, rv = true;
            float vf;
            if (!interior) {
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
            const float w1 = wa * fv, w3 = wb * fv;
            const float w0 = wa - w1, w2 = wb - w3;
            const unsigned a = box + (unsigned)(((u0 - u_lo) * C::BW + (vi - v_lo)) * 8);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float2 e0 = lds64f(a + j * BOX), e1 = lds64f(a + j * BOX + 8);
                const float2 e2 = lds64f(a + j * BOX + RB), e3 = lds64f(a + j * BOX + RB + 8);
                const float sm = fmaf(e3.x, w3, fmaf(e2.x, w2, fmaf(e1.x, w1, e0.x * w0)));
                const float sr = fmaf(e3.y, w3, fmaf(e2.y, w2, fmaf(e1.y, w1, e0.y * w0)));
                if (mv) am[j][k] += sm;
                if (rv) ar[j][k] += sr;
            }
        }
    }
}

#ifndef FDK_SYM_MAXNREG
// 2 CTAs of 288 threads per SM: registers are allocated for an even number of warps (10 of
// the 9), so 2 x 10 x 32 x 96 <= 65536.  (At 112 the SM held one CTA: 9 warps, 14% active.)
// With 4 x 2 x R accumulators, R = 6 fits without spills (R = 8 spills at 96).
#define FDK_SYM_MAXNREG 96
#endif
template <typename E>
__global__ void __maxnreg__(FDK_SYM_MAXNREG)
    bp_sym_kernel(const __grid_constant__ CUtensorMap tmap, BpSymArgs a) {
    using C = SymCfg<E>;
    constexpr int R = C::R, NQ = C::NQ, S = C::S;
    constexpr int BOX = sym_box_bytes<E>();
    constexpr unsigned BOX_TX = C::BW * C::BH * sizeof(E);
    extern __shared__ __align__(128) unsigned char smem[];
    TmaMeta *meta = reinterpret_cast<TmaMeta *>(smem + S * NQ * 4 * BOX);
    uint64_t *bars = reinterpret_cast<uint64_t *>(meta + S * NQ);
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

    const int n_chunks = (a.n_quads + NQ - 1) / NQ;
    const int n_tiles = a.tiles_q * a.tiles_q * a.tiles_z;
    const int half = a.n >> 1;

    if (warp == 8) {
        // ---------------- producer
        int it = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
            const int tx = tile % a.tiles_q, ty = (tile / a.tiles_q) % a.tiles_q;
            const int tz = a.tz0 + tile / (a.tiles_q * a.tiles_q);
            const float xa = (float)(tx * 16), xb = (float)(min(tx * 16 + 16, half) - 1);
            const float ya = (float)(ty * 16), yb = (float)(min(ty * 16 + 16, half) - 1);
            const float za = (float)(a.z0 + tz * R), zb = za + (float)(R - 1);
            for (int c = 0; c < n_chunks; c++, it++) {
                const int s = it % S;
                const unsigned ph = (unsigned)(it / S) & 1u;
                if (it >= S && !mbar_wait_backoff(empty0 + 8 * s, ph ^ 1u, a.wait_ns, FDK_PRODUCER_SLEEP_NS)) {
                    ok = false;
                    break;
                }
                if (a.withhold && blockIdx.x == 0 && it == 0) continue;  // the consumers' wait runs out
                const int qd = c * NQ + lane;
                if (lane < NQ) {
                    TmaMeta &md = meta[s * NQ + lane];
                    if (qd < a.n_quads) {
                        const float *mg = a.mats + 12 * (long long)__ldg(a.q_view + qd);
#pragma unroll
                        for (int i = 0; i < 12; i++) md.m[i] = __ldg(mg + i);
                        sym_tile_box<E>(md.m, xa, xb, ya, yb, za, zb, a.nu, a.nv, md);
                    } else {
                        md.staged = 0;
                        md.interior = 0;
                    }
                }
                __syncwarp();
                if (lane == 0) {
                    unsigned n_staged = 0, n_quads = 0;
                    for (int l = 0; l < NQ; l++)
                        if (c * NQ + l < a.n_quads) {
                            n_quads++;
                            if (meta[s * NQ + l].staged) n_staged++;
                        }
                    if (n_staged != n_quads) atomicOr(a.err, kErrFootprint);  // skipped: an error, never silent
                    mbar_arrive_tx(full0 + 8 * s, n_staged * 4u * BOX_TX);
                    for (int l = 0; l < NQ; l++) {
                        const int ql = c * NQ + l;
                        const TmaMeta &md = meta[s * NQ + l];
                        if (ql < a.n_quads && md.staged) {
                            const int4 sl = __ldg(a.q_slot + ql);
                            const unsigned dst = boxes + (s * NQ + l) * 4 * BOX;
                            tma_load_3d(dst, &tmap, md.v_lo, md.u_lo, sl.x, full0 + 8 * s);
                            tma_load_3d(dst + BOX, &tmap, md.v_lo, md.u_lo, sl.y, full0 + 8 * s);
                            tma_load_3d(dst + 2 * BOX, &tmap, md.v_lo, md.u_lo, sl.z, full0 + 8 * s);
                            tma_load_3d(dst + 3 * BOX, &tmap, md.v_lo, md.u_lo, sl.w, full0 + 8 * s);
                        }
                    }
                }
                __syncwarp();
            }
        }
        if (!ok && lane == 0) atomicOr(a.err, kErrTimeout);
        // drain (always): wait, bounded, for the copies of the last stages to land before the CTA
        // may exit -- consumers that gave up on a wait have left already
        if (lane == 0)
            for (int k = (it > S ? it - S : 0); k < it; k++)
                mbar_wait(full0 + 8 * (k % S), (unsigned)(k / S) & 1u, a.wait_ns);
        return;
    }

    // ---------------- consumers: warps 0..7, lanes = 8 x 4 base columns
    const int wx = warp & 1, wy = warp >> 1;
    const int lx = lane & 7, ly = lane >> 3;
    int it = 0;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int tx = tile % a.tiles_q, ty = (tile / a.tiles_q) % a.tiles_q;
        const int tz = a.tz0 + tile / (a.tiles_q * a.tiles_q);
        const int xi = tx * 16 + wx * 8 + lx, yi = ty * 16 + wy * 4 + ly;
        const bool col_ok = xi < half && yi < half;
        const int zt = tz * R;
        const float zf0 = (float)(a.z0 + zt);
        // the base column and its quarter turns: column j takes member view j's samples (the
        // offsets are formed again for the write-back rather than kept live through the views)
        if (col_ok) {
#pragma unroll
            for (int j = 0; j < 4; j++) prefetch_column<R>(a.vol, a.comp, sym_column_base(xi, yi, j, a), a.D, zt);
        }
        float am[4][R], ar[4][R];
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int k = 0; k < R; k++) am[j][k] = ar[j][k] = 0.f;
        for (int c = 0; c < n_chunks; c++, it++) {
            const int s = it % S;
            const unsigned ph = (unsigned)(it / S) & 1u;
            if (!mbar_wait(full0 + 8 * s, ph, a.wait_ns)) {
                if (lane == 0) atomicOr(a.err, kErrTimeout);
                return;
            }
            if (col_ok) {
                for (int l = 0; l < NQ; l++) {
                    const int ql = c * NQ + l;
                    if (ql >= a.n_quads) break;
                    const TmaMeta &md = meta[s * NQ + l];
                    if (!md.staged) continue;  // never for checked geometries; reported by the producer
                    column_quad<E>(md, boxes + (s * NQ + l) * 4 * BOX, (float)xi, (float)yi, zf0, a.nu, a.nv,
                                   a.wscale, am, ar);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty0 + 8 * s);
        }
        if (col_ok) {
            const float sc = (a.scale ? *a.scale : 1.0f) / a.wscale;
            const int nrun = min(R, a.nzz - zt);
#pragma unroll
            for (int j = 0; j < 4; j++)
                write_back<R>(a.vol, a.comp, sym_column_base(xi, yi, j, a), a.D, zt, nrun, sc, am[j], ar[j]);
        }
    }
}

}  // namespace fdk

// ---------------------------------------------------------------------------------------
// host side
namespace fdk {

// 3-D map over MIRROR views [n][nu][nv] with this kernel's box.
template <typename E>
inline int encode_sym_map(CUtensorMap *map, const void *base, int nu, int nv, int n) {
    EncodeTiledFn enc = tensor_map_encoder();
    if (!enc) return fail(FDK_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t dims[3] = {(cuuint64_t)nv, (cuuint64_t)nu, (cuuint64_t)n};
    const cuuint64_t strides[2] = {(cuuint64_t)nv * sizeof(E), (cuuint64_t)nu * nv * sizeof(E)};
    const cuuint32_t box[3] = {(cuuint32_t)SymCfg<E>::BW, (cuuint32_t)SymCfg<E>::BH, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapDataType dt = sizeof(E) == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    CUresult r = enc(map, dt, 3, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(FDK_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return FDK_OK;
}

template <typename E>
inline int sym_prepare(int &ctas, int device) {
    const int smem = sym_smem_bytes<E>();
    FDK_CUDA(cudaFuncSetAttribute(bp_sym_kernel<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    // room for two CTAs' boxes per SM
    FDK_CUDA(cudaFuncSetAttribute(bp_sym_kernel<E>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    int per_sm = 0, sms = 0;
    FDK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_sym_kernel<E>, 288, smem));
    FDK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    ctas = sms * (per_sm > 0 ? per_sm : 1);
    return FDK_OK;
}

// Backproject nq quadruples (slots into a views buffer of n_slots views, base views' matrices in
// d_mats / host_mats indexed by view) into the top slices [z_begin, z_end) of the slab pair and
// their mirrors.  The plan's sub-volume must be the whole square x-y grid.  q: the host record,
// checked here; d_q: its device copy, which the kernel reads (uploaded on st before this launch).
template <typename E>
inline int bp_sym_launch(const BpFastPlan &p, int ctas, float *vol, float *comp, const void *views, int n_slots,
                         const float *d_mats, const float *host_mats, const SymQuads &q, const SymQuads *d_q, int nq,
                         int rot, cudaStream_t st, const float *scale, long long z_begin, long long z_end) {
    using C = SymCfg<E>;
    FDK_CHECK_ARG(((uintptr_t)views & 15) == 0, "TMA views must start on a 16-byte boundary");
    FDK_CHECK_ARG(nq > 0 && nq <= kSymMaxQuads, "quadruples %d outside 1..%d", nq, kSymMaxQuads);
    FDK_CHECK_ARG(p.x0 == 0 && p.y0 == 0 && p.nxs == p.nys && p.nxs % 2 == 0 && rot != 0,
                  "the quarter-turn kernel needs the whole square grid (even side)");
    for (int i = 0; i < nq; i++) {
        const int4 s = q.slot[i];
        FDK_CHECK_ARG(s.x >= 0 && s.x < n_slots && s.y >= 0 && s.y < n_slots && s.z >= 0 && s.z < n_slots &&
                          s.w >= 0 && s.w < n_slots,
                      "quadruple %d: slot outside the views buffer", i);
    }
    CUtensorMap map;
    FDK_TRY(encode_sym_map<E>(&map, views, p.nu, p.nv, n_slots));
    BpSymArgs a;
    a.vol = vol;
    a.comp = comp;
    a.proj = views;
    a.mats = d_mats;
    a.scale = scale;
    a.err = p.d_err;
    a.n_quads = nq;
    a.nu = p.nu;
    a.nv = p.nv;
    a.n = p.nxs;
    a.z0 = p.z0;
    a.nzz = p.nzz;
    a.D = p.D;
    const float *m0 = host_mats + 12 * (long long)q.view[0];
    a.wscale = weight_scale(m0, 0.5f * (p.nxs - 1), 0.5f * (p.nys - 1));
    a.tiles_q = (int)ceil_div(p.nxs / 2, 16);
    const int tz_all = (int)ceil_div(p.nzz, C::R);
    const int tzb = (int)(z_begin / C::R), tze = z_end < 0 ? tz_all : (int)std::min<long long>(ceil_div(z_end, C::R), tz_all);
    FDK_CHECK_ARG(z_begin % C::R == 0 && tzb >= 0 && tzb < tze, "z range [%lld, %lld) does not split into %d-slice tiles",
                  z_begin, z_end, C::R);
    a.tz0 = tzb;
    a.tiles_z = tze - tzb;
    a.rot = rot;
    a.wait_ns = bp_wait_ns();
    a.withhold = bp_test_withhold();
    FDK_CHECK_ARG(d_q != nullptr, "quadruples need their device copy");
    const char *dq = reinterpret_cast<const char *>(d_q);  // addresses inside the device copy
    a.q_slot = reinterpret_cast<const int4 *>(dq + offsetof(SymQuads, slot));
    a.q_view = reinterpret_cast<const int *>(dq + offsetof(SymQuads, view));
    const long long n_tiles = (long long)a.tiles_q * a.tiles_q * a.tiles_z;
    FDK_CHECK_ARG(n_tiles < (1ll << 31), "too many tiles");
    const int grid = (int)std::min<long long>(n_tiles, ctas);
    bp_sym_kernel<E><<<grid, 288, sym_smem_bytes<E>(), st>>>(map, a);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
}

}  // namespace fdk
