// bp_fast.cuh -- shared-memory staged voxel-driven backprojection for sm_100a.
//
// Geometry contract (circular orbit, the reference's bSymmetric path, backprojectionFDK.cu:
// 90-126): rows 0 and 2 of every 3x4 matrix have no z term, so for a voxel column (x, y) the
// detector column U = (m0.(x,y,1)) / w and the weight 1/w^2, w = m2.(x,y,1), do not depend on
// z, and the detector row is linear in z: v(z) = A + B z.  The mirror voxel nz-1-z of the
// slab pair lands on detector row nv-1-v.
//
// Data layout.  Filtered views arrive in the MIRROR layout: element (u, v) holds the pair
// (P[u][v], P[u][nv-1-v]) as float2 (FP32) or half2 (MIXED).  One bilinear gather of four
// pair elements therefore serves a voxel and its mirror: with vi = floor(v), fv = v - vi,
//     main   = (1-fv) lerp_u(E[vi].x) + fv lerp_u(E[vi+1].x)
//     mirror = (1-fv) lerp_u(E[vi].y) + fv lerp_u(E[vi+1].y)
// because the mirror row nv-1-v interpolates P[nv-1-vi] (weight 1-fv) and P[nv-2-vi]
// (weight fv).  Bounds follow SUBPIXEL (backprojectionFDK.cu:18): a sample is zero unless
// 0 <= u < nu-1 and 0 <= v < nv-1 (main) / 0 <= nv-1-v < nv-1 (mirror).
//
// Work decomposition.  A CTA owns a 16 x 16 block of voxel columns and a run of R top-slab z
// values (plus their R mirrors): one thread per column, 2R FP32 accumulators in registers.
// Views are processed in chunks of NCH: for each view the CTA stages the detector footprint
// box of its voxels (all pairs it can touch) into shared memory, then every thread gathers
// from shared memory.  Views whose footprint exceeds the staging capacity are gathered from
// global memory instead (same arithmetic, slower).  After the last view each thread adds its
// accumulators to the volume ([x][y][zs] with zs = top slab then bottom slab ascending, the
// reference's storage), once per launch.
#pragma once
#include <cuda_fp16.h>

#include "common.h"

namespace fdk {

constexpr int kFastTile = 16;     // columns per CTA side
constexpr int kFastR = 8;         // top-slab z values per thread
constexpr int kFastNch = 8;       // views per staging chunk
constexpr int kFastBoxW = 24;     // staged box width (v extent, elements)
constexpr int kFastBoxH = 48;     // staged box height capacity (u extent, rows)

struct BpFastPlan {
    int precision = 0;
    int nu = 0, nv = 0;       // detector columns (frame rows) and rows (frame width)
    int x0 = 0, y0 = 0, z0 = 0;
    int nxs = 0, nys = 0, nzz = 0;
    long long D = 0;
    int device = 0;
    float *d_scale = nullptr; // device scalar: accumulator scale of the MIXED path
    bool tma_ok = false;      // the TMA kernel applies (row stride a multiple of 16 B)
    int tma_ctas = 0;         // persistent grid size of the TMA kernel
    unsigned int *d_err = nullptr;  // device error word of the TMA kernel
};

struct BpFastArgs {
    float *vol;
    float *comp;
    const void *proj;     // MIRROR layout, nu rows x nv pairs per view
    const float *mats;    // 12 floats per view
    const float *scale;   // MIXED: device scalar multiplying the accumulators (view scale); else null
    int n_proj, nu, nv;
    int x0, y0, z0, nxs, nys, nzz;
    long long D;
    float wscale;         // weights are f^2 * wscale (keeps FP16 products in range)
};

struct ViewBox {
    int u_lo, v_lo, rows, cols;
    int staged;   // 1: box in shared memory, 0: gather from global
    int interior; // 1: every sample of the tile is inside the detector (no per-sample checks)
};

template <typename E>
struct PairOps;

template <>
struct PairOps<float2> {
    static __device__ __forceinline__ float2 load_g(const float2 *p) { return __ldg(p); }
};
template <>
struct PairOps<__half2> {
    static __device__ __forceinline__ __half2 load_g(const __half2 *p) {
        unsigned int r = __ldg(reinterpret_cast<const unsigned int *>(p));
        return *reinterpret_cast<__half2 *>(&r);
    }
};

// Footprint of the CTA's voxels in view s: corners of the column block x the z run.
__device__ __forceinline__ void view_footprint(const float *m, float xa, float xb, float ya, float yb, float za,
                                               float zb, float &umin, float &umax, float &vmin, float &vmax) {
    umin = vmin = 3.0e38f;
    umax = vmax = -3.0e38f;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float x = (c & 1) ? xb : xa, y = (c & 2) ? yb : ya;
        const float w = fmaf(m[8], x, fmaf(m[9], y, m[11]));
        const float rw = 1.0f / w;
        const float U = fmaf(m[0], x, fmaf(m[1], y, m[3])) * rw;
        const float vw = fmaf(m[4], x, fmaf(m[5], y, m[7]));
        const float va = fmaf(m[6], za, vw) * rw, vb = fmaf(m[6], zb, vw) * rw;
        umin = fminf(umin, U);
        umax = fmaxf(umax, U);
        vmin = fminf(vmin, fminf(va, vb));
        vmax = fmaxf(vmax, fmaxf(va, vb));
    }
}

template <typename E>
__device__ __forceinline__ void accumulate_pair(float &am, float &ar, E e0, E e1, E e2, E e3, float fu, float fv,
                                                float w, bool mvalid, bool rvalid);

template <>
__device__ __forceinline__ void accumulate_pair<float2>(float &am, float &ar, float2 e0, float2 e1, float2 e2,
                                                        float2 e3, float fu, float fv, float w, bool mvalid,
                                                        bool rvalid) {
    // e0 = E[u0][vi], e1 = E[u0][vi+1], e2 = E[u0+1][vi], e3 = E[u0+1][vi+1]
    const float c0x = fmaf(fu, e2.x - e0.x, e0.x), c0y = fmaf(fu, e2.y - e0.y, e0.y);
    const float c1x = fmaf(fu, e3.x - e1.x, e1.x), c1y = fmaf(fu, e3.y - e1.y, e1.y);
    const float rx = fmaf(fv, c1x - c0x, c0x), ry = fmaf(fv, c1y - c0y, c0y);
    am = fmaf(mvalid ? w : 0.0f, rx, am);
    ar = fmaf(rvalid ? w : 0.0f, ry, ar);
}

template <>
__device__ __forceinline__ void accumulate_pair<__half2>(float &am, float &ar, __half2 e0, __half2 e1, __half2 e2,
                                                         __half2 e3, float fu, float fv, float w, bool mvalid,
                                                         bool rvalid) {
    const __half2 fu2 = __float2half2_rn(fu);
    const __half2 c0 = __hfma2(fu2, __hsub2(e2, e0), e0);
    const __half2 c1 = __hfma2(fu2, __hsub2(e3, e1), e1);
    const __half2 r = __hfma2(__float2half2_rn(fv), __hsub2(c1, c0), c0);
    const float2 rf = __half22float2(r);
    am = fmaf(mvalid ? w : 0.0f, rf.x, am);
    ar = fmaf(rvalid ? w : 0.0f, rf.y, ar);
}

template <typename E>
__global__ void __launch_bounds__(256) bp_fast_kernel(BpFastArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    E *stage = reinterpret_cast<E *>(smem_raw);
    __shared__ float4 smat[kFastNch * 3];
    __shared__ ViewBox sbox[kFastNch];

    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int cx0 = blockIdx.x * kFastTile, cy0 = blockIdx.y * kFastTile;
    const int zt = blockIdx.z * kFastR;  // first top-slab z (relative) of the run
    const int xi = cx0 + tx, yi = cy0 + ty;
    const bool col_ok = xi < a.nxs && yi < a.nys;
    const float x = (float)(a.x0 + xi), y = (float)(a.y0 + yi);
    const float zf0 = (float)(a.z0 + zt);
    const int nrun = min(kFastR, a.nzz - zt);
    const long long frame = (long long)a.nu * a.nv;
    const E *proj = reinterpret_cast<const E *>(a.proj);

    float am[kFastR], ar[kFastR];
#pragma unroll
    for (int k = 0; k < kFastR; k++) am[k] = ar[k] = 0.f;

    // CTA footprint corners (voxel centres of the block and run)
    const float xa = (float)(a.x0 + cx0), xb = (float)(a.x0 + min(cx0 + kFastTile, a.nxs) - 1);
    const float ya = (float)(a.y0 + cy0), yb = (float)(a.y0 + min(cy0 + kFastTile, a.nys) - 1);
    // the footprint covers the whole run of kFastR even past the slab end: those voxels are
    // computed (and discarded), so their gathers must stay inside the staged box too
    const float za = zf0, zb = zf0 + (float)(kFastR - 1);

    for (int c0 = 0; c0 < a.n_proj; c0 += kFastNch) {
        const int nch = min(kFastNch, a.n_proj - c0);
        __syncthreads();  // previous chunk fully consumed
        if (tid < nch * 3) smat[tid] = reinterpret_cast<const float4 *>(a.mats + 12 * c0)[tid];
        __syncthreads();
        if (tid < nch) {
            const float *m = reinterpret_cast<const float *>(&smat[tid * 3]);
            float umin, umax, vmin, vmax;
            view_footprint(m, xa, xb, ya, yb, za, zb, umin, umax, vmin, vmax);
            ViewBox b;
            // one element of margin on every side absorbs FP32 rounding differences between
            // the corner footprint and the per-column coordinates
            const int u_lo = (int)fmaxf(floorf(umin) - 1.f, 0.f);
            const int v_lo = (int)fmaxf(floorf(vmin) - 1.f, 0.f);
            const int u_hi = (int)fminf(floorf(umax) + 2.f, (float)(a.nu - 1));
            const int v_hi = (int)fminf(floorf(vmax) + 2.f, (float)(a.nv - 1));
            b.u_lo = u_lo;
            b.v_lo = v_lo;
            b.rows = max(0, u_hi - u_lo + 1);
            b.cols = max(0, v_hi - v_lo + 1);
            b.staged = (b.rows <= kFastBoxH && b.cols <= kFastBoxW) ? 1 : 0;
            // interior: every U in [0, nu-1) and every v in (0, nv-1) with a margin
            b.interior = (umin >= 0.f && umax < (float)(a.nu - 1) - 1e-3f && vmin > 1e-3f &&
                          vmax < (float)(a.nv - 1) - 1e-3f)
                             ? 1
                             : 0;
            if (b.rows == 0 || b.cols == 0) b.staged = 1;  // nothing to stage, all samples zero
            sbox[tid] = b;
        }
        __syncthreads();
        // cooperative staging of the boxes
        for (int s = 0; s < nch; s++) {
            const ViewBox b = sbox[s];
            if (!b.staged) continue;
            const E *src = proj + (long long)(c0 + s) * frame;
            E *dst = stage + s * (kFastBoxH * kFastBoxW);
            const int n = b.rows * b.cols;
            for (int q = tid; q < n; q += 256) {
                const int r = q / b.cols, c = q - r * b.cols;
                dst[r * kFastBoxW + c] = PairOps<E>::load_g(src + (long long)(b.u_lo + r) * a.nv + b.v_lo + c);
            }
        }
        __syncthreads();
        if (!col_ok) continue;
        for (int s = 0; s < nch; s++) {
            const float *m = reinterpret_cast<const float *>(&smat[s * 3]);
            const ViewBox b = sbox[s];
            const float w = fmaf(m[8], x, fmaf(m[9], y, m[11]));
            const float rw = 1.0f / w;
            const float U = fmaf(m[0], x, fmaf(m[1], y, m[3])) * rw;
            const float A = fmaf(m[4], x, fmaf(m[5], y, fmaf(m[6], zf0, m[7]))) * rw;
            const float B = m[6] * rw;
            const float wt = rw * rw * a.wscale;
            const bool u_ok = U >= 0.f && U < (float)(a.nu - 1);
            if (!u_ok) continue;  // every sample of this column is zero in this view
            const float fuf = floorf(U);
            const float fu = U - fuf;
            const int u0 = (int)fuf;
            if (b.staged) {
                const E *row0 = stage + s * (kFastBoxH * kFastBoxW) + (u0 - b.u_lo) * kFastBoxW - b.v_lo;
                const E *row1 = row0 + kFastBoxW;
                if (b.interior) {
#pragma unroll
                    for (int k = 0; k < kFastR; k++) {
                        const float v = fmaf(B, (float)k, A);
                        const float vf = floorf(v);
                        const int vi = (int)vf;
                        accumulate_pair<E>(am[k], ar[k], row0[vi], row0[vi + 1], row1[vi], row1[vi + 1], fu, v - vf,
                                           wt, true, true);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < kFastR; k++) {
                        const float v = fmaf(B, (float)k, A);
                        const float vr = (float)(a.nv - 1) - v;
                        const bool mv = v >= 0.f && v < (float)(a.nv - 1);
                        const bool rv = vr >= 0.f && vr < (float)(a.nv - 1);
                        if (mv || rv) {
                            const float vf = fminf(floorf(v), (float)(a.nv - 2));
                            const int vi = (int)vf;
                            accumulate_pair<E>(am[k], ar[k], row0[vi], row0[vi + 1], row1[vi], row1[vi + 1], fu,
                                               v - vf, wt, mv, rv);
                        }
                    }
                }
            } else {
                const E *g0 = proj + (long long)(c0 + s) * frame + (long long)u0 * a.nv;
                const E *g1 = g0 + a.nv;
#pragma unroll
                for (int k = 0; k < kFastR; k++) {
                    const float v = fmaf(B, (float)k, A);
                    const float vr = (float)(a.nv - 1) - v;
                    const bool mv = v >= 0.f && v < (float)(a.nv - 1);
                    const bool rv = vr >= 0.f && vr < (float)(a.nv - 1);
                    if (mv || rv) {
                        const float vf = fminf(floorf(v), (float)(a.nv - 2));
                        const int vi = (int)vf;
                        accumulate_pair<E>(am[k], ar[k], PairOps<E>::load_g(g0 + vi), PairOps<E>::load_g(g0 + vi + 1),
                                           PairOps<E>::load_g(g1 + vi), PairOps<E>::load_g(g1 + vi + 1), fu, v - vf,
                                           wt, mv, rv);
                    }
                }
            }
        }
    }
    if (!col_ok) return;
    const float sc = (a.scale ? *a.scale : 1.0f) / a.wscale;
    float *out = a.vol + ((long long)xi * a.nys + yi) * a.D;
    float *cmp = a.comp ? a.comp + ((long long)xi * a.nys + yi) * a.D : nullptr;
    for (int k = 0; k < nrun; k++) {
        const long long it = zt + k, ib = a.D - 1 - it;
        const float dm = am[k] * sc, dr = ar[k] * sc;
        if (cmp) {
            // compensated (Kahan) accumulation across launches
            float y1 = dm - cmp[it];
            float t1 = out[it] + y1;
            cmp[it] = (t1 - out[it]) - y1;
            out[it] = t1;
            float y2 = dr - cmp[ib];
            float t2 = out[ib] + y2;
            cmp[ib] = (t2 - out[ib]) - y2;
            out[ib] = t2;
        } else {
            out[it] += dm;
            out[ib] += dr;
        }
    }
}

// Adds the compensation term into the volume and clears it (before the volume is read).
__global__ void fold_comp_kernel(float *vol, float *comp, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        vol[i] -= comp[i];
        comp[i] = 0.f;
    }
}

inline int bp_fast_fold_compensation(float *vol, float *comp, long long n, cudaStream_t st) {
    fold_comp_kernel<<<148 * 8, 256, 0, st>>>(vol, comp, n);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
}

inline int bp_fast_plan(BpFastPlan &p, int precision, int proj_w, int proj_h, int x0, int y0, int z0, int nxs,
                        int nys, int depth_top, long long D, int device, cudaStream_t st) {
    p.precision = precision;
    p.nv = proj_w;  // transposed frame: width = detector rows
    p.nu = proj_h;
    p.x0 = x0;
    p.y0 = y0;
    p.z0 = z0;
    p.nxs = nxs;
    p.nys = nys;
    p.nzz = depth_top;
    p.D = D;
    p.device = device;
    FDK_CUDA(cudaMalloc(&p.d_scale, sizeof(float)));
    const float one = 1.0f;
    FDK_CUDA(cudaMemcpyAsync(p.d_scale, &one, sizeof(float), cudaMemcpyHostToDevice, st));  // pageable: staged now
    const size_t smem = (size_t)kFastNch * kFastBoxH * kFastBoxW * (precision == FDK_BP_MIXED ? 4 : 8);
    if (precision == FDK_BP_MIXED)
        FDK_CUDA(cudaFuncSetAttribute(bp_fast_kernel<__half2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else
        FDK_CUDA(cudaFuncSetAttribute(bp_fast_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return FDK_OK;
}

inline void bp_fast_release(BpFastPlan &p) {
    if (p.d_scale) cudaFree(p.d_scale);
    if (p.d_err) cudaFree(p.d_err);
    p.d_scale = nullptr;
    p.d_err = nullptr;
}

// wscale: 1/w^2 is ~1e-6 for mm geometries; multiplying by the squared source distance of the
// volume centre keeps FP16 products near 1.  The factor is divided out when the accumulators
// are folded into the volume.
inline int bp_fast_launch(const BpFastPlan &p, float *vol, float *comp, const void *proj, const float *mats, int n,
                          cudaStream_t st, float wscale = 1.0e6f, const float *scale = nullptr) {
    BpFastArgs a;
    a.vol = vol;
    a.comp = comp;
    a.proj = proj;
    a.mats = mats;
    a.scale = scale;
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
    a.wscale = wscale;
    const dim3 grid((unsigned)ceil_div(p.nxs, kFastTile), (unsigned)ceil_div(p.nys, kFastTile),
                    (unsigned)ceil_div(p.nzz, kFastR));
    if (p.precision == FDK_BP_MIXED) {
        const size_t smem = (size_t)kFastNch * kFastBoxH * kFastBoxW * sizeof(__half2);
        bp_fast_kernel<__half2><<<grid, 256, smem, st>>>(a);
    } else {
        const size_t smem = (size_t)kFastNch * kFastBoxH * kFastBoxW * sizeof(float2);
        bp_fast_kernel<float2><<<grid, 256, smem, st>>>(a);
    }
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
}

}  // namespace fdk
