// bp.cu -- BackProjectionFDK behind the C ABI (cudaBP/backprojection.cuh:246-271,
// cudaBP/backprojectionFDK.cu:161-362).
//
// Device state per handle: the sub-volume in the reference's layout [x][y][zs] (zs fastest,
// top slab then bottom slab, backprojectionFDK.cu:119-126), two staging buffers for host
// views so the copy of batch k+1 overlaps the kernel of batch k (copy stream + events), the
// per-view matrices, and the kernel timer.
#include <cuda_fp16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>
#include <thread>
#include <vector>

#include "bp_exact.cuh"
#include "bp_fast.cuh"
#include "bp_sym.cuh"
#include "bp_tma.cuh"
#include "common.h"

namespace fdk {

// [x][y][zs] -> [zs][y][x] for zs in [z_begin, z_begin + dz), x fastest
// (kernelTransformVolume, backprojectionFDK.cu:131-148).  One warp per block walks 32 x 32
// (x, zs) tiles grid-stride.  A readback runs beside the persistent backprojection, whose
// warps leave each SM sub-partition room for about one more warp of 32 registers: single-warp
// blocks capped at 32 registers fit there, larger blocks wait for the backprojection to end.
template <bool COMP>
__global__ void __maxnreg__(32) transform_volume_kernel(const float *__restrict__ src, const float *__restrict__ comp,
                                                      float *__restrict__ dst, int nxs, int nys, long long D,
                                                      long long z_begin, int dz) {
    __shared__ float tile[32][33];
    const int lane = threadIdx.x;
    const int ntx = (nxs + 31) / 32, ntz = (dz + 31) / 32;
    const long long n_tiles = (long long)ntx * ntz * nys;
    const long long xs = (long long)nys * D, zs = (long long)nys * nxs;  // strides of x in src, z in dst
    for (long long t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const int x0 = (int)(t % ntx) * 32;
        const long long r = t / ntx;
        const int z0 = (int)(r % ntz) * 32, y = (int)(r / ntz);
        const int nx = min(32, nxs - x0), nz = min(32, dz - z0);
        // read: lanes walk zs (contiguous in src)
        if (lane < nz) {
            const long long o = ((long long)x0 * nys + y) * D + z_begin + z0 + lane;
            const float *s = src + o;
            const float *c = COMP ? comp + o : nullptr;
#pragma unroll 4
            for (int row = 0; row < nx; row++, s += xs) {
                if (COMP) {
                    tile[row][lane] = *s - *c;  // MIXED folds its compensation
                    c += xs;
                } else {
                    tile[row][lane] = *s;
                }
            }
        }
        __syncwarp();
        if (lane < nx) {
            float *d = dst + ((long long)z0 * nys + y) * nxs + x0 + lane;
#pragma unroll 4
            for (int row = 0; row < nz; row++, d += zs) *d = tile[lane][row];
        }
        __syncwarp();
    }
}

// TRANSPOSED f32 views (height = nu rows of width = nv) -> MIRROR pairs (u, v) = (v, nv-1-v).
template <typename T2>
__global__ void to_mirror_kernel(const float *__restrict__ src, T2 *__restrict__ dst, int width, int height,
                                 int n) {
    const long long frame = (long long)width * height;
    const long long total = frame * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long f = i / frame;
        const long long r = i - f * frame;
        const int row = (int)(r / width), v = (int)(r - (long long)row * width);
        const float *p = src + f * frame + (long long)row * width;
        const float a = p[v], b = p[width - 1 - v];
        if constexpr (sizeof(T2) == 8) dst[i] = make_float2(a, b);
        else dst[i] = __floats2half2_rn(a, b);
    }
}

// Largest magnitude of n floats, as the bit pattern of a non-negative float (atomicMax on
// the unsigned bits orders non-negative floats correctly).
__global__ void absmax_kernel(const float *__restrict__ x, long long n, unsigned int *out) {
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(x[i]));
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// Power-of-two scale that brings the batch maximum to at most 2^14 in FP16 (exact scaling).
__device__ __forceinline__ float half_scale(unsigned int absmax_bits) {
    const float m = fmaxf(__uint_as_float(absmax_bits), 1e-30f);
    return exp2f(floorf(log2f(16384.f / m)));
}

// TRANSPOSED f32 views -> MIRROR half2 pairs scaled by half_scale(); acc_scale = 1/scale.
__global__ void to_mirror_half_kernel(const float *__restrict__ src, __half2 *__restrict__ dst, int width, int height,
                                      int n, const unsigned int *absmax, float *acc_scale) {
    const float sc = half_scale(*absmax);
    if (blockIdx.x == 0 && threadIdx.x == 0) *acc_scale = 1.0f / sc;
    const long long frame = (long long)width * height;
    const long long total = frame * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long f = i / frame;
        const long long r = i - f * frame;
        const int row = (int)(r / width), v = (int)(r - (long long)row * width);
        const float *p = src + f * frame + (long long)row * width;
        dst[i] = __floats2half2_rn(p[v] * sc, p[width - 1 - v] * sc);
    }
}

// rows-layout f32 views (nv rows of nu) -> TRANSPOSED f32 (nu rows of nv)
__global__ void transpose_views_kernel(const float *__restrict__ src, float *__restrict__ dst, int nu, int nv) {
    __shared__ float tile[32][33];
    const long long f = blockIdx.z;
    const float *s = src + f * nu * (long long)nv;
    float *d = dst + f * nu * (long long)nv;
    const int u0 = blockIdx.x * 32, v0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int v = v0 + r, u = u0 + threadIdx.x;
        if (u < nu && v < nv) tile[r][threadIdx.x] = s[(long long)v * nu + u];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int u = u0 + r, v = v0 + threadIdx.x;
        if (u < nu && v < nv) d[(long long)u * nv + v] = tile[threadIdx.x][r];
    }
}

// Largest magnitude of the FP16 values of n half2 pairs, as the bits of a non-negative float
// (as absmax_kernel).  16-byte loads; pairs past the last whole group of four one by one.
__global__ void absmax_half2_kernel(const __half2 *__restrict__ x, long long n, unsigned int *out) {
    float m = 0.f;
    const long long n4 = n / 4;
    const uint4 *x4 = reinterpret_cast<const uint4 *>(x);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
        const uint4 q = x4[i];
        const unsigned w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&w[j]));
            m = fmaxf(m, fmaxf(fabsf(f.x), fabsf(f.y)));
        }
    }
    for (long long i = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
        const float2 f = __half22float2(x[i]);
        m = fmaxf(m, fmaxf(fabsf(f.x), fabsf(f.y)));
    }
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

__device__ __forceinline__ float pow2i(int e) { return __int_as_float((127 + e) << 23); }  // -126 <= e <= 127

// MIRROR FP16 views -> the interpolation layout (HalfLerp), scaled by 2^-k with 2^k just above
// the batch's largest magnitude M (absmax): e = E(v) 2^-k (exact unless it falls below the FP16
// normal range), d = (E(v+1) - E(v)) 2^(14-k) rounded to FP16 (|d| < 2^15; 0 at v = nv-1).  A
// sample at v + fv is then e + (fv 2^-14) d, fv 2^-14 being the FP16 subnormal whose mantissa
// is the fixed-point fraction, so the sample carries the roundings of E(v) and of d only.
// out_scale = acc_scale (1 if null) * 2^k, the accumulator scale of the launches that read dst.
__global__ void to_lerp_kernel(const __half2 *__restrict__ src, HalfLerp *__restrict__ dst, long long rows,
                               int nv, const unsigned int *absmax, const float *acc_scale, float *out_scale) {
    const float M = __uint_as_float(*absmax);
    const int k = (M > 0.f && M < 65536.f) ? ilogbf(M) + 1 : 0;  // M is an FP16 magnitude: -23 <= k <= 16
    const float se = pow2i(-k), sd = pow2i(14 - k);
    if (blockIdx.x == 0 && threadIdx.x == 0) *out_scale = (acc_scale ? *acc_scale : 1.0f) * pow2i(k);
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        const __half2 *s = src + r * nv;
        HalfLerp *d = dst + r * nv;
        for (int v = threadIdx.x; v < nv; v += blockDim.x) {
            const float2 e0 = __half22float2(s[v]);
            const float2 e1 = v + 1 < nv ? __half22float2(s[v + 1]) : e0;
            HalfLerp o;
            o.e = __floats2half2_rn(e0.x * se, e0.y * se);
            o.d = __floats2half2_rn((e1.x - e0.x) * sd, (e1.y - e0.y) * sd);
            d[v] = o;
        }
    }
}

// Gather listed voxels (x, y, z of the whole volume) from the slab-pair volume [x][y][zs];
// voxels outside the handle's boxes read NaN.  MIXED folds its compensation term.
__global__ void sample_voxels_kernel(const float *__restrict__ vol, const float *__restrict__ comp,
                                     const int *__restrict__ xyz, long long n, float *__restrict__ out, int x0,
                                     int y0, int nxs, int nys, long long tz0, long long td, long long bz0,
                                     long long bd, long long D) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = xyz[3 * i] - x0, y = xyz[3 * i + 1] - y0;
        const long long z = xyz[3 * i + 2];
        long long zs = -1;
        if (z >= tz0 && z < tz0 + td) zs = z - tz0;
        else if (bd > 0 && z >= bz0 && z < bz0 + bd) zs = td + (z - bz0);
        float v = __int_as_float(0x7fc00000);
        if (zs >= 0 && x >= 0 && x < nxs && y >= 0 && y < nys) {
            const long long o = ((long long)x * nys + y) * D + zs;
            v = comp ? vol[o] - comp[o] : vol[o];
        }
        out[i] = v;
    }
}

}  // namespace fdk

using namespace fdk;

namespace {
// Most z bands per batch (tuning macro).  On the 2048^3 workload 8 bands against 4: the same
// device time (2383 against 2386 GUPS) and e2e 2182 against 2117 GUPS, as the readback of the
// last band, which no backprojection hides, halves.  16 against 8 with the current kernels
// (64-slice bands, 221 tiles per persistent CTA): 3044 against 3014 GUPS and e2e 2776 against
// 2743 (one box, each twice).
#ifndef FDK_MAX_BANDS
#define FDK_MAX_BANDS 16
#endif
constexpr int kMaxBands = FDK_MAX_BANDS;
}

struct fdk_bp {
    int device = 0, precision = FDK_BP_FP32_EXACT;
    int proj_w = 0, proj_h = 0, proj_count = 0;
    int nx = 0, ny = 0, nz = 0;
    fdk_box top{}, bottom{};
    bool sym = false;
    long long D = 0;
    float *d_vol = nullptr;
    float *d_comp = nullptr;      // compensation term of the MIXED accumulation
    float *d_stage[2] = {nullptr, nullptr};  // host-view staging (f32, as received)
    void *d_mirror = nullptr;     // converted views for the fast kernels
    float *d_mats = nullptr;      // 2 x 128 x 12
    int slot = 0;
    cudaStream_t stream = nullptr, copy_stream = nullptr;
    cudaEvent_t copied[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timers, free_timers;
    long long bp_count = 0;
    double kernel_ms = 0;
    BpFastPlan plan;
    // MIXED: word 0 the largest |value| of the f32 views of a call; words 1-3 that of the FP16
    // views of interpolation-layout buffer 0, 1 and the calls' buffer, words 5-7 (as floats) the
    // accumulator scales of the launches that read those buffers (to_lerp_kernel)
    unsigned int *d_absmax = nullptr;
    const float *ext_scale = nullptr;  // accumulator scale of FP16 views pushed by the reconstructor
    // The staged kernel runs each batch as n_bands launches over bands of z tiles (top slices
    // [band_z[k], band_z[k+1]) with their mirrors), each recording band_done[k]; a readback
    // copies band k to the host while the later bands of the last batch still run.
    int n_bands = 1;
    long long band_z[kMaxBands + 1] = {};
    int band_tz[kMaxBands + 1] = {};          // the same bounds in z tiles of the staged kernel
    cudaEvent_t band_done[kMaxBands] = {};
    cudaStream_t rb[2] = {nullptr, nullptr};  // readback streams
    float *d_rb = nullptr;                    // readback staging, 2 x rb_planes z planes
    long long rb_planes = 0;
    long long launches = 0;                   // kernel launches since creation or reset
    cudaEvent_t sync_ev[3] = {};              // scratch events of the bounded host waits
    unsigned int *h_err = nullptr;            // pinned host copy of the device error word
    int sym_rot = 0;                          // quarter-turn kernel: its column map (0: not set up)
    int sym_ctas = 0;                         // its persistent grid
    // Ring of launch view lists (fdk_bp_bp_lists_internal): a pinned host record per entry,
    // uploaded on the launch stream to the entry's device copy, which the kernel reads; an entry
    // is written again once the event recorded after its launch has passed.
    union ListRec {
        SymQuads quads;
        ViewList views;
    };
    static constexpr int kListRing = 64;
    // MIXED views of the list launches converted to the interpolation layout (HalfLerp), one
    // buffer per source views buffer (the held and the filling batch of a reconstructor), tagged
    // with the source; reserved by fdk_bp_reserve_lerp_internal
    HalfLerp *d_lerp[2] = {nullptr, nullptr};
    const void *lerp_src[2] = {nullptr, nullptr};
    long long lerp_slots = 0;
    int lerp_next = 0;
    // MIXED views of the BackProjectionFDK calls (fdk_bp_bp, fdk_bp_bp_device) in the
    // interpolation layout: allocated at the first call, reused once the event recorded after
    // the last call's launches has passed on the next call's stream
    HalfLerp *d_lerp_call = nullptr;
    long long lerp_call_cap = 0;
    cudaEvent_t lerp_call_ev = nullptr;
    bool lerp_call_used = false;
    // the reconstructor's MIXED launches read through the compact boxes (every tile fits them)
    bool lerp_compact = false;
    bool lerp_compact_ok = false;  // the compact kernel runs at the same grid
    ListRec *h_list = nullptr, *d_list = nullptr;
    cudaEvent_t list_ev[kListRing] = {};
    bool list_used[kListRing] = {};
    int list_next = 0;
};

namespace bpi {

int collect_timers(fdk_bp *h) {
    for (auto &t : h->timers) {
        FDK_TRY(wait_event(t.second, "backprojection"));
        float ms = 0;
        FDK_CUDA(cudaEventElapsedTime(&ms, t.first, t.second));
        h->kernel_ms += ms;
        h->free_timers.push_back(t);
    }
    h->timers.clear();
    return FDK_OK;
}

int take_timer(fdk_bp *h, std::pair<cudaEvent_t, cudaEvent_t> &t) {
    if (h->free_timers.empty()) {
        if (h->timers.size() >= 64) FDK_TRY(collect_timers(h));
    }
    if (!h->free_timers.empty()) {
        t = h->free_timers.back();
        h->free_timers.pop_back();
        return FDK_OK;
    }
    FDK_CUDA(cudaEventCreate(&t.first));
    FDK_CUDA(cudaEventCreate(&t.second));
    return FDK_OK;
}

// Backproject n views already resident on the device.
//   layout TRANSPOSED: f32 frames of proj_h rows x proj_w (the reference's BP input)
//   layout MIRROR: mirror pairs (f32x2 or f16x2 per precision), proj_h rows x proj_w pairs
//   band: -1 = every z band (the whole volume), else that band only (views counted with band 0;
//   kernels without bands run whole with band 0 and do nothing for the others)
// The largest-magnitude word (j: 0, 1 the list buffers, 2 the calls' buffer) and the accumulator
// scale of interpolation-layout buffer j.
unsigned int *lerp_absmax(fdk_bp *h, int j) { return h->d_absmax + 1 + j; }
float *lerp_scale(fdk_bp *h, int j) { return reinterpret_cast<float *>(h->d_absmax + 5 + j); }

// n_views MIRROR FP16 views at src -> the interpolation layout at dst (buffer j): their largest
// magnitude, then the scaled conversion, on st.
int convert_lerp(fdk_bp *h, const void *src, HalfLerp *dst, long long n_views, int j, const float *acc_scale,
                 cudaStream_t st) {
    FDK_CHECK_ARG(((uintptr_t)src & 15) == 0, "views must start on a 16-byte boundary");
    const long long rows = n_views * h->plan.nu;
    const long long pairs = rows * h->plan.nv;
    FDK_CUDA(cudaMemsetAsync(lerp_absmax(h, j), 0, sizeof(unsigned int), st));
    absmax_half2_kernel<<<(int)std::min<long long>(ceil_div(pairs / 4 + 1, 256), 148 * 8), 256, 0, st>>>(
        static_cast<const __half2 *>(src), pairs, lerp_absmax(h, j));
    FDK_CUDA(cudaGetLastError());
    to_lerp_kernel<<<(int)std::min<long long>(rows, 148 * 16), 256, 0, st>>>(
        static_cast<const __half2 *>(src), dst, rows, h->plan.nv, lerp_absmax(h, j), acc_scale, lerp_scale(h, j));
    FDK_CUDA(cudaGetLastError());
    h->launches += 2;
    return FDK_OK;
}

// The n MIRROR FP16 views of a BackProjectionFDK call converted to the interpolation layout on
// st (after the previous call's launches, which may have read the buffer on another stream);
// scale: the accumulator scale of the launches that read them.
int lerp_call_views(fdk_bp *h, const void *dev_proj, int n, cudaStream_t st, const float *acc_scale, HalfLerp **out,
                    const float **scale) {
    const long long frame = (long long)h->plan.nu * h->plan.nv;
    if (!h->lerp_call_ev) FDK_CUDA(cudaEventCreateWithFlags(&h->lerp_call_ev, cudaEventDisableTiming));
    if (h->lerp_call_cap < n) {
        if (h->lerp_call_used) FDK_TRY(wait_event(h->lerp_call_ev, "view conversion"));
        if (h->d_lerp_call) cudaFree(h->d_lerp_call);
        h->d_lerp_call = nullptr;
        h->lerp_call_cap = 0;
        FDK_CUDA(cudaMalloc(&h->d_lerp_call, sizeof(HalfLerp) * frame * n));
        h->lerp_call_cap = n;
    }
    if (h->lerp_call_used) FDK_CUDA(cudaStreamWaitEvent(st, h->lerp_call_ev, 0));
    FDK_TRY(convert_lerp(h, dev_proj, h->d_lerp_call, n, 2, acc_scale, st));
    *out = h->d_lerp_call;
    *scale = lerp_scale(h, 2);
    return FDK_OK;
}

int launch_bp(fdk_bp *h, const void *dev_proj, int layout, int transpose, const float *d_mats,
              const float *host_mats, int n, int width, int height, cudaStream_t st,
              const float *acc_scale = nullptr, int band = -1) {
    FDK_CHECK_ARG(band < h->n_bands, "band %d outside 0..%d", band, h->n_bands - 1);
    const int kb = band < 0 ? 0 : band, ke = band < 0 ? h->n_bands : band + 1;
    std::pair<cudaEvent_t, cudaEvent_t> tm;
    FDK_TRY(take_timer(h, tm));
    FDK_CUDA(cudaEventRecord(tm.first, st));
    if (h->precision == FDK_BP_FP32_EXACT) {
        FDK_CHECK_ARG(layout == FDK_LAYOUT_TRANSPOSED || layout == FDK_LAYOUT_ROWS,
                      "FP32_EXACT reads f32 frames (TRANSPOSED or ROWS layout)");
        BpExactArgs a;
        a.vol = h->d_vol;
        a.proj = (const float *)dev_proj;
        a.mats = d_mats;
        a.width = width;
        a.height = height;
        a.n_proj = n;
        a.x0 = (int)h->top.x;
        a.y0 = (int)h->top.y;
        a.z0 = (int)h->top.z;
        a.nxs = (int)h->top.width;
        a.nys = (int)h->top.height;
        a.nzz = h->sym ? (int)(h->D / 2) : (int)h->top.depth;
        a.D = h->D;
        a.transpose = transpose;
        const dim3 grid((unsigned)ceil_div(a.nzz, 32), (unsigned)ceil_div(a.nys, 8), a.nxs);
        if (kb == 0) {
            if (h->sym && transpose) bp_exact_kernel<true, true><<<grid, dim3(32, 8), 0, st>>>(a);
            else if (h->sym) bp_exact_kernel<true, false><<<grid, dim3(32, 8), 0, st>>>(a);
            else if (transpose) bp_exact_kernel<false, true><<<grid, dim3(32, 8), 0, st>>>(a);
            else bp_exact_kernel<false, false><<<grid, dim3(32, 8), 0, st>>>(a);
            FDK_CUDA(cudaGetLastError());
            h->launches++;
        }
        for (int k = kb; k < ke; k++) FDK_CUDA(cudaEventRecord(h->band_done[k], st));
    } else {
        FDK_CHECK_ARG(layout == FDK_LAYOUT_MIRROR, "fast backprojection reads the MIRROR layout");
        if (h->plan.tma_ok && ((uintptr_t)dev_proj & 15) == 0) {
            // MIXED: the views once in the interpolation layout, read by every band's launch
            HalfLerp *lv = nullptr;
            const float *lerp_sc = nullptr;
            if (h->precision == FDK_BP_MIXED) FDK_TRY(lerp_call_views(h, dev_proj, n, st, acc_scale, &lv, &lerp_sc));
            for (int k = kb; k < ke; k++) {
                if (lv)
                    FDK_TRY(bp_tma_launch<HalfLerp>(h->plan, h->d_vol, h->d_comp, lv, d_mats, host_mats, n, st,
                                                    lerp_sc, h->band_tz[k], h->band_tz[k + 1]));
                else
                    FDK_TRY(bp_tma_launch<float2>(h->plan, h->d_vol, h->d_comp, dev_proj, d_mats, host_mats, n, st,
                                                  acc_scale, h->band_tz[k], h->band_tz[k + 1]));
                h->launches++;
                FDK_CUDA(cudaEventRecord(h->band_done[k], st));
            }
            if (lv) {
                FDK_CUDA(cudaEventRecord(h->lerp_call_ev, st));
                h->lerp_call_used = true;
            }
        } else {
            const float ws = weight_scale(host_mats, h->top.x + 0.5f * (h->top.width - 1),
                                          h->top.y + 0.5f * (h->top.height - 1));
            if (kb == 0) {
                FDK_TRY(bp_fast_launch(h->plan, h->d_vol, h->d_comp, dev_proj, d_mats, n, st, ws, acc_scale));
                h->launches++;
            }
            for (int k = kb; k < ke; k++) FDK_CUDA(cudaEventRecord(h->band_done[k], st));
        }
    }
    FDK_CUDA(cudaEventRecord(tm.second, st));
    h->timers.push_back(tm);
    if (kb == 0) h->bp_count += n;
    return FDK_OK;
}

// The TMA kernel's bounded waits report through a device error word; read it (on the handle's
// stream, a bounded wait) once the kernels that may set it have finished.
int check_device_error(fdk_bp *h) {
    if (!h->plan.d_err) return FDK_OK;
    FDK_CUDA(cudaMemcpyAsync(h->h_err, h->plan.d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, h->stream));
    FDK_TRY(wait_stream(h->stream, h->sync_ev[2], "error word"));
    const unsigned int e = *h->h_err;
    if (e) {
        FDK_CUDA(cudaMemsetAsync(h->plan.d_err, 0, sizeof(e), h->stream));
        FDK_TRY(wait_stream(h->stream, h->sync_ev[2], "error word"));
        if (e & kErrTimeout)
            return fail(FDK_ERR_DEVICE_CHECK, "backprojection pipeline wait timed out on the device (error word %u)", e);
        return fail(FDK_ERR_DEVICE_CHECK, "backprojection: a tile footprint exceeded its shared-memory box and was "
                                          "skipped (error word %u)", e);
    }
    return FDK_OK;
}

// Volume -> host as [zs][y][x], band by band: each chunk of z planes waits only for the launch
// of its band (the band events of the latest batch), so the copies of the first bands overlap
// the backprojection of the later ones.  Two streams alternate over two staging buffers; the
// MIXED compensation is folded in on the way out (the device state keeps both terms).
int read_volume(fdk_bp *h, float *host) {
    const int nxs = (int)h->top.width, nys = (int)h->top.height;
    const long long plane = (long long)nxs * nys, D = h->D, dz = h->rb_planes;
    struct Range {
        long long z, n;
        int band;
    };
    std::vector<Range> ranges;
    if (h->n_bands == 1) {
        ranges.push_back({0, D, 0});
    } else {
        for (int k = 0; k < h->n_bands; k++) {
            const long long za = h->band_z[k], zb = h->band_z[k + 1];
            ranges.push_back({za, zb - za, k});          // top slices
            ranges.push_back({D - zb, zb - za, k});      // their mirrors in the bottom slab
        }
    }
    int waited[2] = {-1, -1};
    long long j = 0;
    for (const Range &r : ranges) {
        for (long long z = r.z; z < r.z + r.n; z += dz, j++) {
            const int q = (int)(j & 1);
            const cudaStream_t st = h->rb[q];
            if (waited[q] != r.band) {
                FDK_CUDA(cudaStreamWaitEvent(st, h->band_done[r.band], 0));
                waited[q] = r.band;
            }
            const int n = (int)std::min(dz, r.z + r.n - z);
            float *buf = h->d_rb + q * plane * dz;
            const long long tiles = ceil_div((long long)nxs, 32) * ceil_div((long long)n, 32) * nys;
            const int grid = (int)std::min<long long>(tiles, 148 * 32);
            if (h->d_comp)
                transform_volume_kernel<true><<<grid, 32, 0, st>>>(h->d_vol, h->d_comp, buf, nxs, nys, D, z, n);
            else
                transform_volume_kernel<false><<<grid, 32, 0, st>>>(h->d_vol, nullptr, buf, nxs, nys, D, z, n);
            FDK_CUDA(cudaGetLastError());
            FDK_CUDA(cudaMemcpyAsync(host + plane * z, buf, sizeof(float) * plane * n, cudaMemcpyDeviceToHost, st));
        }
    }
    FDK_TRY(wait_stream(h->rb[0], h->sync_ev[0], "volume readback"));
    FDK_TRY(wait_stream(h->rb[1], h->sync_ev[1], "volume readback"));
    return FDK_OK;
}

// z bands: up to kMaxBands launches per batch (FDK_BP_BANDS lowers the cap) when each still
// gives every CTA of the persistent grid at least 8 tiles (the split costs nothing measurable
// then).  Boundaries fall on whole `unit`s of slices: the staged kernel's tile height R, or a
// common multiple of it and the quarter-turn kernel's once that kernel is set up; each boundary
// is the whole unit nearest an even split of the slices.
void set_bands(fdk_bp *h, int unit) {
    const int R = h->precision == FDK_BP_MIXED ? TmaCfg<HalfLerp>::R : TmaCfg<float2>::R;
    const long long depth = (long long)h->top.depth;
    const long long cols = ceil_div((long long)h->top.width, 16) * ceil_div((long long)h->top.height, 16);
    const int tiles_z = (int)ceil_div(depth, R);
    const int units = (int)ceil_div(depth, unit);
    const char *cap = getenv("FDK_BP_BANDS");
    const int max_bands = cap ? std::max(1, std::min(kMaxBands, atoi(cap))) : kMaxBands;
    int nb = std::min(max_bands, units);
    while (nb > 1 && cols * (tiles_z / nb) < 8ll * h->plan.tma_ctas) nb--;
    h->n_bands = nb;
    for (int k = 0; k <= nb; k++) {
        h->band_z[k] = std::min<long long>((long long)k * units / nb * unit, depth);
        if (k > 0 && k < nb) h->band_z[k] = std::min<long long>((k * depth / nb + unit / 2) / unit * unit, depth);
        h->band_tz[k] = k == nb ? tiles_z : (int)(h->band_z[k] / R);
    }
    for (int k = 1; k <= nb; k++)  // rounding must leave no band empty
        if (h->band_z[k] <= h->band_z[k - 1]) {
            for (int j = 0; j <= nb; j++) {
                h->band_z[j] = std::min<long long>((long long)j * units / nb * unit, depth);
                h->band_tz[j] = j == nb ? tiles_z : (int)(h->band_z[j] / R);
            }
            break;
        }
}

// The fast kernels need circular-orbit matrices: rows 0 and 2 without a z term.
int check_circular(const float *mats, int n) {
    for (int i = 0; i < n; i++)
        FDK_CHECK_ARG(mats[12 * i + 2] == 0.0f && mats[12 * i + 10] == 0.0f,
                      "view %d: matrix rows 0/2 have a z term; the staged kernels need a circular orbit "
                      "(use FDK_BP_FP32_EXACT or the RTK entry point)", i);
    return FDK_OK;
}

}  // namespace bpi

using namespace bpi;


namespace {

// Quarter-turn symmetry of the scan (bp_sym.cuh): for every base view p < N/4 and k = 1..3, view
// p + kN/4 must put column T^k(x, y) where view p puts (x, y), within 1e-3 px, at test voxels
// spread over the grid; rot is the sign of T (see BpSymArgs::rot).  FP64 arithmetic on the FP32
// matrices the kernels use.
bool quarter_turn_holds(const float *mats, int n_proj, int n, int nz, int rot) {
    const int q = n_proj / 4;
    const int pts[6][3] = {{0, 0, 0}, {n - 1, 0, nz - 1}, {0, n - 1, nz / 2}, {n - 1, n - 1, 0},
                           {n / 3, (2 * n) / 3, nz / 3}, {n / 2, n / 5, nz - 1}};
    auto proj = [&](const float *m, double x, double y, double z, double &u, double &v) {
        const double w = (double)m[8] * x + (double)m[9] * y + (double)m[10] * z + (double)m[11];
        u = ((double)m[0] * x + (double)m[1] * y + (double)m[2] * z + (double)m[3]) / w;
        v = ((double)m[4] * x + (double)m[5] * y + (double)m[6] * z + (double)m[7]) / w;
    };
    for (int p = 0; p < q; p++)
        for (const auto &t : pts) {
            double u0, v0;
            proj(mats + 12 * (long long)p, t[0], t[1], t[2], u0, v0);
            int x = t[0], y = t[1];
            for (int k = 1; k < 4; k++) {
                const int nx_ = rot > 0 ? y : n - 1 - y, ny_ = rot > 0 ? n - 1 - x : x;
                x = nx_;
                y = ny_;
                double u, v;
                proj(mats + 12 * (long long)(p + k * q), x, y, t[2], u, v);
                if (!(std::fabs(u - u0) <= 1e-3 && std::fabs(v - v0) <= 1e-3)) return false;
            }
        }
    return true;
}

// Every staged tile (16 x 16 columns of the sub-box x R slices; the first and last z tiles of the
// top slab bound the rest, as in sym_footprints_fit) fits a BW x BH box in every checked view
// (all views, or 256 spread over the scan), by the producer's box rule (tile_box) in double with
// one element of slack for its FP32 rounding.  A footprint that does not fit is still
// backprojected, through global memory, so this only picks the faster box.
bool lerp_compact_fits(const float *mats, int n_proj, const BpFastPlan &p, int R, int BW, int BH) {
    const int tiles_x = (p.nxs + 15) / 16, tiles_y = (p.nys + 15) / 16;
    const int last = (int)((ceil_div(p.nzz, R) - 1) * R);
    const int step = std::max(1, n_proj / 256);
    for (int j = 0; j < n_proj; j += step) {
        const float *m = mats + 12 * (long long)j;
        for (int tx = 0; tx < tiles_x; tx++)
            for (int ty = 0; ty < tiles_y; ty++)
                for (int e = 0; e < 2; e++) {
                    const double xa = p.x0 + tx * 16, xb = p.x0 + std::min(tx * 16 + 16, p.nxs) - 1;
                    const double ya = p.y0 + ty * 16, yb = p.y0 + std::min(ty * 16 + 16, p.nys) - 1;
                    const double za = p.z0 + (e ? last : 0), zb = za + R - 1;
                    double umin = 1e300, umax = -1e300, vmin = 1e300, vmax = -1e300;
                    for (int c = 0; c < 4; c++) {
                        const double x = (c & 1) ? xb : xa, y = (c & 2) ? yb : ya;
                        const double rw = 1.0 / ((double)m[8] * x + (double)m[9] * y + (double)m[11]);
                        const double U = ((double)m[0] * x + (double)m[1] * y + (double)m[3]) * rw;
                        const double vw = (double)m[4] * x + (double)m[5] * y + (double)m[7];
                        const double va = ((double)m[6] * za + vw) * rw, vb = ((double)m[6] * zb + vw) * rw;
                        umin = std::min(umin, U);
                        umax = std::max(umax, U);
                        vmin = std::min(vmin, std::min(va, vb));
                        vmax = std::max(vmax, std::max(va, vb));
                    }
                    const double ulo = std::max(std::floor(umin) - 1, -1.0), uhi = std::min(std::floor(umax) + 2, (double)p.nu);
                    const double vlo = std::max(std::floor(vmin) - 1, -8.0), vhi = std::min(std::floor(vmax) + 2, p.nv + 4.0);
                    const long long v_lo = ((long long)vlo) & ~3ll;
                    if ((long long)uhi - (long long)ulo + 1 > BH - 1 || (long long)vhi - v_lo + 1 > BW - 1) return false;
                }
    }
    return true;
}

// Every tile of the quadrant (16 x 16 columns x R slices of the top slab [z0, z0 + nzz)) fits
// the kernel's BW x BH box in every view (each view is the base of a quadruple).  The map is linear-fractional, so a tile's
// extremes sit at its corner columns; the box's u extent (floor(umax) + 2 - (floor(umin) - 1) + 1)
// is below umax - umin + 5 and its v extent (the same with the start rounded down to 4 elements
// for the 16-byte rule) below vmax - vmin + 8, and vmax - vmin over a
// tile (a max minus a min of functions linear in the tile's first slice) is convex along z, so
// the first and last z tiles bound every z tile.
bool sym_footprints_fit(const float *mats, int n_proj, int n, int z0, int nzz, int R, int BW, int BH) {
    const int half = n / 2, tq = (half + 15) / 16;
    const int last = z0 + (int)((ceil_div(nzz, R) - 1) * R);
    for (int p = 0; p < n_proj; p++) {  // every view is the base of a quadruple
        const float *m = mats + 12 * (long long)p;
        for (int tx = 0; tx < tq; tx++)
            for (int ty = 0; ty < tq; ty++) {
                const double xa = tx * 16, xb = std::min(tx * 16 + 16, half) - 1;
                const double ya = ty * 16, yb = std::min(ty * 16 + 16, half) - 1;
                double umin = 1e300, umax = -1e300, spread = 0;
                double vlo[2] = {1e300, 1e300}, vhi[2] = {-1e300, -1e300};
                for (int c = 0; c < 4; c++) {
                    const double x = (c & 1) ? xb : xa, y = (c & 2) ? yb : ya;
                    const double w = (double)m[8] * x + (double)m[9] * y + (double)m[11];
                    const double U = ((double)m[0] * x + (double)m[1] * y + (double)m[3]) / w;
                    umin = std::min(umin, U);
                    umax = std::max(umax, U);
                    for (int e = 0; e < 2; e++) {
                        const double zs = e ? last : z0;
                        const double va = ((double)m[4] * x + (double)m[5] * y + (double)m[6] * zs + (double)m[7]) / w;
                        const double vb = va + (double)m[6] * (R - 1) / w;
                        vlo[e] = std::min(vlo[e], std::min(va, vb));
                        vhi[e] = std::max(vhi[e], std::max(va, vb));
                    }
                }
                for (int e = 0; e < 2; e++) spread = std::max(spread, vhi[e] - vlo[e]);
                if (umax - umin + 5.01 > BH || spread + 8.01 > BW) return false;
            }
    }
    return true;
}

}  // namespace

extern "C" {

int fdk_bp_create(fdk_bp **out, int32_t proj_width, int32_t proj_height, int32_t proj_count, int32_t nx, int32_t ny,
                  int32_t nz, const fdk_box *sub_top, const fdk_box *sub_bottom, int32_t precision, int32_t device) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(out && sub_top && sub_bottom, "NULL argument");
    *out = nullptr;
    FDK_CHECK_ARG(proj_width > 1 && proj_height > 1 && proj_count > 0 && proj_count <= 128,
                  "projection size/count out of range (count <= 128)");
    FDK_CHECK_ARG(nx > 0 && ny > 0 && nz > 0, "volume size must be positive");
    FDK_CHECK_ARG(precision >= FDK_BP_FP32_EXACT && precision <= FDK_BP_MIXED, "bad precision");
    const fdk_box t = *sub_top, b = *sub_bottom;
    FDK_CHECK_ARG(t.width > 0 && t.height > 0 && t.depth > 0, "empty top box");
    FDK_CHECK_ARG(precision == FDK_BP_FP32_EXACT || b.depth > 0,
                  "the staged backprojection kernels need the mirror slab pair (subBottom.depth > 0)");
    FDK_CHECK_ARG(t.x + t.width <= (uint64_t)nx && t.y + t.height <= (uint64_t)ny && t.z + t.depth <= (uint64_t)nz,
                  "top box outside the volume");
    const bool sym = b.depth > 0;
    if (sym) {
        // mirror-symmetric slab pair (backprojectionFDK.cu:171-173)
        FDK_CHECK_ARG(t.z + b.z + b.depth - 1 == (uint64_t)nz - 1, "subTop.MinZ + subBottom.MaxZ != nz - 1");
        FDK_CHECK_ARG(b.depth == t.depth, "mirror slabs must have equal depth");
        FDK_CHECK_ARG(b.x == t.x && b.y == t.y && b.width == t.width && b.height == t.height,
                      "mirror slabs must share their x/y extent");
    }
    DeviceGuard dg(device);
    FDK_TRY(dg.status);
    fdk_bp *h = new fdk_bp();
    h->device = device;
    h->precision = precision;
    h->proj_w = proj_width;
    h->proj_h = proj_height;
    h->proj_count = proj_count;
    h->nx = nx;
    h->ny = ny;
    h->nz = nz;
    h->top = t;
    h->bottom = b;
    h->sym = sym;
    h->D = (long long)t.depth + (sym ? b.depth : 0);
    const size_t nvox = (size_t)t.width * t.height * h->D;
    const size_t frame = (size_t)proj_width * proj_height;
    int s = FDK_OK;
    auto ck = [&](cudaError_t e, const char *what) {
        if (s == FDK_OK && e != cudaSuccess) s = cuda_status(e, what, __FILE__, __LINE__);
    };
    ck(cudaMalloc(&h->d_vol, sizeof(float) * nvox), "volume");
    for (int i = 0; i < 3 && s == FDK_OK; i++)
        ck(cudaEventCreateWithFlags(&h->sync_ev[i], cudaEventDisableTiming), "event");
    if (s == FDK_OK) ck(cudaHostAlloc((void **)&h->h_err, sizeof(unsigned int), 0), "error word");
    for (int i = 0; i < 2 && s == FDK_OK; i++) {
        ck(cudaMalloc(&h->d_stage[i], sizeof(float) * frame * proj_count), "view staging");
        ck(cudaEventCreateWithFlags(&h->copied[i], cudaEventDisableTiming), "event");
        ck(cudaEventCreateWithFlags(&h->consumed[i], cudaEventDisableTiming), "event");
    }
    if (s == FDK_OK) ck(cudaMalloc(&h->d_mats, sizeof(float) * 2 * 128 * 12), "matrices");
    if (s == FDK_OK) ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
    if (s == FDK_OK) ck(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking), "copy stream");
    if (s == FDK_OK) ck(cudaMemsetAsync(h->d_vol, 0, sizeof(float) * nvox, h->stream), "volume zero");
    if (s == FDK_OK && precision != FDK_BP_FP32_EXACT) {
        const size_t esz = precision == FDK_BP_MIXED ? sizeof(__half2) : sizeof(float2);
        ck(cudaMalloc(&h->d_mirror, esz * frame * proj_count), "mirror staging");
        if (s == FDK_OK && precision == FDK_BP_MIXED) {
            ck(cudaMalloc(&h->d_absmax, sizeof(unsigned int) * 8), "absmax");  // + the lerp words (lerp_word)
            ck(cudaMalloc(&h->d_comp, sizeof(float) * nvox), "compensation");
            if (s == FDK_OK) ck(cudaMemsetAsync(h->d_comp, 0, sizeof(float) * nvox, h->stream), "compensation zero");
        }
        if (s == FDK_OK)
            s = bp_fast_plan(h->plan, precision, proj_width, proj_height, (int)t.x, (int)t.y, (int)t.z,
                             (int)t.width, (int)t.height, (int)t.depth, h->D, device, h->stream);
        if (s == FDK_OK) {
            // The TMA kernel needs 16-byte row strides; FDK_BP_KERNEL=staged selects the
            // synchronous-staging kernel instead (kept for comparison and as the fallback).
            const char *sel = getenv("FDK_BP_KERNEL");
            h->plan.tma_ok = ((size_t)proj_width * esz) % 16 == 0 && !(sel && std::string(sel) == "staged");
            if (h->plan.tma_ok) {
                s = precision == FDK_BP_MIXED ? tma_prepare<HalfLerp>(h->plan.tma_ctas, device)
                                              : tma_prepare<float2>(h->plan.tma_ctas, device);
                if (s == FDK_OK && precision == FDK_BP_MIXED) {
                    int c = 0;
                    s = tma_prepare<HalfLerpCompact>(c, device);
                    h->lerp_compact_ok = s == FDK_OK && c == h->plan.tma_ctas;
                }
                if (s == FDK_OK) ck(cudaMalloc(&h->plan.d_err, sizeof(unsigned int)), "error word");
                if (s == FDK_OK) ck(cudaMemsetAsync(h->plan.d_err, 0, sizeof(unsigned int), h->stream), "error word");
                if (s == FDK_OK)
                    ck(cudaHostAlloc((void **)&h->h_list, sizeof(fdk_bp::ListRec) * fdk_bp::kListRing, 0), "view lists");
                if (s == FDK_OK)
                    ck(cudaMalloc(&h->d_list, sizeof(fdk_bp::ListRec) * fdk_bp::kListRing), "view lists");
                for (int i = 0; i < fdk_bp::kListRing && s == FDK_OK; i++)
                    ck(cudaEventCreateWithFlags(&h->list_ev[i], cudaEventDisableTiming), "event");
            }
        }
    }
    h->band_z[0] = 0;
    h->band_z[1] = (long long)t.depth;
    if (s == FDK_OK && h->plan.tma_ok && sym)
        set_bands(h, precision == FDK_BP_MIXED ? TmaCfg<HalfLerp>::R : TmaCfg<float2>::R);
    for (int k = 0; k < kMaxBands && s == FDK_OK; k++)
        ck(cudaEventCreateWithFlags(&h->band_done[k], cudaEventDisableTiming), "event");
    for (int i = 0; i < 2 && s == FDK_OK; i++)
        ck(cudaStreamCreateWithFlags(&h->rb[i], cudaStreamNonBlocking), "readback stream");
    if (s == FDK_OK) {
        // Load the kernels that run beside a backprojection now.  With lazy module loading (the
        // CUDA 12 default) a kernel's code is loaded at its first launch, and that load waits for
        // the device to go idle: a first readback issued beside the last batch waited for all of
        // its backprojection (measured: the volume returned 0.6 s after the last band instead of
        // overlapping the bands), and so would a first view conversion beside a batch.
        cudaFuncAttributes fa;
        const void *kernels[] = {(const void *)transform_volume_kernel<true>,
                                 (const void *)transform_volume_kernel<false>, (const void *)absmax_kernel,
                                 (const void *)to_mirror_half_kernel, (const void *)to_mirror_kernel<float2>,
                                 (const void *)fold_comp_kernel, (const void *)to_lerp_kernel,
                                 (const void *)absmax_half2_kernel};
        for (const void *kf : kernels)
            if (s == FDK_OK) ck(cudaFuncGetAttributes(&fa, kf), "kernel load");
    }
    if (s == FDK_OK) {
        // readback staging: two buffers of whole 32-plane tiles (32 planes, or about 128 MB where
        // planes are small), allocated here so that a readback never calls the allocator while
        // the last batch runs
        const long long plane = (long long)t.width * t.height;
        const long long want = std::max(32ll, (128ll << 20) / (plane * 4)) / 32 * 32;
        h->rb_planes = std::max(1ll, std::min(h->D, want));
        ck(cudaMalloc(&h->d_rb, sizeof(float) * 2 * plane * h->rb_planes), "readback staging");
    }
    // the zeroed volume, the error word and the scale are in place before any readback or launch
    // on another stream: a bounded wait for the handle's stream, not for the device
    if (s == FDK_OK) s = wait_stream(h->stream, h->sync_ev[0], "fdk_bp_create");
    if (s != FDK_OK) {
        fdk_bp_destroy(h);
        return s;
    }
    *out = h;
    return FDK_OK;
    FDK_ABI_END
}

int fdk_bp_bp(fdk_bp *h, int32_t transpose, const float *host_proj, int32_t width, int32_t height,
              const float *proj_mat, int32_t n_proj) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && host_proj && proj_mat, "NULL argument");
    FDK_CHECK_ARG(n_proj > 0 && n_proj <= h->proj_count, "n_proj %d outside 1..%d", n_proj, h->proj_count);
    FDK_CHECK_ARG((long long)width * height <= (long long)h->proj_w * h->proj_h && width > 1 && height > 1,
                  "view %dx%d larger than the handle's %dx%d", width, height, h->proj_w, h->proj_h);
    if (h->precision != FDK_BP_FP32_EXACT) {
        FDK_CHECK_ARG(transpose == 1 && width == h->proj_w && height == h->proj_h,
                      "fast precisions take the handle's transposed view size");
        FDK_TRY(check_circular(proj_mat, n_proj));
    }
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    const int k = h->slot;
    h->slot ^= 1;
    const size_t frame = (size_t)width * height;
    // staging slot k is free once the kernel that last read it has finished
    FDK_CUDA(cudaStreamWaitEvent(h->copy_stream, h->consumed[k], 0));
    FDK_CUDA(cudaMemcpyAsync(h->d_stage[k], host_proj, sizeof(float) * frame * n_proj, cudaMemcpyHostToDevice,
                             h->copy_stream));
    float *d_mats = h->d_mats + k * 128 * 12;
    FDK_CUDA(cudaMemcpyAsync(d_mats, proj_mat, sizeof(float) * 12 * n_proj, cudaMemcpyHostToDevice, h->copy_stream));
    FDK_CUDA(cudaEventRecord(h->copied[k], h->copy_stream));
    // The caller may reuse host_proj on return: wait for the copy (not for the kernel).
    FDK_TRY(wait_event(h->copied[k], "view copy"));
    FDK_CUDA(cudaStreamWaitEvent(h->stream, h->copied[k], 0));
    if (h->precision == FDK_BP_FP32_EXACT) {
        FDK_TRY(launch_bp(h, h->d_stage[k], transpose ? FDK_LAYOUT_TRANSPOSED : FDK_LAYOUT_ROWS, transpose, d_mats,
                          proj_mat, n_proj, width, height, h->stream));
    } else {
        const long long total = (long long)frame * n_proj;
        const int blocks = (int)std::min<long long>(ceil_div(total, 256), 148 * 16);
        const float *acc_scale = nullptr;
        if (h->precision == FDK_BP_MIXED) {
            FDK_CUDA(cudaMemsetAsync(h->d_absmax, 0, sizeof(unsigned int), h->stream));
            absmax_kernel<<<blocks, 256, 0, h->stream>>>(h->d_stage[k], total, h->d_absmax);
            to_mirror_half_kernel<<<blocks, 256, 0, h->stream>>>(h->d_stage[k], (__half2 *)h->d_mirror, width, height,
                                                                 n_proj, h->d_absmax, h->plan.d_scale);
            acc_scale = h->plan.d_scale;
            h->launches += 2;
        } else {
            to_mirror_kernel<float2><<<blocks, 256, 0, h->stream>>>(h->d_stage[k], (float2 *)h->d_mirror, width,
                                                                    height, n_proj);
            h->launches++;
        }
        FDK_CUDA(cudaGetLastError());
        FDK_TRY(launch_bp(h, h->d_mirror, FDK_LAYOUT_MIRROR, 1, d_mats, proj_mat, n_proj, width, height, h->stream,
                          acc_scale));
    }
    FDK_CUDA(cudaEventRecord(h->consumed[k], h->stream));
    return FDK_OK;
    FDK_ABI_END
}

int fdk_bp_bp_device(fdk_bp *h, const void *dev_proj, int32_t layout, const float *proj_mat, int32_t n_proj,
                     void *stream) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && dev_proj && proj_mat, "NULL argument");
    FDK_CHECK_ARG(n_proj > 0 && n_proj <= 128, "n_proj %d outside 1..128", n_proj);
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    cudaStream_t st = (cudaStream_t)stream;
    if (h->precision != FDK_BP_FP32_EXACT) FDK_TRY(check_circular(proj_mat, n_proj));
    const int k = h->slot;
    h->slot ^= 1;
    float *d_mats = h->d_mats + k * 128 * 12;
    FDK_CUDA(cudaStreamWaitEvent(st, h->consumed[k], 0));
    FDK_CUDA(cudaMemcpyAsync(d_mats, proj_mat, sizeof(float) * 12 * n_proj, cudaMemcpyHostToDevice, st));
    // the matrices come from pageable host memory: the async copy completes before returning
    FDK_TRY(launch_bp(h, dev_proj, layout, 1, d_mats, proj_mat, n_proj, h->proj_w, h->proj_h, st,
                      h->precision == FDK_BP_MIXED ? h->ext_scale : nullptr));
    FDK_CUDA(cudaEventRecord(h->consumed[k], st));
    return FDK_OK;
    FDK_ABI_END
}

int fdk_bp_get_volume(fdk_bp *h, float *host_vol, int64_t size) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && host_vol, "NULL argument");
    const long long nvox = (long long)h->top.width * h->top.height * h->D;
    FDK_CHECK_ARG(size >= nvox, "size %lld < %lld voxels", (long long)size, nvox);
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    FDK_TRY(read_volume(h, host_vol));
    return check_device_error(h);
    FDK_ABI_END
}

int fdk_bp_volume_device(fdk_bp *h, float **dev_vol, int64_t *count) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(h && dev_vol && count, "NULL argument");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    FDK_TRY(collect_timers(h));  // every launch of the handle has finished (bounded waits)
    FDK_TRY(check_device_error(h));
    const long long nvox = (long long)h->top.width * h->top.height * h->D;
    if (h->d_comp) FDK_TRY(bp_fast_fold_compensation(h->d_vol, h->d_comp, nvox, h->stream));
    FDK_TRY(wait_stream(h->stream, h->sync_ev[0], "fdk_bp_volume_device"));
    *dev_vol = h->d_vol;
    *count = nvox;
    return FDK_OK;
    FDK_ABI_END
}

int fdk_bp_sample(fdk_bp *h, const int32_t *host_xyz, int64_t n, float *host_out) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && host_xyz && host_out && n >= 0, "NULL argument or negative count");
    if (n == 0) return FDK_OK;
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    FDK_TRY(collect_timers(h));  // every launch of the handle has finished (bounded waits)
    FDK_TRY(check_device_error(h));
    int *d_xyz = nullptr;
    float *d_out = nullptr;
    int s = cuda_status(cudaMalloc(&d_xyz, sizeof(int) * 3 * n), "sample indices", __FILE__, __LINE__);
    if (s == FDK_OK) s = cuda_status(cudaMalloc(&d_out, sizeof(float) * n), "sample values", __FILE__, __LINE__);
    if (s == FDK_OK)
        s = cuda_status(cudaMemcpyAsync(d_xyz, host_xyz, sizeof(int) * 3 * n, cudaMemcpyHostToDevice, h->stream),
                        "sample indices", __FILE__, __LINE__);
    if (s == FDK_OK) {
        const int grid = (int)std::min<long long>(ceil_div(n, 256), 148 * 8);
        sample_voxels_kernel<<<grid, 256, 0, h->stream>>>(
            h->d_vol, h->d_comp, d_xyz, n, d_out, (int)h->top.x, (int)h->top.y, (int)h->top.width,
            (int)h->top.height, (long long)h->top.z, (long long)h->top.depth, (long long)h->bottom.z,
            h->sym ? (long long)h->bottom.depth : 0ll, h->D);
        s = cuda_status(cudaGetLastError(), "sample kernel", __FILE__, __LINE__);
    }
    if (s == FDK_OK)
        s = cuda_status(cudaMemcpyAsync(host_out, d_out, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream),
                        "sample values", __FILE__, __LINE__);
    if (s == FDK_OK) s = wait_stream(h->stream, h->sync_ev[0], "fdk_bp_sample");
    cudaStreamSynchronize(h->stream);  // error paths: the buffers are freed below
    cudaFree(d_xyz);
    cudaFree(d_out);
    return s;
    FDK_ABI_END
}

int fdk_bp_stats(fdk_bp *h, int64_t *bp_count, double *kernel_ms) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(h != nullptr, "NULL handle");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    FDK_TRY(collect_timers(h));
    FDK_TRY(check_device_error(h));
    if (bp_count) *bp_count = h->bp_count;
    if (kernel_ms) *kernel_ms = h->kernel_ms;
    return FDK_OK;
    FDK_ABI_END
}

int fdk_bp_reset(fdk_bp *h) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(h != nullptr, "NULL handle");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    FDK_TRY(collect_timers(h));  // every launch of the handle has finished (bounded waits)
    const size_t nvox = (size_t)h->top.width * h->top.height * h->D;
    FDK_CUDA(cudaMemsetAsync(h->d_vol, 0, sizeof(float) * nvox, h->stream));
    if (h->d_comp) FDK_CUDA(cudaMemsetAsync(h->d_comp, 0, sizeof(float) * nvox, h->stream));
    // zeroed before the next launch or readback on another stream
    FDK_TRY(wait_stream(h->stream, h->sync_ev[0], "fdk_bp_reset"));
    h->bp_count = 0;
    h->kernel_ms = 0;
    h->launches = 0;
    return FDK_OK;
    FDK_ABI_END
}

int fdk_bp_destroy(fdk_bp *h) {
    if (!h) return FDK_OK;
    {
        DeviceGuard dg(h->device);
        if (h->stream) cudaStreamSynchronize(h->stream);
        if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
        for (auto &t : h->timers) {
            cudaEventDestroy(t.first);
            cudaEventDestroy(t.second);
        }
        for (auto &t : h->free_timers) {
            cudaEventDestroy(t.first);
            cudaEventDestroy(t.second);
        }
        for (int i = 0; i < 2; i++) {
            if (h->d_stage[i]) cudaFree(h->d_stage[i]);
            if (h->copied[i]) cudaEventDestroy(h->copied[i]);
            if (h->consumed[i]) cudaEventDestroy(h->consumed[i]);
        }
        if (h->d_mirror) cudaFree(h->d_mirror);
        if (h->d_vol) cudaFree(h->d_vol);
        if (h->d_comp) cudaFree(h->d_comp);
        if (h->d_mats) cudaFree(h->d_mats);
        if (h->d_absmax) cudaFree(h->d_absmax);
        bp_fast_release(h->plan);
        for (int k = 0; k < kMaxBands; k++)
            if (h->band_done[k]) cudaEventDestroy(h->band_done[k]);
        for (int i = 0; i < 2; i++)
            if (h->rb[i]) {
                cudaStreamSynchronize(h->rb[i]);
                cudaStreamDestroy(h->rb[i]);
            }
        if (h->d_rb) cudaFree(h->d_rb);
        for (int i = 0; i < fdk_bp::kListRing; i++)
            if (h->list_ev[i]) {
                if (h->list_used[i]) wait_event(h->list_ev[i], "view list");  // its upload has been read
                cudaEventDestroy(h->list_ev[i]);
            }
        if (h->h_list) cudaFreeHost(h->h_list);
        for (int i = 0; i < 2; i++)
            if (h->d_lerp[i]) cudaFree(h->d_lerp[i]);
        if (h->lerp_call_ev) {
            if (h->lerp_call_used) wait_event(h->lerp_call_ev, "view conversion");
            cudaEventDestroy(h->lerp_call_ev);
        }
        if (h->d_lerp_call) cudaFree(h->d_lerp_call);
        if (h->d_list) cudaFree(h->d_list);
        for (int i = 0; i < 3; i++)
            if (h->sync_ev[i]) cudaEventDestroy(h->sync_ev[i]);
        if (h->h_err) cudaFreeHost(h->h_err);
        if (h->stream) cudaStreamDestroy(h->stream);
        if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    }
    delete h;
    return FDK_OK;
}

}  // extern "C"

// Kernel launches of the handle since creation or the last reset (internal: recon.cu).
long long fdk_bp_launches_internal(const fdk_bp *h) { return h ? h->launches : 0; }

// Two interpolation-layout buffers of n_slots MIXED views each for fdk_bp_bp_lists_internal
// (the held and the filling batch), allocated once, before the first launch.  Internal to the
// library (recon.cu).
int fdk_bp_reserve_lerp_internal(fdk_bp *h, int n_slots) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(h && n_slots > 0, "NULL handle or no views");
    if (h->precision != FDK_BP_MIXED || !h->plan.tma_ok || h->lerp_slots >= n_slots) return FDK_OK;
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    FDK_TRY(collect_timers(h));  // no launch may still read the old buffers
    const long long frame = (long long)h->plan.nu * h->plan.nv;
    for (int i = 0; i < 2; i++) {
        if (h->d_lerp[i]) cudaFree(h->d_lerp[i]);
        h->d_lerp[i] = nullptr;
        h->lerp_src[i] = nullptr;
    }
    h->lerp_slots = 0;
    for (int i = 0; i < 2; i++)
        FDK_CUDA(cudaMalloc(&h->d_lerp[i], sizeof(HalfLerp) * frame * n_slots));
    h->lerp_slots = n_slots;
    return FDK_OK;
    FDK_ABI_END
}

// The reconstructor's scan (every view's matrix): MIXED list launches read through the compact
// boxes when every tile fits them (lerp_compact_fits).  Before the first launch.  Internal to the
// library (recon.cu).
int fdk_bp_choose_lerp_box_internal(fdk_bp *h, const float *mats, int n_proj) {
    FDK_CHECK_ARG(h && mats && n_proj > 0, "NULL argument or no views");
    h->lerp_compact = false;
    if (h->precision != FDK_BP_MIXED || !h->plan.tma_ok || !h->lerp_compact_ok || h->launches > 0) return FDK_OK;
    if (check_circular(mats, n_proj) != FDK_OK) {
        clear_error();
        return FDK_OK;
    }
    using C = TmaCfg<HalfLerpCompact>;
    h->lerp_compact = lerp_compact_fits(mats, n_proj, h->plan, C::R, C::BW, C::BH);
    return FDK_OK;
}

// Device scalar multiplying the MIXED accumulators of device-resident FP16 views (their
// producer divided the filtered values by it).  Internal to the library (recon.cu).
int fdk_bp_set_acc_scale_internal(fdk_bp *h, const float *d_scale) {
    if (!h) return FDK_ERR_INVALID_ARG;
    h->ext_scale = d_scale;
    return FDK_OK;
}

// Backprojection of device-resident views with device-resident matrices, for the
// reconstructor (recon.cu): no host round trip per batch, so consecutive batches queue on the
// stream without the host waiting for the GPU.  band: -1 = the whole volume, else one z band
// (0 .. fdk_bp_band_count_internal - 1).  Internal to the library.
int fdk_bp_bp_device_mats_internal(fdk_bp *h, const void *dev_proj, int32_t layout, const float *dev_mats,
                                   int32_t n_proj, const float *host_mats, void *stream, int32_t band) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(h && dev_proj && dev_mats && host_mats, "NULL argument");
    FDK_CHECK_ARG(n_proj > 0 && n_proj <= 512, "n_proj %d outside 1..512", n_proj);
    if (h->precision != FDK_BP_FP32_EXACT) FDK_TRY(check_circular(host_mats, n_proj));
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    return launch_bp(h, dev_proj, layout, 1, dev_mats, host_mats, n_proj, h->proj_w, h->proj_h,
                     (cudaStream_t)stream, h->precision == FDK_BP_MIXED ? h->ext_scale : nullptr, band);
    FDK_ABI_END
}

// The staged kernels' device error word (bounded waits that ran out), read and cleared after
// the handle's launches have finished.  Internal to the library (recon.cu).
int fdk_bp_check_internal(fdk_bp *h) {
    if (!h) return FDK_ERR_INVALID_ARG;
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    FDK_TRY(collect_timers(h));
    return check_device_error(h);
}

// z bands of a batch (1 where the kernel has none).  Internal to the library (recon.cu).
int fdk_bp_band_count_internal(const fdk_bp *h) { return h ? h->n_bands : 1; }

// Quarter-turn kernel set-up for device-resident batches (recon.cu): returns in *rot the column
// map of the scan's quarter-turn symmetry, or 0 where the kernel does not apply (FP32_EXACT, not
// the whole square grid, n_proj % 4 != 0, matrices without the symmetry, a footprint larger
// than the box), or is not chosen (MIXED unless FDK_BP_SYM=1; FDK_BP_SYM=0 for every
// precision).  mats: all n_proj views' matrices (host).  Internal.
int fdk_bp_sym_setup_internal(fdk_bp *h, const float *mats, int n_proj, int *rot) {
    FDK_CHECK_ARG(h && mats && rot, "NULL argument");
    *rot = 0;
    h->sym_rot = 0;
    // FDK_BP_SYM: unset = FP32 only (where it measured faster), 1 = FP32 and MIXED, 0 = off
    const char *env = getenv("FDK_BP_SYM");
    const std::string mode = env ? env : "";
    if (mode == "0") return FDK_OK;
    if (h->precision == FDK_BP_FP32_EXACT || !h->plan.tma_ok || !h->sym) return FDK_OK;
    if (h->precision == FDK_BP_MIXED && mode != "1") return FDK_OK;
    // the set-up moves the z band boundaries: only before the first launch (or after a reset),
    // so that no readback waits on a band event of launches over the old boundaries
    if (h->launches > 0) return FDK_OK;
    const BpFastPlan &p = h->plan;
    if (p.x0 != 0 || p.y0 != 0 || p.nxs != p.nys || p.nxs != h->nx || h->nx != h->ny || (p.nxs & 1) || n_proj % 4)
        return FDK_OK;
    if (check_circular(mats, n_proj) != FDK_OK) {
        clear_error();
        return FDK_OK;
    }
    int r = 0;
    for (int cand : {1, -1})
        if (quarter_turn_holds(mats, n_proj, h->nx, h->nz, cand)) {
            r = cand;
            break;
        }
    if (!r) return FDK_OK;
    const bool mixed = h->precision == FDK_BP_MIXED;
    // MIXED pairs views over the interpolation layout (8-byte elements)
    const int R = mixed ? SymCfg<HalfLerp>::R : SymCfg<float2>::R;
    const int BW = mixed ? SymCfg<HalfLerp>::BW : SymCfg<float2>::BW;
    const int BH = mixed ? SymCfg<HalfLerp>::BH : SymCfg<float2>::BH;
    if (!sym_footprints_fit(mats, n_proj, h->nx, p.z0, p.nzz, R, BW, BH)) return FDK_OK;
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    FDK_TRY(mixed ? sym_prepare<HalfLerp>(h->sym_ctas, h->device) : sym_prepare<float2>(h->sym_ctas, h->device));
    // bands on whole tiles of both kernels (set up before the first launch)
    const int Rt = mixed ? TmaCfg<HalfLerp>::R : TmaCfg<float2>::R;
    int unit = Rt;
    while (unit % R) unit += Rt;
    set_bands(h, unit);
    h->sym_rot = r;
    *rot = r;
    return FDK_OK;
}

namespace {
// The interpolation-layout copy of slots 0..n_slots-1 of a MIXED views buffer: converted on st
// when the first (or only) band of a batch is launched (band <= 0), reused by its later bands;
// scale: the accumulator scale of the launches that read it (acc_scale times the copy's 2^k).
int lerp_views(fdk_bp *h, const void *views, int n_slots, int band, cudaStream_t st, const float *acc_scale,
               HalfLerp **out, const float **scale) {
    FDK_CHECK_ARG(h->lerp_slots >= n_slots, "interpolation-layout buffers of %lld views for a batch of %d",
                  h->lerp_slots, n_slots);
    int j = h->lerp_src[0] == views ? 0 : h->lerp_src[1] == views ? 1 : -1;
    if (j < 0 || band <= 0) {
        if (j < 0) {
            j = h->lerp_next;
            h->lerp_next ^= 1;
        }
        FDK_TRY(convert_lerp(h, views, h->d_lerp[j], n_slots, j, acc_scale, st));
        h->lerp_src[j] = views;
    }
    *out = h->d_lerp[j];
    *scale = lerp_scale(h, j);
    return FDK_OK;
}

// The next entry of the handle's list ring, once the launch that last read it has finished (a
// bounded wait; immediate unless the host runs kListRing launches ahead of the device).
int take_list(fdk_bp *h, fdk_bp::ListRec **rec, fdk_bp::ListRec **dev, int *entry) {
    FDK_CHECK_ARG(h->h_list && h->d_list, "no view-list ring (staged precisions only)");
    const int i = h->list_next;
    h->list_next = (i + 1) % fdk_bp::kListRing;
    if (h->list_used[i]) FDK_TRY(wait_event(h->list_ev[i], "view list"));
    h->list_used[i] = false;
    *rec = h->h_list + i;
    *dev = h->d_list + i;
    *entry = i;
    return FDK_OK;
}
// Entry i is busy until the work queued on st so far (its upload and launch) has finished.
int release_list(fdk_bp *h, int i, cudaStream_t st) {
    FDK_CUDA(cudaEventRecord(h->list_ev[i], st));
    h->list_used[i] = true;
    return FDK_OK;
}
}  // namespace

// One batch of views held in a device views buffer (n_slots views, any order), for the
// reconstructor (recon.cu): `n_single` views by (slot, view) through the staged kernel and
// `n_quad` quarter-turn quadruples (4 slots each, members b, b + N/4, b + N/2, b + 3N/4 mod N, and
// the base view b; one per view of each whole orbit) through the quarter-turn kernel.  d_mats / host_mats: every view's matrix.
// band: -1 = every z band, else one.  Internal to the library.
int fdk_bp_bp_lists_internal(fdk_bp *h, const void *views, int n_slots, const float *d_mats, const float *host_mats,
                             const int *s_slot, const int *s_view, int n_single, const int *q_slot,
                             const int *q_view, int n_quad, void *stream, int band) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(h && views && d_mats && host_mats, "NULL argument");
    FDK_CHECK_ARG(h->precision != FDK_BP_FP32_EXACT && h->plan.tma_ok, "view lists need a staged precision (TMA)");
    FDK_CHECK_ARG(n_single >= 0 && n_quad >= 0 && n_single + 4 * n_quad > 0, "empty batch");
    FDK_CHECK_ARG(n_quad == 0 || h->sym_rot != 0, "quadruples without the quarter-turn set-up");
    FDK_CHECK_ARG(band < h->n_bands, "band %d outside 0..%d", band, h->n_bands - 1);
    FDK_CHECK_ARG(((uintptr_t)views & 15) == 0, "TMA views must start on a 16-byte boundary");
    for (int i = 0; i < n_single; i++) FDK_TRY(check_circular(host_mats + 12 * (long long)s_view[i], 1));
    for (int i = 0; i < n_quad; i++) FDK_TRY(check_circular(host_mats + 12 * (long long)q_view[i], 1));
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    cudaStream_t st = (cudaStream_t)stream;
    const bool mixed = h->precision == FDK_BP_MIXED;
    const float *acc_scale = mixed ? h->ext_scale : nullptr;
    const int kb = band < 0 ? 0 : band, ke = band < 0 ? h->n_bands : band + 1;
    std::pair<cudaEvent_t, cudaEvent_t> tm;
    FDK_TRY(take_timer(h, tm));
    FDK_CUDA(cudaEventRecord(tm.first, st));
    HalfLerp *lv = nullptr;
    const float *lerp_sc = nullptr;  // accumulator scale of the launches that read lv
    if (mixed) {
        int used = 0;  // slots the launches read (a partial batch converts only its own)
        for (int i = 0; i < n_single; i++) used = std::max(used, s_slot[i] + 1);
        for (int i = 0; i < 4 * n_quad; i++) used = std::max(used, q_slot[i] + 1);
        FDK_CHECK_ARG(used <= n_slots, "slot outside the views buffer");
        FDK_TRY(lerp_views(h, views, used, band, st, acc_scale, &lv, &lerp_sc));
    }
    for (int k = kb; k < ke; k++) {
        for (int q0 = 0; q0 < n_quad; q0 += kSymMaxQuads) {
            const int nq = std::min(kSymMaxQuads, n_quad - q0);
            fdk_bp::ListRec *rec = nullptr, *dev = nullptr;
            int e = 0;
            FDK_TRY(take_list(h, &rec, &dev, &e));
            SymQuads &sq = rec->quads;
            for (int i = 0; i < nq; i++) {
                const int *s4 = q_slot + 4 * (q0 + i);
                sq.slot[i] = make_int4(s4[0], s4[1], s4[2], s4[3]);
                sq.view[i] = q_view[q0 + i];
            }
            FDK_CUDA(cudaMemcpyAsync(dev, rec, sizeof(SymQuads), cudaMemcpyHostToDevice, st));
            const int r = mixed ? bp_sym_launch<HalfLerp>(h->plan, h->sym_ctas, h->d_vol, h->d_comp, lv, n_slots,
                                                          d_mats, host_mats, sq, &dev->quads, nq, h->sym_rot, st,
                                                          lerp_sc, h->band_z[k], h->band_z[k + 1])
                                : bp_sym_launch<float2>(h->plan, h->sym_ctas, h->d_vol, h->d_comp, views, n_slots,
                                                        d_mats, host_mats, sq, &dev->quads, nq, h->sym_rot, st,
                                                        acc_scale, h->band_z[k], h->band_z[k + 1]);
            FDK_TRY(release_list(h, e, st));
            FDK_TRY(r);
            h->launches++;
        }
        for (int s0 = 0; s0 < n_single; s0 += kMaxListViews) {
            const int ns = std::min(kMaxListViews, n_single - s0);
            bool run = s_slot[s0] >= 0 && s_slot[s0] + ns <= n_slots;
            for (int i = 1; i < ns && run; i++)
                run = s_slot[s0 + i] == s_slot[s0] + i && s_view[s0 + i] == s_view[s0] + i;
            if (run) {
                // consecutive views in consecutive slots: a launch without a list, over the
                // buffer from the run's first slot (the kernel's loop then reads no list)
                const size_t esz = lv ? sizeof(HalfLerp) : mixed ? sizeof(__half2) : sizeof(float2);
                const size_t frame = (size_t)h->plan.nu * h->plan.nv * esz;
                const void *pv = static_cast<const char *>(lv ? (const void *)lv : views) + frame * s_slot[s0];
                const long long m0 = 12 * (long long)s_view[s0];
                FDK_TRY(lv && h->lerp_compact
                            ? bp_tma_launch<HalfLerpCompact>(h->plan, h->d_vol, h->d_comp, pv, d_mats + m0,
                                                             host_mats + m0, ns, st, lerp_sc, h->band_tz[k],
                                                             h->band_tz[k + 1])
                        : lv ? bp_tma_launch<HalfLerp>(h->plan, h->d_vol, h->d_comp, pv, d_mats + m0, host_mats + m0,
                                                     ns, st, lerp_sc, h->band_tz[k], h->band_tz[k + 1])
                        : bp_tma_launch<float2>(h->plan, h->d_vol, h->d_comp, pv, d_mats + m0, host_mats + m0, ns,
                                                st, acc_scale, h->band_tz[k], h->band_tz[k + 1]));
                h->launches++;
                continue;
            }
            fdk_bp::ListRec *rec = nullptr, *dev = nullptr;
            int e = 0;
            FDK_TRY(take_list(h, &rec, &dev, &e));
            ViewList &vl = rec->views;
            vl.n = ns;
            for (int i = 0; i < ns; i++) {
                vl.slot[i] = s_slot[s0 + i];
                vl.view[i] = s_view[s0 + i];
            }
            FDK_CUDA(cudaMemcpyAsync(dev, rec, sizeof(ViewList), cudaMemcpyHostToDevice, st));
            const int r = lv && h->lerp_compact
                              ? bp_tma_launch<HalfLerpCompact>(h->plan, h->d_vol, h->d_comp, lv, d_mats, host_mats, ns,
                                                               st, lerp_sc, h->band_tz[k], h->band_tz[k + 1], &vl,
                                                               &dev->views, n_slots)
                          : lv ? bp_tma_launch<HalfLerp>(h->plan, h->d_vol, h->d_comp, lv, d_mats, host_mats, ns, st,
                                                       lerp_sc, h->band_tz[k], h->band_tz[k + 1], &vl, &dev->views,
                                                       n_slots)
                          : bp_tma_launch<float2>(h->plan, h->d_vol, h->d_comp, views, d_mats, host_mats, ns, st,
                                                  acc_scale, h->band_tz[k], h->band_tz[k + 1], &vl, &dev->views, n_slots);
            FDK_TRY(release_list(h, e, st));
            FDK_TRY(r);
            h->launches++;
        }
        FDK_CUDA(cudaEventRecord(h->band_done[k], st));
    }
    FDK_CUDA(cudaEventRecord(tm.second, st));
    h->timers.push_back(tm);
    if (kb == 0) h->bp_count += n_single + n_quad;  // one quadruple per view of a whole orbit
    return FDK_OK;
    FDK_ABI_END
}
