// rtk.cu -- the RTK-style backprojection drop-in, CUDA_reconstruct_conebeam
// (cudaBP/rtkCudaFDKBackProjectionImageFilter.cu:200-330, kernel_fdk_3Dgrid :156-191,
// RtkSUBPIXEL :83-112).
//
// General 3x4 geometry: every voxel evaluates its own projection for every view (no
// circular-orbit shortcut), so tilted or non-circular trajectories are handled.
// vol_out = vol_in + sum_p bilinear(proj_p; u, v) / w^2, x fastest; a sample is zero outside
// [0, W-1) x [0, H-1).  Two kernels with the same arithmetic (bit-identical results):
//
//  * rtk_tma_kernel (default): persistent CTAs walk 16 x 16 column x 8 slice tiles.  A producer
//    warp projects each tile's 8 corners per view (a linear-fractional map takes its extremes
//    there), and one lane loads the footprint box of every view of a chunk into shared memory
//    with TMA (cp.async.bulk.tensor, mbarrier ring) -- the staging of the circular-orbit
//    kernel, for the general matrix.  Views whose box does not fit fall back to global gathers;
//    views whose box misses the detector are skipped.
//  * rtk_bp_kernel: the same gathers through L1 (__ldg).  Used where TMA cannot address the
//    views (width not a multiple of 4 floats, base not 16-byte aligned) or when the environment
//    sets FDK_RTK_KERNEL=l1.
#include <string>

#include "common.h"
#include "tma_common.cuh"

namespace fdk {

constexpr int kRtkMaxViews = 128;
struct RtkMats {  // by value in the kernel parameters: no device copy per call
    float m[kRtkMaxViews * 12];
};

constexpr int kRtkR = 8;  // consecutive z voxels per thread

// Thread = voxel column (i, j), a run of kRtkR voxels along z.  Per view the x, y and w rows of
// the matrix are evaluated once at z = 0 for the column; each voxel of the run adds its m[.][2] z
// term with one FMA per row.  Four __ldg texels per sample, bilinear in FP32, zero outside
// [0, W-1) x [0, H-1) (RtkSUBPIXEL), weight 1/w^2.
__global__ void __launch_bounds__(256) rtk_bp_kernel(const float *__restrict__ vol_in, float *__restrict__ vol_out,
                                                     const float *__restrict__ proj, const __grid_constant__ RtkMats mats,
                                                     int W, int H, int n, int nx, int ny, int nz) {
    __shared__ float sm[kRtkMaxViews * 12];
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int q = tid; q < n * 12; q += 256) sm[q] = mats.m[q];
    __syncthreads();
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int k0 = blockIdx.z * kRtkR;
    if (i >= nx || j >= ny) return;
    const float fi = (float)i, fj = (float)j;
    const float wm1 = (float)(W - 1), hm1 = (float)(H - 1);
    const long long frame = (long long)W * H;
    float acc[kRtkR];
#pragma unroll
    for (int kk = 0; kk < kRtkR; kk++) acc[kk] = 0.f;
    for (int p = 0; p < n; p++) {
        const float *m = sm + 12 * p;
        const float X = fmaf(m[0], fi, fmaf(m[1], fj, m[3]));
        const float Y = fmaf(m[4], fi, fmaf(m[5], fj, m[7]));
        const float Z = fmaf(m[8], fi, fmaf(m[9], fj, m[11]));
        const float *pv = proj + p * frame;
#pragma unroll
        for (int kk = 0; kk < kRtkR; kk++) {
            const float fk = (float)(k0 + kk);
            const float rw = __fdividef(1.0f, fmaf(m[10], fk, Z));
            const float u = fmaf(m[2], fk, X) * rw, v = fmaf(m[6], fk, Y) * rw;
            float s = 0.f;
            if (u >= 0.f && u < wm1 && v >= 0.f && v < hm1) {
                const float iu = floorf(u), iv = floorf(v);
                const float du = u - iu, dv = v - iv;
                const float *p0 = pv + (long long)iv * W + (int)iu;
                const float *p1 = p0 + W;
                const float a = fmaf(du, __ldg(p0 + 1) - __ldg(p0), __ldg(p0));
                const float b = fmaf(du, __ldg(p1 + 1) - __ldg(p1), __ldg(p1));
                s = fmaf(dv, b - a, a);
            }
            acc[kk] = fmaf(s * rw, rw, acc[kk]);
        }
    }
#pragma unroll
    for (int kk = 0; kk < kRtkR; kk++) {
        const int k = k0 + kk;
        if (k >= nz) break;
        const long long idx = i + ((long long)j + (long long)k * ny) * nx;
        vol_out[idx] = vol_in[idx] + acc[kk];
    }
}

// ---------------------------------------------------------------------------------------
// TMA-staged kernel

namespace rtkt {
constexpr int TX = 16, TY = 16;  // voxel columns per tile (x, y)
constexpr int R = kRtkR;         // slices per thread
constexpr int BW = 40;           // box width: u elements (160-byte rows; TMA x multiple of 4)
constexpr int BH = 24;           // box height: v rows
constexpr int NV = 8;            // views per stage
constexpr int S = 2;             // stages
constexpr int BOX = BW * BH * 4;  // 3840 bytes, a multiple of 128
constexpr int THREADS = TX * TY + 32;
constexpr int kStaged = 1;    // the box holds every sample of the tile
constexpr int kSkip = 2;      // no voxel of the tile projects inside the detector
constexpr int kInterior = 4;  // every voxel projects inside [0, W-1) x [0, H-1): no bounds checks
constexpr int kZFree = 8;     // m[2] = m[10] = 0: u and w do not depend on z (circular orbit)
struct Meta {
    int u_lo, v_lo;
    int flags;
    int pad;
};
constexpr int SMEM = S * NV * BOX + S * NV * (int)sizeof(Meta) + kRtkMaxViews * 12 * 4 + 2 * S * 8;
struct Args {
    const float *vol_in;
    float *vol_out;
    const float *proj;
    int W, H, n, nx, ny, nz;
    int tiles_x, tiles_y, tiles_z;
};
}  // namespace rtkt

// Device error word of the staged kernel (bounded waits that ran out); read and cleared by
// the synchronous entry points.
static __device__ unsigned int g_rtk_err;

// Footprint of a tile in one view: the 8 corners' projections, with the voxel arithmetic of the
// gathers; one element of margin absorbs FP32 differences between corners and inner voxels.
__device__ __forceinline__ void rtk_tile_box(const float *m, float xa, float xb, float ya, float yb, float za,
                                             float zb, int W, int H, rtkt::Meta &md) {
    using namespace rtkt;
    float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f;
    bool front = true;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const float x = (c & 1) ? xb : xa, y = (c & 2) ? yb : ya, z = (c & 4) ? zb : za;
        const float X = fmaf(m[0], x, fmaf(m[1], y, m[3]));
        const float Y = fmaf(m[4], x, fmaf(m[5], y, m[7]));
        const float Z = fmaf(m[8], x, fmaf(m[9], y, m[11]));
        const float w = fmaf(m[10], z, Z);
        front = front && w > 0.f;
        const float rw = __fdividef(1.0f, w);
        const float u = fmaf(m[2], z, X) * rw, v = fmaf(m[6], z, Y) * rw;
        umin = fminf(umin, u);
        umax = fmaxf(umax, u);
        vmin = fminf(vmin, v);
        vmax = fmaxf(vmax, v);
    }
    md.flags = (m[2] == 0.f && m[10] == 0.f) ? kZFree : 0;
    md.u_lo = md.v_lo = 0;
    // the box is only trusted when every corner lies in front of the source and the values are
    // finite and moderate (a linear-fractional map is monotone along each edge there)
    if (!(front && umin > -1.0e6f && umax < 1.0e6f && vmin > -1.0e6f && vmax < 1.0e6f)) return;
    if (umax + 1.f < 0.f || umin - 1.f >= (float)(W - 1) || vmax + 1.f < 0.f || vmin - 1.f >= (float)(H - 1)) {
        md.flags |= kSkip;
        return;
    }
    const int u_lo = ((int)floorf(umin) - 1) & ~3;  // 16-byte aligned TMA x coordinate
    const int v_lo = (int)floorf(vmin) - 1;
    const int u_last = (int)floorf(umax) + 2, v_last = (int)floorf(vmax) + 2;
    md.u_lo = u_lo;
    md.v_lo = v_lo;
    if (u_last - u_lo + 1 <= BW && v_last - v_lo + 1 <= BH) md.flags |= kStaged;
    if (umin >= 1.f && umax < (float)(W - 2) && vmin >= 1.f && vmax < (float)(H - 2)) md.flags |= kInterior;
}

// One view's contribution to a thread's run of R voxels along z at column (X, Y, Z) (the
// matrix rows evaluated at z = 0).  src: the staged box (pitch BW, origin (u_lo, v_lo)) or the
// global view (pitch W, origin 0).  CHECK: the per-sample bounds rule of RtkSUBPIXEL and the
// run's end at nz; without it the caller guarantees both.  ZFREE: u and w are the column's.
// The arithmetic of every sample is that of rtk_bp_kernel, so results are bit-identical.
template <bool CHECK, bool ZFREE>
__device__ __forceinline__ void rtk_view(const float *m, float X, float Y, float Z, int k0, int nk,
                                         const float *src, int pitch, int u_lo, int v_lo, float wm1, float hm1,
                                         float (&acc)[rtkt::R]) {
    constexpr int R = rtkt::R;
    const float fk0 = (float)k0;  // one conversion per run; the slices add small exact integers
    if constexpr (ZFREE) {
        const float rw = __fdividef(1.0f, Z);  // fmaf(0, k, Z) == Z
        const float u = X * rw;                 // fmaf(0, k, X) == X
        if (!(u >= 0.f && u < wm1)) return;     // every sample of the column is zero
        const float iu = floorf(u);
        const float du = u - iu;
        const float *col = src + ((int)iu - u_lo) - v_lo * pitch;
#pragma unroll
        for (int kk = 0; kk < R; kk++) {
            const float fk = fk0 + (float)kk;  // == (float)(k0 + kk): integers below 2^24
            const float v = fmaf(m[6], fk, Y) * rw;
            float sv = 0.f;
            if (!CHECK || (kk < nk && v >= 0.f && v < hm1)) {
                const float iv = floorf(v);
                const float dv = v - iv;
                const float *p0 = col + (int)iv * pitch;
                const float *p1 = p0 + pitch;
                const float e0 = fmaf(du, p0[1] - p0[0], p0[0]);
                const float e1 = fmaf(du, p1[1] - p1[0], p1[0]);
                sv = fmaf(dv, e1 - e0, e0);
            }
            acc[kk] = fmaf(sv * rw, rw, acc[kk]);
        }
    } else {
#pragma unroll
        for (int kk = 0; kk < R; kk++) {
            const float fk = fk0 + (float)kk;  // == (float)(k0 + kk): integers below 2^24
            const float rw = __fdividef(1.0f, fmaf(m[10], fk, Z));
            const float u = fmaf(m[2], fk, X) * rw, v = fmaf(m[6], fk, Y) * rw;
            float sv = 0.f;
            if (!CHECK || (kk < nk && u >= 0.f && u < wm1 && v >= 0.f && v < hm1)) {
                const float iu = floorf(u), iv = floorf(v);
                const float du = u - iu, dv = v - iv;
                const float *p0 = src + ((int)iv - v_lo) * pitch + ((int)iu - u_lo);
                const float *p1 = p0 + pitch;
                const float e0 = fmaf(du, p0[1] - p0[0], p0[0]);
                const float e1 = fmaf(du, p1[1] - p1[0], p1[0]);
                sv = fmaf(dv, e1 - e0, e0);
            }
            acc[kk] = fmaf(sv * rw, rw, acc[kk]);
        }
    }
}

// CTAs per SM the register budget is set for (tuning macro).  Measured on 512^3 from 32 views of
// 512^2: 2 CTAs (96 registers) 910 / 654 GUPS circular / tilted, 3 CTAs (72 registers, no
// spills) 966 / 671 GUPS; the L1 kernel 602 / 602.
#ifndef FDK_RTK_MIN_BLOCKS
#define FDK_RTK_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(rtkt::THREADS, FDK_RTK_MIN_BLOCKS)
    rtk_tma_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ RtkMats mats, rtkt::Args a) {
    using namespace rtkt;
    extern __shared__ __align__(128) unsigned char smem[];
    Meta *meta = reinterpret_cast<Meta *>(smem + S * NV * BOX);
    float *smat = reinterpret_cast<float *>(meta + S * NV);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smat + kRtkMaxViews * 12);
    const unsigned boxes = smem_u32(smem);
    const unsigned full0 = smem_u32(bars), empty0 = smem_u32(bars + S);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = threadIdx.x; q < a.n * 12; q += blockDim.x) smat[q] = mats.m[q];
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, TX * TY / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int n_chunks = (a.n + NV - 1) / NV;
    const int n_tiles = a.tiles_x * a.tiles_y * a.tiles_z;
    const long long frame = (long long)a.W * a.H;

    if (warp == TX * TY / 32) {
        // ---------------- producer
        int it = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
            const int tx = tile % a.tiles_x, ty = (tile / a.tiles_x) % a.tiles_y;
            const int tz = tile / (a.tiles_x * a.tiles_y);
            const float xa = (float)(tx * TX), xb = (float)(min(tx * TX + TX, a.nx) - 1);
            const float ya = (float)(ty * TY), yb = (float)(min(ty * TY + TY, a.ny) - 1);
            const float za = (float)(tz * R), zb = (float)(min(tz * R + R, a.nz) - 1);
            for (int c = 0; c < n_chunks; c++, it++) {
                const int s = it % S;
                const unsigned ph = (unsigned)(it / S) & 1u;
                if (it >= S && !mbar_wait(empty0 + 8 * s, ph ^ 1u)) {
                    ok = false;
                    break;
                }
                const int view = c * NV + lane;
                if (lane < NV) {
                    Meta &md = meta[s * NV + lane];
                    if (view < a.n) rtk_tile_box(smat + 12 * view, xa, xb, ya, yb, za, zb, a.W, a.H, md);
                    else md.flags = kSkip;
                }
                __syncwarp();
                if (lane == 0) {
                    unsigned n_staged = 0;
                    for (int l = 0; l < NV; l++)
                        if ((meta[s * NV + l].flags & (kStaged | kSkip)) == kStaged) n_staged++;
                    mbar_arrive_tx(full0 + 8 * s, n_staged * (unsigned)BOX);
                    for (int l = 0; l < NV; l++) {
                        const Meta &md = meta[s * NV + l];
                        if ((md.flags & (kStaged | kSkip)) == kStaged)
                            tma_load_3d(boxes + (s * NV + l) * BOX, &tmap, md.u_lo, md.v_lo, c * NV + l, full0 + 8 * s);
                    }
                }
                __syncwarp();
            }
        }
        if (!ok && lane == 0) atomicOr(&g_rtk_err, kErrTimeout);
        // drain (always): wait, bounded, for the copies of the last stages to land before the CTA
        // may exit -- consumers that gave up on a wait have left already.  Immediate when the
        // consumers have waited for these stages themselves.
        if (lane == 0)
            for (int k = (it > S ? it - S : 0); k < it; k++) mbar_wait(full0 + 8 * (k % S), (unsigned)(k / S) & 1u);
        return;
    }

    // ---------------- consumers: 16 x 16 columns, R slices each
    const int cx = threadIdx.x % TX, cy = threadIdx.x / TX;
    const float wm1 = (float)(a.W - 1), hm1 = (float)(a.H - 1);
    int it = 0;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int tx = tile % a.tiles_x, ty = (tile / a.tiles_x) % a.tiles_y;
        const int tz = tile / (a.tiles_x * a.tiles_y);
        const int i = tx * TX + cx, j = ty * TY + cy, k0 = tz * R;
        const bool col_ok = i < a.nx && j < a.ny;
        const int nk = min(R, a.nz - k0);  // slices of the run inside the volume (the box covers only these)
        const float fi = (float)i, fj = (float)j;
        float acc[R];
#pragma unroll
        for (int kk = 0; kk < R; kk++) acc[kk] = 0.f;
        for (int c = 0; c < n_chunks; c++, it++) {
            const int s = it % S;
            const unsigned ph = (unsigned)(it / S) & 1u;
            if (!mbar_wait(full0 + 8 * s, ph)) {
                if (lane == 0) atomicOr(&g_rtk_err, kErrTimeout);
                return;
            }
            if (col_ok) {
                for (int l = 0; l < NV; l++) {
                    const int p = c * NV + l;
                    if (p >= a.n) break;
                    const Meta md = meta[s * NV + l];
                    if (md.flags & kSkip) continue;
                    const float *m = smat + 12 * p;
                    const float X = fmaf(m[0], fi, fmaf(m[1], fj, m[3]));
                    const float Y = fmaf(m[4], fi, fmaf(m[5], fj, m[7]));
                    const float Z = fmaf(m[8], fi, fmaf(m[9], fj, m[11]));
                    const bool zfree = md.flags & kZFree;
                    if (md.flags & kStaged) {
                        const float *box = reinterpret_cast<const float *>(smem + (s * NV + l) * BOX);
                        if ((md.flags & kInterior) && nk == R) {
                            if (zfree) rtk_view<false, true>(m, X, Y, Z, k0, nk, box, BW, md.u_lo, md.v_lo, wm1, hm1, acc);
                            else rtk_view<false, false>(m, X, Y, Z, k0, nk, box, BW, md.u_lo, md.v_lo, wm1, hm1, acc);
                        } else {
                            if (zfree) rtk_view<true, true>(m, X, Y, Z, k0, nk, box, BW, md.u_lo, md.v_lo, wm1, hm1, acc);
                            else rtk_view<true, false>(m, X, Y, Z, k0, nk, box, BW, md.u_lo, md.v_lo, wm1, hm1, acc);
                        }
                    } else {
                        const float *pv = a.proj + p * frame;
                        if (zfree) rtk_view<true, true>(m, X, Y, Z, k0, nk, pv, a.W, 0, 0, wm1, hm1, acc);
                        else rtk_view<true, false>(m, X, Y, Z, k0, nk, pv, a.W, 0, 0, wm1, hm1, acc);
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty0 + 8 * s);
        }
        if (col_ok) {
#pragma unroll
            for (int kk = 0; kk < R; kk++) {
                const int k = k0 + kk;
                if (k >= a.nz) break;
                const long long idx = i + ((long long)j + (long long)k * a.ny) * a.nx;
                a.vol_out[idx] = a.vol_in[idx] + acc[kk];
            }
        }
    }
}

}  // namespace fdk

using namespace fdk;

namespace fdk {

// Staged kernel where TMA can address the views (rows a multiple of 16 bytes, 16-byte aligned
// base, a detector at least one box wide and high); the L1 kernel otherwise.
int rtk_launch(const int32_t proj_size[3], const int32_t vol_size[3], const float *host_mats, const float *dev_vol_in,
               float *dev_vol_out, const float *dev_proj, cudaStream_t st) {
    const int W = proj_size[0], H = proj_size[1], n = proj_size[2];
    const int nx = vol_size[0], ny = vol_size[1], nz = vol_size[2];
    RtkMats m;
    for (int i = 0; i < 12 * n; i++) m.m[i] = host_mats[i];
    const char *sel = getenv("FDK_RTK_KERNEL");
    const bool l1 = sel && std::string(sel) == "l1";
    const bool tma_ok = !l1 && W % 4 == 0 && ((uintptr_t)dev_proj & 15) == 0 && W >= rtkt::BW && H >= rtkt::BH &&
                        tensor_map_encoder() != nullptr;
    if (!tma_ok) {
        const dim3 grid((unsigned)ceil_div(nx, 32), (unsigned)ceil_div(ny, 8), (unsigned)ceil_div(nz, kRtkR));
        rtk_bp_kernel<<<grid, dim3(32, 8), 0, st>>>(dev_vol_in, dev_vol_out, dev_proj, m, W, H, n, nx, ny, nz);
        FDK_CUDA(cudaGetLastError());
        return FDK_OK;
    }
    CUtensorMap map;
    const cuuint64_t dims[3] = {(cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)n};
    const cuuint64_t strides[2] = {(cuuint64_t)W * 4, (cuuint64_t)W * H * 4};
    const cuuint32_t box[3] = {(cuuint32_t)rtkt::BW, (cuuint32_t)rtkt::BH, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = tensor_map_encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(dev_proj),
                                            dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(FDK_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    FDK_CUDA(cudaFuncSetAttribute(rtk_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, rtkt::SMEM));
    int dev = 0, per_sm = 0, sms = 0;
    FDK_CUDA(cudaGetDevice(&dev));
    FDK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rtk_tma_kernel, rtkt::THREADS, rtkt::SMEM));
    FDK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    rtkt::Args a;
    a.vol_in = dev_vol_in;
    a.vol_out = dev_vol_out;
    a.proj = dev_proj;
    a.W = W;
    a.H = H;
    a.n = n;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.tiles_x = (int)ceil_div(nx, rtkt::TX);
    a.tiles_y = (int)ceil_div(ny, rtkt::TY);
    a.tiles_z = (int)ceil_div(nz, rtkt::R);
    const long long tiles = (long long)a.tiles_x * a.tiles_y * a.tiles_z;
    FDK_CHECK_ARG(tiles < (1ll << 31), "too many tiles");
    const int grid = (int)std::min<long long>(tiles, (long long)sms * std::max(per_sm, 1));
    rtk_tma_kernel<<<grid, rtkt::THREADS, rtkt::SMEM, st>>>(map, m, a);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
}

// Read and clear the staged kernel's device error word (after the work has finished).
int rtk_check_device_error() {
    unsigned int e = 0;
    FDK_CUDA(cudaMemcpyFromSymbol(&e, g_rtk_err, sizeof(e)));
    if (e) {
        const unsigned int zero = 0;
        cudaMemcpyToSymbol(g_rtk_err, &zero, sizeof(zero));
        return fail(FDK_ERR_DEVICE_CHECK, "RTK backprojection pipeline wait timed out on the device (error word %u)",
                    e);
    }
    return FDK_OK;
}

}  // namespace fdk

extern "C" {

int fdk_rtk_reconstruct_conebeam(const int32_t proj_size[3], const int32_t vol_size[3], const float *matrices,
                                 const float *dev_vol_in, float *dev_vol_out, const float *proj) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(proj_size && vol_size && matrices && dev_vol_in && dev_vol_out && proj, "NULL argument");
    const int W = proj_size[0], H = proj_size[1], n = proj_size[2];
    const int nx = vol_size[0], ny = vol_size[1], nz = vol_size[2];
    FDK_CHECK_ARG(W > 1 && H > 1 && n > 0 && n <= 32, "proj_size out of range (views <= 32)");
    FDK_CHECK_ARG(nx > 0 && ny > 0 && nz > 0 && nz <= 65535, "vol_size out of range");
    const size_t bytes = sizeof(float) * (size_t)W * H * n;
    float *d_proj = nullptr;
    FDK_CUDA(cudaMalloc(&d_proj, bytes));
    int s = FDK_OK;
    cudaError_t e = cudaMemcpy(d_proj, proj, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        s = rtk_launch(proj_size, vol_size, matrices, dev_vol_in, dev_vol_out, d_proj, nullptr);
        if (s == FDK_OK) e = cudaStreamSynchronize(cudaStreamLegacy);  // synchronous, as the reference
    }
    if (s == FDK_OK && e != cudaSuccess) s = cuda_status(e, "CUDA_reconstruct_conebeam", __FILE__, __LINE__);
    if (s == FDK_OK) s = rtk_check_device_error();
    cudaFree(d_proj);
    return s;
    FDK_ABI_END
}

int fdk_rtk_backproject_device(const int32_t proj_size[3], const int32_t vol_size[3], const float *host_mats,
                               const float *dev_vol_in, float *dev_vol_out, const float *dev_proj, void *stream) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(proj_size && vol_size && host_mats && dev_vol_in && dev_vol_out && dev_proj, "NULL argument");
    FDK_CHECK_ARG(proj_size[0] > 1 && proj_size[1] > 1 && proj_size[2] > 0 && proj_size[2] <= kRtkMaxViews,
                  "proj_size out of range (views <= %d)", kRtkMaxViews);
    FDK_CHECK_ARG(vol_size[0] > 0 && vol_size[1] > 0 && vol_size[2] > 0 && vol_size[2] <= 65535,
                  "vol_size out of range");
    return rtk_launch(proj_size, vol_size, host_mats, dev_vol_in, dev_vol_out, dev_proj, (cudaStream_t)stream);
    FDK_ABI_END
}

int fdk_rtk_sync(void *stream) {
    FDK_ABI_BEGIN
    clear_error();
    cudaEvent_t ev = nullptr;
    FDK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    const int s = wait_stream((cudaStream_t)stream, ev, "fdk_rtk_sync");  // bounded
    cudaEventDestroy(ev);
    FDK_TRY(s);
    return rtk_check_device_error();
    FDK_ABI_END
}

}  // extern "C"
