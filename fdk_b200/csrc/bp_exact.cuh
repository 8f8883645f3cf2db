// bp_exact.cuh -- backprojection kernel with the reference kernel's arithmetic.
//
// Same per-voxel operations, in the same order and rounding, as cudaFdkBP<TRANSPOSE, false,
// bSymmetric> (cudaBP/backprojectionFDK.cu:50-129, SUBPIXEL :15-48, dotIJKW and the
// mad.rz.ftz blend cudaBP/cudaBpLib.cuh:5-44), so the results are bit-identical; including the
// way each warp obtains (U, 1/w) for view s from lane s and broadcasts it.  The launch shape
// differs: 256-thread CTAs (32 z-lanes x 8 columns), 64-bit volume offsets (the reference's
// 32-bit `uint offset` wraps beyond 2^32 voxels), and partial last warps stay alive through
// the shuffles and only skip the store.
#pragma once
#include "common.h"

namespace fdk {

struct BpExactArgs {
    float *vol;          // [x][y][zs] sub-volume, zs extent D
    const float *proj;   // n_proj frames of height x width (pitch = width)
    const float *mats;   // 12 floats per view
    int width, height, n_proj;
    int x0, y0, z0;      // origin of the top slab (minA)
    int nxs, nys, nzz;   // top slab extent; nzz = z count processed per thread column
    long long D;         // storage depth (top + bottom)
    int transpose;       // 1: frame rows are detector columns (u), 0: detector rows (v)
};

__device__ __forceinline__ float fma_rz(float a, float b, float c) {
    float d;
    asm("fma.rz.ftz.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

__device__ __forceinline__ float dot_ijkw(const float4 m, const float4 p) {
    float s = m.w;
    s = fma_rz(m.x, p.x, s);
    s = fma_rz(m.y, p.y, s);
    s = fma_rz(m.z, p.z, s);
    return s;
}

// Bilinear sample at (x along the frame row, y across rows), zero outside
// [0, width-1) x [0, height-1).
__device__ __forceinline__ float subpixel_exact(const float *p, int pitch, int width, int height, float x,
                                                float y) {
    float s = 0.0f;
    if (x >= 0 && x < width - 1 && y >= 0 && y < height - 1) {
        const float ix = floorf(x), iy = floorf(y);
        const int nx = (int)ix, ny = (int)iy;
        const float dx = x - ix, dy = y - iy;
        const float _dx = 1.0f - dx, _dy = 1.0f - dy;
        const float *p0 = p + (long long)ny * pitch + nx;
        const float *p1 = p0 + pitch;
        float x0 = __ldg(p0), x1 = __ldg(p0 + 1), x2 = __ldg(p1), x3 = __ldg(p1 + 1);
        x0 = fma_rz(x0, _dx, x1 * dx);
        x2 = fma_rz(x2, _dx, x3 * dx);
        s = fma_rz(x0, _dy, x2 * dy);
    }
    return s;
}

template <bool SYM, bool TRANSPOSE>
__global__ void __launch_bounds__(256) bp_exact_kernel(BpExactArgs a) {
    __shared__ float4 sm[128 * 3];
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int q = tid; q < a.n_proj * 3; q += 256) sm[q] = reinterpret_cast<const float4 *>(a.mats)[q];
    __syncthreads();

    const unsigned lane = threadIdx.x;
    const unsigned ii = blockIdx.x * 32 + lane;
    const unsigned jj = blockIdx.y * 8 + threadIdx.y;
    const unsigned kk = blockIdx.z;
    const bool valid = ii < (unsigned)a.nzz && jj < (unsigned)a.nys;
    const float4 ijkw = make_float4((float)(kk + a.x0), (float)(jj + a.y0), (float)(ii + a.z0), 1.f);
    const long long frame = (long long)a.width * a.height;

    float sum = 0.f, _sum = 0.f;
    // views are taken 32 at a time: lane s provides (U, 1/w) of view base+s
    for (int base = 0; base < a.n_proj; base += 32) {
        const int nb = min(32, a.n_proj - base);
        float Z = 0.f, U = 0.f;
        if ((int)lane < nb) {
            Z = 1.f / dot_ijkw(sm[(base + lane) * 3 + 2], ijkw);
            U = dot_ijkw(sm[(base + lane) * 3 + 0], ijkw) * Z;
        }
        for (int s = 0; s < nb; s++) {
            const float u = __shfl_sync(0xffffffffu, U, s);
            const float f = __shfl_sync(0xffffffffu, Z, s);
            const float f2 = f * f;
            const float v = dot_ijkw(sm[(base + s) * 3 + 1], ijkw) * f;
            const float *p = a.proj + (long long)(base + s) * frame;
            if (TRANSPOSE) {
                sum = fma_rz(subpixel_exact(p, a.width, a.width, a.height, v, u), f2, sum);
                if (SYM) {
                    const float _v = (float)(a.width - 1) - v;
                    _sum = fma_rz(subpixel_exact(p, a.width, a.width, a.height, _v, u), f2, _sum);
                }
            } else {
                sum = fma_rz(subpixel_exact(p, a.width, a.width, a.height, u, v), f2, sum);
                if (SYM) {
                    const float _v = (float)(a.height - 1) - v;
                    _sum = fma_rz(subpixel_exact(p, a.width, a.width, a.height, u, _v), f2, _sum);
                }
            }
        }
        if (base + 32 < a.n_proj) {
            // The reference launches at most 32 views; a longer batch is a sequence of
            // 32-view launches, each adding its own partial sum to the volume.
            if (valid) {
                float *out = a.vol + ((long long)kk * a.nys + jj) * a.D;
                out[ii] += sum;
                if (SYM) out[a.D - 1 - ii] += _sum;
            }
            sum = 0.f;
            _sum = 0.f;
        }
    }
    if (valid) {
        float *out = a.vol + ((long long)kk * a.nys + jj) * a.D;
        out[ii] += sum;
        if (SYM) out[a.D - 1 - ii] += _sum;
    }
}

}  // namespace fdk
