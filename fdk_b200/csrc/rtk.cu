// rtk.cu -- the RTK-style backprojection drop-in, CUDA_reconstruct_conebeam
// (cudaBP/rtkCudaFDKBackProjectionImageFilter.cu:200-330, kernel_fdk_3Dgrid :156-191,
// RtkSUBPIXEL :83-112).
//
// General 3x4 geometry: every voxel evaluates its own projection for every view (no
// circular-orbit shortcut), so tilted or non-circular trajectories are handled.  Views are
// read from global memory through L1 with explicit FP32 bilinear interpolation (the reference
// used point-sampled layered textures); a sample is zero outside [0, W-1) x [0, H-1).
// vol_out = vol_in + sum_p bilinear(proj_p; u, v) / w^2, x fastest.
#include "common.h"

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

}  // namespace fdk

using namespace fdk;

namespace fdk {

int rtk_launch(const int32_t proj_size[3], const int32_t vol_size[3], const float *host_mats, const float *dev_vol_in,
               float *dev_vol_out, const float *dev_proj, cudaStream_t st) {
    const int W = proj_size[0], H = proj_size[1], n = proj_size[2];
    const int nx = vol_size[0], ny = vol_size[1], nz = vol_size[2];
    RtkMats m;
    for (int i = 0; i < 12 * n; i++) m.m[i] = host_mats[i];
    const dim3 grid((unsigned)ceil_div(nx, 32), (unsigned)ceil_div(ny, 8), (unsigned)ceil_div(nz, kRtkR));
    rtk_bp_kernel<<<grid, dim3(32, 8), 0, st>>>(dev_vol_in, dev_vol_out, dev_proj, m, W, H, n, nx, ny, nz);
    FDK_CUDA(cudaGetLastError());
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
        if (s == FDK_OK) e = cudaDeviceSynchronize();
    }
    if (s == FDK_OK && e != cudaSuccess) s = cuda_status(e, "CUDA_reconstruct_conebeam", __FILE__, __LINE__);
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

}  // extern "C"
