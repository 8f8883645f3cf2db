// phantom.cu -- exact line integrals of ellipsoid phantoms, computed on the device in FP64.
//
// The ray through detector pixel (u, v) of a view is the preimage of that view's projection
// matrix (CalculateProjMat, common/type.h:4898-4944): it starts at the source (camera origin)
// and has camera-frame direction ((u-cu) du, (v-cv) dv, SID).  Camera -> rotated world:
// X_r = X_c, Y_r = Z_c - SOD, Z_r = -Y_c; world = Rz(angle)^T * rotated.  Each ellipsoid
// contributes rho * (length of the chord the ray cuts through it).
#include <vector>

#include "common.h"

namespace fdk {

constexpr int kMaxEll = 64;

__global__ void __launch_bounds__(256) phantom_kernel(const double *__restrict__ ell_g, int n_ell,
                                                      const double *__restrict__ angles, int nu, int nv, double du,
                                                      double dv, double sid, double sod, float *out) {
    __shared__ double ell[kMaxEll * 16];
    for (int q = threadIdx.x; q < n_ell * 16; q += blockDim.x) ell[q] = ell_g[q];
    __syncthreads();
    const long long view = blockIdx.y;
    const int pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= nu * nv) return;
    const int r = pix / nu, q = pix - r * nu;
    const double a = angles[view];
    const double c = cos(a), s = sin(a);
    const double cu = (nu - 1) / 2.0, cv = (nv - 1) / 2.0;
    const double o[3] = {-s * sod, -c * sod, 0.0};  // source: rotated (0, -SOD, 0)
    const double xr = (q - cu) * du, yr = sid, zr = -(r - cv) * dv;
    const double d[3] = {c * xr + s * yr, -s * xr + c * yr, zr};
    const double dl = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double sum = 0.0;
    for (int k = 0; k < n_ell; k++) {
        const double *e = ell + 16 * k;
        const double p0 = o[0] - e[0], p1 = o[1] - e[1], p2 = o[2] - e[2];
        double A = 0.0, B = 0.0, C = -1.0;
#pragma unroll
        for (int t = 0; t < 3; t++) {
            // local = R^T (p - c), R row major
            const double lo = e[6 + t] * p0 + e[9 + t] * p1 + e[12 + t] * p2;
            const double ld = e[6 + t] * d[0] + e[9 + t] * d[1] + e[12 + t] * d[2];
            const double iq = 1.0 / (e[3 + t] * e[3 + t]);
            A += ld * ld * iq;
            B += 2.0 * lo * ld * iq;
            C += lo * lo * iq;
        }
        const double disc = B * B - 4.0 * A * C;
        if (disc > 0.0 && A > 0.0) sum += e[15] * sqrt(disc) / A * dl;
    }
    out[view * (long long)nu * nv + pix] = (float)sum;
}

}  // namespace fdk

using namespace fdk;

extern "C" int fdk_phantom_project(const fdk_geometry *g, const double *ell, int32_t n_ell, int64_t first, int64_t n,
                                   float *dev_out, void *stream) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(g && ell && dev_out, "NULL argument");
    FDK_CHECK_ARG(n_ell >= 0 && n_ell <= kMaxEll, "n_ell must be 0..%d", kMaxEll);
    FDK_CHECK_ARG(first >= 0 && n > 0 && first + n <= g->n_proj && n <= 65535, "view range out of bounds");
    FDK_CHECK_ARG(g->nu * g->nv < (1ll << 31), "detector too large");
    std::vector<double> ang(g->n_proj);
    FDK_TRY(fdk_view_angles(g, ang.data()));
    cudaStream_t st = (cudaStream_t)stream;
    double *d_ell = nullptr, *d_ang = nullptr;
    FDK_CUDA(cudaMallocAsync((void **)&d_ell, sizeof(double) * 16 * (n_ell > 0 ? n_ell : 1), st));
    FDK_CUDA(cudaMallocAsync((void **)&d_ang, sizeof(double) * n, st));
    if (n_ell > 0) FDK_CUDA(cudaMemcpyAsync(d_ell, ell, sizeof(double) * 16 * n_ell, cudaMemcpyHostToDevice, st));
    FDK_CUDA(cudaMemcpyAsync(d_ang, ang.data() + first, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    const dim3 grid((unsigned)ceil_div(g->nu * g->nv, 256), (unsigned)n);
    phantom_kernel<<<grid, 256, 0, st>>>(d_ell, n_ell, d_ang, (int)g->nu, (int)g->nv, g->du, g->dv, g->sid, g->sod,
                                         dev_out);
    FDK_CUDA(cudaGetLastError());
    FDK_CUDA(cudaFreeAsync(d_ell, st));
    FDK_CUDA(cudaFreeAsync(d_ang, st));
    // the host angle vector is copied asynchronously: wait for the copies before it goes away
    FDK_CUDA(cudaStreamSynchronize(st));
    return FDK_OK;
    FDK_ABI_END
}
