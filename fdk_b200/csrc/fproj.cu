// fproj.cu -- ray-marching forward projector (the reference's genProj kernel_forwardProject,
// genProj/cudaForwardProjection.cu:174-254, with Text3DLinear, genProj/cudaIterType.cuh:232-276).
//
// One thread per detector pixel.  The ray runs from the source to the pixel centre; it is
// clipped to the box spanned by the voxel centres (cuIntersectBox, :28-48), then sampled every
// tStep = min(dx, dy, dz) mm from the entry point (t < t_far), each sample trilinear on the voxel
// grid with texel indices truncated toward zero and clamped to the volume (the reference's
// point-sampled, clamp-addressed 3-D texture read at integer coordinates); the pixel value is
// sum * tStep.  Geometry: for BP view angle a the projector rotates by -a (:426), i.e. the source
// sits at R(a)^T (0, -SOD, 0) and the detector plane at distance SID, consistent with
// CalculateProjMat.  The volume is [z][y][x], x fastest, in the world frame
// X = (x-(nx-1)/2) dx, Y = -(y-(ny-1)/2) dy, Z = -(z-(nz-1)/2) dz.
#include <vector>

#include "common.h"

namespace fdk {

struct FprojArgs {
    const float *vol;
    float *out;
    const double *angles;  // BP view angles of the launched views
    int nx, ny, nz, nu, nv;
    float dx, dy, dz, du, dv, sid, sod, off_u, off_v;
};

__device__ __forceinline__ float vox(const FprojArgs &a, int x, int y, int z) {
    x = min(max(x, 0), a.nx - 1);
    y = min(max(y, 0), a.ny - 1);
    z = min(max(z, 0), a.nz - 1);
    return __ldg(a.vol + ((long long)z * a.ny + y) * a.nx + x);
}

__global__ void __launch_bounds__(256) fproj_kernel(FprojArgs a) {
    const int pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= a.nu * a.nv) return;
    const int j = pix / a.nu, i = pix - j * a.nu;  // detector column i, row j
    const long long view = blockIdx.y;
    const double ang = -a.angles[view];
    const float c = (float)cos(ang), s = (float)sin(ang);
    // source and detector pixel in mm, rotated (cuRotate: x' = x c - y s, y' = x s + y c)
    const float src_y = -a.sod, det_y = a.sid - a.sod;
    const float ox = -src_y * s, oy = src_y * c, oz = 0.f;
    const float cu = (a.nu - 1) / 2.0f + a.off_u, cv = (a.nv - 1) / 2.0f + a.off_v;
    const float umm = ((float)i - cu) * a.du, vmm = (cv - (float)j) * a.dv;
    const float px = umm * c - det_y * s, py = umm * s + det_y * c, pz = vmm;
    float dxr = px - ox, dyr = py - oy, dzr = pz - oz;
    const float inv = rsqrtf(dxr * dxr + dyr * dyr + dzr * dzr);
    dxr *= inv;
    dyr *= inv;
    dzr *= inv;
    // voxel-centre box in mm
    const float bx = (a.nx - 1) / 2.0f * a.dx, by = (a.ny - 1) / 2.0f * a.dy, bz = (a.nz - 1) / 2.0f * a.dz;
    const float ix = 1.0f / dxr, iy = 1.0f / dyr, iz = 1.0f / dzr;
    const float tx0 = (-bx - ox) * ix, tx1 = (bx - ox) * ix;
    const float ty0 = (-by - oy) * iy, ty1 = (by - oy) * iy;
    const float tz0 = (-bz - oz) * iz, tz1 = (bz - oz) * iz;
    const float tnear = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fminf(tz0, tz1));
    const float tfar = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1));
    const float step = fminf(fminf(a.dx, a.dy), a.dz);
    float sum = 0.f;
    if (tfar > tnear) {
        // index-space origin and direction: i = X/dx + cx, j = cy - Y/dy, k = cz - Z/dz
        const float cxv = (a.nx - 1) / 2.0f, cyv = (a.ny - 1) / 2.0f, czv = (a.nz - 1) / 2.0f;
        const float si = ox / a.dx + cxv, sj = cyv - oy / a.dy, sk = czv - oz / a.dz;
        const float vi = dxr / a.dx, vj = -dyr / a.dy, vk = -dzr / a.dz;
        for (float t = tnear; t < tfar; t += step) {
            const float pi = si + vi * t, pj = sj + vj * t, pk = sk + vk * t;
            const int ai = (int)pi, aj = (int)pj, ak = (int)pk;  // truncation, as int3(pos)
            const float fi = pi - ai, fj = pj - aj, fk = pk - ak;
            const float c00 = vox(a, ai, aj, ak) * (1 - fk) + vox(a, ai, aj, ak + 1) * fk;
            const float c10 = vox(a, ai + 1, aj, ak) * (1 - fk) + vox(a, ai + 1, aj, ak + 1) * fk;
            const float c01 = vox(a, ai, aj + 1, ak) * (1 - fk) + vox(a, ai, aj + 1, ak + 1) * fk;
            const float c11 = vox(a, ai + 1, aj + 1, ak) * (1 - fk) + vox(a, ai + 1, aj + 1, ak + 1) * fk;
            const float f0 = c00 * (1 - fj) + c01 * fj, f1 = c10 * (1 - fj) + c11 * fj;
            sum += f0 * (1 - fi) + f1 * fi;
        }
    }
    a.out[view * (long long)a.nu * a.nv + pix] = sum * step;
}

}  // namespace fdk

using namespace fdk;

extern "C" int fdk_forward_project(const fdk_geometry *g, const float *dev_vol, int64_t first, int64_t n,
                                   float *dev_out, void *stream) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(g && dev_vol && dev_out, "NULL argument");
    FDK_CHECK_ARG(first >= 0 && n > 0 && first + n <= g->n_proj && n <= 65535, "view range out of bounds");
    FDK_CHECK_ARG(g->nu * g->nv < (1ll << 31), "detector too large");
    std::vector<double> ang(g->n_proj);
    FDK_TRY(fdk_view_angles(g, ang.data()));
    cudaStream_t st = (cudaStream_t)stream;
    double *d_ang = nullptr;
    FDK_CUDA(cudaMallocAsync((void **)&d_ang, sizeof(double) * n, st));
    FDK_CUDA(cudaMemcpyAsync(d_ang, ang.data() + first, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    FprojArgs a;
    a.vol = dev_vol;
    a.out = dev_out;
    a.angles = d_ang;
    a.nx = (int)g->nx;
    a.ny = (int)g->ny;
    a.nz = (int)g->nz;
    a.nu = (int)g->nu;
    a.nv = (int)g->nv;
    a.dx = (float)g->dx;
    a.dy = (float)g->dy;
    a.dz = (float)g->dz;
    a.du = (float)g->du;
    a.dv = (float)g->dv;
    a.sid = (float)g->sid;
    a.sod = (float)g->sod;
    a.off_u = (float)g->offset_nu;
    a.off_v = (float)g->offset_nv;
    const dim3 grid((unsigned)ceil_div(g->nu * g->nv, 256), (unsigned)n);
    fproj_kernel<<<grid, 256, 0, st>>>(a);
    FDK_CUDA(cudaGetLastError());
    FDK_CUDA(cudaFreeAsync(d_ang, st));
    FDK_CUDA(cudaStreamSynchronize(st));  // the host angle table goes out of scope
    return FDK_OK;
    FDK_ABI_END
}
