// ref_gpu_harness.cu -- extern "C" entry points around the reference's own GPU
// code, compiled in place from the reference tree for sm_100a by
// oracle/build_ref.sh.  TEST INFRASTRUCTURE ONLY: the parity checker for the
// product's GPU path, never the product.
//
//   refg_bp_*      BackProjectionFDK ctor / BP / GetVolumeData / nBpCount
//                  (cudaBP/backprojection.cuh:246-271, backprojectionFDK.cu:161-362),
//                  kernel cudaFdkBP (backprojectionFDK.cu:50-129)
#include "cudaBP/backprojectionFDK.cu"
#include <string>

extern "C" void* refg_bp_create(int projW, int projH, int projCount, int nx, int ny, int nz,
                                const long top[6], const long bottom[6]) {
    try {
        geo::BoxT<size_t> t(top[0], top[1], top[2], top[3], top[4], top[5]);
        geo::BoxT<size_t> b(bottom[0], bottom[1], bottom[2], bottom[3], bottom[4], bottom[5]);
        return new BackProjectionFDK(projW, projH, projCount, nx, ny, nz, t, b, false);
    } catch (...) {
        return nullptr;
    }
}

extern "C" int refg_bp(void* h, int transpose, const float* host_proj, int width, int height,
                       float* mats, int n) {
    try {
        return static_cast<BackProjectionFDK*>(h)->BP(transpose, host_proj, width, height, mats, n) ? 0 : -1;
    } catch (...) {
        return -2;
    }
}

extern "C" int refg_bp_get_volume(void* h, float* host_vol, long size) {
    try {
        return static_cast<BackProjectionFDK*>(h)->GetVolumeData(host_vol, (int)size) ? 0 : -1;
    } catch (...) {
        return -2;
    }
}

extern "C" void refg_bp_destroy(void* h) { delete static_cast<BackProjectionFDK*>(h); }

// Device time of n_launch launches of the reference kernel exactly as BP(TRANSPOSE = 1) issues
// it for a symmetric slab pair (inBP<1, true>, backprojectionFDK.cu:240-276: same grid, block and
// arguments), over the views and matrices the last BP() call left on the device -- BP() itself
// times nothing and copies its views synchronously inside the call.  Milliseconds per launch,
// or a negative value on error.
extern "C" float refg_bp_kernel_ms(void* hv, int nProj, int n_launch) {
    try {
        BackProjectionFDK* h = static_cast<BackProjectionFDK*>(hv);
        if (h->subBottom.depth == 0 || n_launch <= 0) return -1.f;
        dim3 blockSize(WarpSize, 8, 4);
        dim3 gridSize(UpDivide(h->subTop.depth, blockSize.x), UpDivide(h->subTop.height, blockSize.y),
                      UpDivide(h->subTop.width, blockSize.z));
        int3 minA = {(int)h->subTop.MinX(), (int)h->subTop.MinY(), (int)h->subTop.MinZ()};
        int3 minB = {(int)h->subBottom.MinX(), (int)h->subBottom.MinY(), (int)h->subBottom.MinZ()};
        int3 sub_vol_dim = {(int)h->subTop.width, (int)h->subTop.height, (int)(h->subTop.depth + h->subBottom.depth)};
        int3 vol_dim = {(int)h->nx, (int)h->ny, (int)h->nz};
        int3 dimImg = {(int)h->projWidth, (int)h->projHeight, nProj};
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        for (int i = 0; i < n_launch; i++)
            cudaFdkBP<1, false, true><<<gridSize, blockSize>>>(h->pDevVolOut->GetData(), minA, minB, sub_vol_dim,
                                                               vol_dim, h->pDevProjData->GetData(),
                                                               h->pDevProjData->DataPitch(), dimImg);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return cudaGetLastError() == cudaSuccess ? ms / n_launch : -2.f;
    } catch (...) {
        return -3.f;
    }
}
