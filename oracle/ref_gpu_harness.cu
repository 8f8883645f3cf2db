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
