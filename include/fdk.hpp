// fdk.hpp -- C++ host API with the reference's class names and call shapes, header-only over the
// C ABI in fdk.h (link libfdk_b200.so).  A reference pipeline (cuFDK/mpiFDK.cpp) switches by
// including this header instead of Filterlib/FilterLib.h and cudaBP/backprojection.cuh:
//
//   fdk::FilterEngine        Filterlib/FilterLib.h:148-203       (Filtering(src, dst, transpose))
//   fdk::FilterRow_Real32    FilterlibCufft/cudaFftFilter.cuh:7  (device DataRef)
//   fdk::CorrectImage_Real32 FilterlibCufft/cudaFftFilter.cuh:9
//   fdk::BackProjectionFDK   cudaBP/backprojection.cuh:246-271   (ctor, BP, GetVolumeData, nBpCount,
//                                                                 fKernelTime)
//   fdk::CUDA_reconstruct_conebeam  cudaBP/rtkCudaFDKBackProjectionImageFilter.cu:200-206
//
// Errors: the reference throws std::string from VERIFY_TRUE / CUDA_CHECK_ERROR
// (common/type.h:194-196, common/cudaLib.cuh:49-56); these wrappers throw fdk::Error (a
// std::runtime_error carrying the FDK_ERR_* code and fdk_last_error()).
#pragma once
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "fdk.h"

namespace fdk {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != FDK_OK) throw Error(rc, std::string("fdk: ") + fdk_last_error());
}

// geo::BoxT<size_t> (cudaBP/backprojection.cuh:66-116)
struct BoxT : fdk_box {
    BoxT() : fdk_box{0, 0, 0, 0, 0, 0} {}
    BoxT(uint64_t x_, uint64_t y_, uint64_t z_, uint64_t w, uint64_t h, uint64_t d) : fdk_box{x_, y_, z_, w, h, d} {}
    uint64_t MinX() const { return x; }
    uint64_t MinY() const { return y; }
    uint64_t MinZ() const { return z; }
    uint64_t MaxX() const { return x + width - 1; }
    uint64_t MaxY() const { return y + height - 1; }
    uint64_t MaxZ() const { return z + depth - 1; }
};

class FilterEngine {
  public:
    // FilterEngine(FrameT<float> cos_image_table, const std::vector<float>& fft_kernel_real_f32);
    // cos table nv rows of nu; pad_edge 4 as the IPP plugin (FilterLib.h:38,44).
    FilterEngine(const float *cos_table, int nu, int nv, const std::vector<float> &H, int pad_edge = 4,
                 int device = 0) : nu_(nu), nv_(nv) {
        check(fdk_filter_create(&h_, cos_table, H.data(), nu, nv, (int64_t)H.size(), pad_edge, device));
    }
    ~FilterEngine() { fdk_filter_destroy(h_); }
    FilterEngine(const FilterEngine &) = delete;
    FilterEngine &operator=(const FilterEngine &) = delete;
    // src (nv x nu) is cosine-weighted in place, as the reference does (FilterLib.h:181).
    FilterEngine &Filtering(float *src, float *dst, bool transpose = false) {
        check(fdk_filter_filtering(h_, src, dst, transpose ? 1 : 0));
        return *this;
    }
    fdk_filter *handle() { return h_; }

  private:
    fdk_filter *h_ = nullptr;
    int nu_, nv_;
};

inline bool CorrectImage_Real32(const fdk_dataref &src, const fdk_dataref &table, fdk_dataref &dst) {
    check(fdk_correct_image_real32(&src, &table, &dst));
    return true;
}
inline bool FilterRow_Real32(const fdk_dataref &src, fdk_dataref &dst, const fdk_dataref &filter) {
    check(fdk_filter_row_real32(&src, &dst, &filter));
    return true;
}

class BackProjectionFDK {
  public:
    enum { MAX_PROJ = 32, PROJ_MAT_ROWS = 3, PROJ_MAT_COLS = 4, PROJ_MAT_SIZE = 12 };
    BackProjectionFDK(int projWidth, int projHeight, int projCount, int nx, int ny, int nz, BoxT subTop,
                      BoxT subBottom, int precision = FDK_BP_FP32_EXACT, int device = 0)
        : top_(subTop), bottom_(subBottom) {
        check(fdk_bp_create(&h_, projWidth, projHeight, projCount, nx, ny, nz, &top_, &bottom_, precision, device));
    }
    ~BackProjectionFDK() { fdk_bp_destroy(h_); }
    BackProjectionFDK(const BackProjectionFDK &) = delete;
    BackProjectionFDK &operator=(const BackProjectionFDK &) = delete;

    // bool BP(int TRANSPOSE, const float* pProjData, int width, int height, float* pProjMat, int nProj)
    bool BP(int TRANSPOSE, const float *pProjData, int width, int height, const float *pProjMat, int nProj) {
        check(fdk_bp_bp(h_, TRANSPOSE, pProjData, width, height, pProjMat, nProj));
        return true;
    }
    // bool GetVolumeData(float* pVol, int size): [zs][y][x], top slab then bottom slab
    bool GetVolumeData(float *pVol, int64_t size) {
        check(fdk_bp_get_volume(h_, pVol, size));
        return true;
    }
    int64_t nBpCount() {
        int64_t n = 0;
        check(fdk_bp_stats(h_, &n, nullptr));
        return n;
    }
    double fKernelTime() {
        double ms = 0;
        check(fdk_bp_stats(h_, nullptr, &ms));
        return ms;
    }
    fdk_bp *handle() { return h_; }

  private:
    BoxT top_, bottom_;
    fdk_bp *h_ = nullptr;
};

// BackProjectionRTK::CUDA_reconstruct_conebeam (device volumes, host projections)
inline void CUDA_reconstruct_conebeam(int proj_size[3], int vol_size[3], const float *matrices,
                                      const float *dev_vol_in, float *dev_vol_out, const float *dev_proj) {
    const int32_t ps[3] = {proj_size[0], proj_size[1], proj_size[2]};
    const int32_t vs[3] = {vol_size[0], vol_size[1], vol_size[2]};
    check(fdk_rtk_reconstruct_conebeam(ps, vs, matrices, dev_vol_in, dev_vol_out, dev_proj));
}

// Single-GPU streaming FDK (filter -> BP handoff of cuFDK), whole volume or one slab pair.
class Reconstructor {
  public:
    Reconstructor(const fdk_geometry &g, int precision = FDK_BP_MIXED, int batch = 128, int device = 0) {
        check(fdk_recon_create(&h_, &g, precision, batch, device));
    }
    Reconstructor(const fdk_geometry &g, int64_t top_z, int64_t depth, int precision, int batch, int device) {
        check(fdk_recon_create_slab(&h_, &g, top_z, depth, precision, batch, device));
    }
    ~Reconstructor() { fdk_recon_destroy(h_); }
    Reconstructor(const Reconstructor &) = delete;
    Reconstructor &operator=(const Reconstructor &) = delete;
    void Push(const float *host_views, int64_t first, int64_t n) { check(fdk_recon_push(h_, host_views, first, n)); }
    void PushDevice(const float *dev_views, int64_t first, int64_t n) {
        check(fdk_recon_push_device(h_, dev_views, first, n));
    }
    // views first..first+n-1 from a projection folder (folder + "img%04d.raw", file v*step+start)
    void PushFolder(const std::string &folder, int64_t first, int64_t n, int step = 1, int start = 0,
                    int threads = 0) {
        check(fdk_recon_push_folder(h_, folder.c_str(), first, n, step, start, threads));
    }
    void Flush() { check(fdk_recon_flush(h_)); }
    void Sync(int64_t timeout_ms = 0) { check(fdk_recon_sync(h_, timeout_ms)); }
    void GetVolume(float *host_vol, int64_t size) { check(fdk_recon_get_volume(h_, host_vol, size)); }
    fdk_recon *handle() { return h_; }

  private:
    fdk_recon *h_ = nullptr;
};

// On-disk formats (common/type.h): projection folders of img%04d.raw, ".vol" volumes, slice files.
inline std::string GetProjPath(const std::string &folder, int64_t view, int step = 1, int start = 0) {
    char buf[4096];
    check(fdk_proj_path(folder.c_str(), view, step, start, buf, (int32_t)sizeof(buf)));
    return buf;
}
inline void LoadProjectionFolder(const std::string &folder, int nu, int nv, int64_t first, int64_t count,
                                 float *host_views, int step = 1, int start = 0, int threads = 0) {
    check(fdk_load_proj_folder(folder.c_str(), nu, nv, first, count, step, start, host_views, threads));
}
inline void SaveProjectionFolder(const std::string &folder, const float *host_views, int nu, int nv, int64_t first,
                                 int64_t count, int step = 1, int threads = 0) {
    check(fdk_save_proj_folder(folder.c_str(), host_views, nu, nv, first, count, step, threads));
}
inline void SaveVolume(const std::string &path, const float *vol, int nx, int ny, int nz) {
    check(fdk_save_volume(path.c_str(), vol, nx, ny, nz));
}
inline std::vector<float> LoadVolume(const std::string &path, int &nx, int &ny, int &nz) {
    int32_t x = 0, y = 0, z = 0;
    check(fdk_load_volume(path.c_str(), nullptr, 0, &x, &y, &z));
    std::vector<float> v((size_t)x * y * z);
    check(fdk_load_volume(path.c_str(), v.data(), (int64_t)v.size(), &x, &y, &z));
    nx = x, ny = y, nz = z;
    return v;
}
inline void SaveVolumeSlices(const std::string &folder, const float *vol, int nx, int ny, int z0, int depth,
                             int threads = 0) {
    check(fdk_save_volume_slices(folder.c_str(), vol, nx, ny, z0, depth, threads));
}

}  // namespace fdk
