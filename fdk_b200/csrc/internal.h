// internal.h -- declarations shared between translation units of libfdk_b200.
#pragma once
#include <string>

#include "common.h"

namespace fdk {

// FP64 3x4 projection matrix of CalculateProjMat for view angle a (geometry.cpp).
void projection_matrix(const fdk_geometry &g, double a, double *m);

// Device tables of one filter length (filter.cu).
struct FilterTables {
    int W = 0, log2W = 0;
    float2 *tw = nullptr;
    float2 *twp = nullptr;  // per FFT pass and group, the group's twiddles (optional)
    float *hb = nullptr;
    // the copies go through a private set-up stream that the call waits for (bounded)
    int create(const double *H, int W_);
    void release();
};

// Fused cosine weight + pad + ramp filter + crop + layout store (filter.cu).
int filter_views(const float *src, int src_pitch, long long src_vstride, void *dst, int dst_pitch,
                 long long dst_vstride, const float *cos, int cos_pitch, const FilterTables &t, int nu, int nv,
                 int pad_n, int n_views, int layout, int dtype, cudaStream_t st, float out_scale = 1.0f,
                 unsigned int *overflow = nullptr);

// Projection-folder files (io.cpp): folder + "img%04d.raw" % file_index, and count views
// (files (first + i) * step + start, sizes checked first) read by `threads` host threads.
std::string proj_file_path(const char *folder, long long file_index);
int read_views(const char *folder, int nu, int nv, long long first, long long count, int step, int start, float *dst,
               int threads);

}  // namespace fdk
