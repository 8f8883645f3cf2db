// ref_gpu_filter_harness.cu -- extern "C" entry points around the reference's
// cuFFT filter plugin, compiled in place for sm_100a by oracle/build_ref.sh.
// TEST INFRASTRUCTURE ONLY (parity checker for the product's filter kernel).
//
//   refg_filter  CorrectImage_Real32 then FilterRow_Real32
//                (FilterlibCufft/cudaFftFilter.cuh:6-8, cudaFftFilter.cu:283-392),
//                the sequence FilterProjImage runs per batch (cudaFftFilter.cu:416-433)
#include "FilterlibCufft/cudaFftFilter.cu"

// d_src/d_dst: device, `depth` views of height rows x width columns (pitch = width).
// d_table: device, height x width.  d_filter: device, W values.  Views are
// cos-weighted in place in d_src, as FilterProjImage does.
extern "C" int refg_filter(float* d_src, float* d_dst, const float* d_table, const float* d_filter,
                           int width, int height, int depth, int W) {
    try {
        DataRef<float> src(d_src, width, height, depth, width, 3);
        DataRef<float> dst(d_dst, width, height, depth, width, 3);
        DataRef<float> table(const_cast<float*>(d_table), width, height, 1, width, 2);
        DataRef<float> filt(const_cast<float*>(d_filter), W, 1, 1, W, 1);
        CorrectImage_Real32(src, table, src);
        FilterRow_Real32(src, dst, filt);
        cudaError_t e = cudaDeviceSynchronize();
        return e == cudaSuccess ? 0 : -3;
    } catch (...) {
        return -2;
    }
}
