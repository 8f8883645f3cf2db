// filter_noalloc.cu -- fdk_filter_row_real32_noalloc: the row filter of fdk_filter_row_real32
// without any device allocation.
//
// fdk_filter_row_real32 allocates two small device tables per call (the FFT twiddles and the
// bit-reversed, 1/W-scaled response) and frees them again.  Some callers cannot allocate device
// memory at that point: applications that reserve the whole device budget up front and hand
// out memory themselves, and processing loops that must not call cudaMalloc/cudaFree because
// those calls can synchronise the device and stall every other stream.  For them this entry
// point keeps the tables in a fixed file-scope device array and builds them there on the GPU.
//
// Limits and sharing rules:
//   * W <= kNoAllocMaxW (4096), the largest filter length of the library; larger W is rejected
//     with FDK_ERR_INVALID_ARG.  The array holds W/2 float2 twiddles + W floats: 32 KiB.
//   * Every loaded process holds the 32 KiB array on every GPU that loads the library, until exit.
//   * All calls in the process share the one array per device.  Each call rewrites every entry it
//     reads before its filter kernel runs (nothing needs to start at zero), and the call returns
//     only after its kernels finish; calls that overlap on the GPU (several host threads calling
//     at once on one device) race on the tables and must be serialised by the caller.
//   * Set-up: every call looks up the array's device address on the caller's current device
//     (cudaGetSymbolAddress, return code checked) instead of keeping one from an earlier call,
//     so a pointer never outlives the context it was taken in (cudaDeviceReset, another
//     context on the same device).  The first call on a device also loads the library's device
//     code there; make that first call before any stream capture begins.
//   * Kernels run on the legacy default stream and the call waits for that stream only (the
//     reference's FilterRow_Real32 is synchronous too), not for the whole device.
#include <cuda_runtime.h>

#include "common.h"
#include "internal.h"

namespace fdk {

constexpr int kNoAllocMaxW = 4096;

// W/2 float2 twiddles followed by W floats of the bit-reversed response: 4096 * 8 bytes.
static __device__ __align__(256) float2 g_filter_scratch[kNoAllocMaxW];

// tw[k] = exp(-2 pi i k / W) (FP64 sincospi, rounded), hb[p] = H[bitrev(p)] / W.
__global__ void build_filter_tables_kernel(const float *__restrict__ H, int W, int log2W, float2 *tw, float *hb) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < W; k += gridDim.x * blockDim.x) {
        if (k < W / 2) {
            double s, c;
            sincospi(-2.0 * (double)k / (double)W, &s, &c);
            tw[k] = make_float2((float)c, (float)s);
        }
        const int r = (int)(__brev((unsigned)k) >> (32 - log2W));
        hb[k] = H[r] / (float)W;
    }
}

// The array's device address on the current device.  A host-side lookup, repeated per call.
static int scratch_address(float2 **out) {
    void *p = nullptr;
    FDK_CUDA(cudaGetSymbolAddress(&p, g_filter_scratch));
    FDK_CHECK_ARG(p != nullptr, "no device address for the filter tables");
    *out = static_cast<float2 *>(p);
    return FDK_OK;
}

}  // namespace fdk

using namespace fdk;

extern "C" int fdk_filter_row_real32_noalloc(const fdk_dataref *src, fdk_dataref *dst, const fdk_dataref *filter) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(src && dst && filter && src->data && dst->data && filter->data, "NULL argument");
    FDK_CHECK_ARG(src->width == dst->width && src->height == dst->height && src->depth <= dst->depth,
                  "src/dst shapes differ (FilterRow, cudaFftFilter.cu:302-305)");
    FDK_CHECK_ARG(filter->height == 1 || filter->height == 0, "filter must be one row");
    const int W = filter->width;
    FDK_CHECK_ARG(W >= 2 && (W & (W - 1)) == 0, "filter length W=%d must be a power of two", W);
    FDK_CHECK_ARG(W <= kNoAllocMaxW,
                  "filter length W=%d exceeds the no-allocation limit of %d (use fdk_filter_row_real32)", W,
                  kNoAllocMaxW);
    FDK_CHECK_ARG(W >= src->width && src->width >= 3 && src->height > 0 && src->depth > 0 && src->height <= 131070 &&
                      src->depth <= 65535 && src->pitch >= src->width && dst->pitch >= dst->width,
                  "shape out of range (need width >= 3, W >= width)");
    float2 *scratch = nullptr;
    FDK_TRY(scratch_address(&scratch));
    FilterTables t;  // points into the static array; never created or released here
    t.W = W;
    t.log2W = 0;
    while ((1 << t.log2W) < W) t.log2W++;
    t.tw = scratch;
    t.hb = reinterpret_cast<float *>(scratch + W / 2);
    build_filter_tables_kernel<<<(W + 255) / 256, 256, 0, cudaStreamLegacy>>>(filter->data, W, t.log2W, t.tw, t.hb);
    FDK_CUDA(cudaGetLastError());
    FDK_TRY(filter_views(src->data, src->pitch, (long long)src->pitch * src->height, dst->data, dst->pitch,
                         (long long)dst->pitch * dst->height, nullptr, 0, t, src->width, src->height, 3, src->depth,
                         FDK_LAYOUT_ROWS, FDK_DTYPE_F32, cudaStreamLegacy));
    FDK_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
    return FDK_OK;
    FDK_ABI_END
}
