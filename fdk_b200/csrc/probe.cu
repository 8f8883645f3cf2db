// probe.cu -- on-device peak probes for the backprojection roofline (no reference
// counterpart).  The backprojection is bound by shared-memory bandwidth or FP32 issue, not by
// HBM or tensor cores, so its roofline denominators are measured here on the same GPU:
//   fdk_probe_smem:  128-bit shared-memory loads, conflict-free, all SMs -> GB/s
//   fdk_probe_fma:   independent FP32 FMA chains, all SMs -> TFLOP/s (2 flops per FMA)
#include "common.h"

namespace fdk {

__global__ void __launch_bounds__(1024) smem_probe_kernel(int iters, float *sink) {
    __shared__ float4 buf[2048];
    for (int i = threadIdx.x; i < 2048; i += blockDim.x) buf[i] = make_float4(i, i + 1, i + 2, i + 3);
    __syncthreads();
    float4 acc = make_float4(0, 0, 0, 0);
    int idx = threadIdx.x;
#pragma unroll 1
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const float4 v = buf[(idx + k * 64) & 2047];
            acc.x += v.x;
            acc.y += v.y;
            acc.z += v.z;
            acc.w += v.w;
        }
        idx ^= 32;
    }
    if (acc.x + acc.y + acc.z + acc.w == -1.0f) sink[threadIdx.x] = acc.x;
}

__global__ void __launch_bounds__(256) fma_probe_kernel(int iters, float *sink) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = threadIdx.x * 1e-3f + k;
    const float b = 0.999999f, c = 1e-7f;
#pragma unroll 1
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int r = 0; r < 16; r++)
#pragma unroll
            for (int k = 0; k < 8; k++) a[k] = fmaf(a[k], b, c);
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == -1.0f) sink[threadIdx.x] = s;
}

}  // namespace fdk

using namespace fdk;

extern "C" {

int fdk_probe_smem(int32_t device, double *gbs) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(gbs != nullptr, "NULL argument");
    DeviceGuard dg(device);
    FDK_TRY(dg.status);
    int sms = 0;
    FDK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    float *sink = nullptr;
    FDK_CUDA(cudaMalloc(&sink, 4096));
    cudaEvent_t e0, e1;
    FDK_CUDA(cudaEventCreate(&e0));
    FDK_CUDA(cudaEventCreate(&e1));
    const int iters = 4096, threads = 1024, blocks = sms * 2;
    smem_probe_kernel<<<blocks, threads>>>(64, sink);  // warm-up
    FDK_CUDA(cudaEventRecord(e0));
    smem_probe_kernel<<<blocks, threads>>>(iters, sink);
    FDK_CUDA(cudaEventRecord(e1));
    FDK_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    FDK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *gbs = (double)blocks * threads * iters * 16 * 16 / (ms * 1e-3) / 1e9;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return FDK_OK;
    FDK_ABI_END
}

int fdk_probe_fma(int32_t device, double *tflops) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(tflops != nullptr, "NULL argument");
    DeviceGuard dg(device);
    FDK_TRY(dg.status);
    int sms = 0;
    FDK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    float *sink = nullptr;
    FDK_CUDA(cudaMalloc(&sink, 4096));
    cudaEvent_t e0, e1;
    FDK_CUDA(cudaEventCreate(&e0));
    FDK_CUDA(cudaEventCreate(&e1));
    const int iters = 8192, threads = 256, blocks = sms * 8;
    fma_probe_kernel<<<blocks, threads>>>(64, sink);
    FDK_CUDA(cudaEventRecord(e0));
    fma_probe_kernel<<<blocks, threads>>>(iters, sink);
    FDK_CUDA(cudaEventRecord(e1));
    FDK_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    FDK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *tflops = (double)blocks * threads * iters * 16 * 8 * 2 / (ms * 1e-3) / 1e12;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return FDK_OK;
    FDK_ABI_END
}

}  // extern "C"
