/* ref_texture_shim.h -- force-included when compiling the reference's own CUDA
 * sources for the parity harness (oracle/build_ref.sh).  CUDA 12 removed the
 * host texture/surface-reference API; the reference only uses it in
 * GpuArray*::BindToTexture helpers (common/cudaLib.cuh:291-312, 630-660) that the
 * kernels under test never call.  These stand-ins keep those helpers compiling
 * and make any call fail with cudaErrorNotSupported. */
#pragma once
#include <cuda_runtime.h>
struct textureReference { int normalized; cudaTextureFilterMode filterMode;
                          cudaTextureAddressMode addressMode[3]; cudaChannelFormatDesc channelDesc; };
struct surfaceReference { cudaChannelFormatDesc channelDesc; };
template <class... A> inline cudaError_t cudaBindTexture(A...) { return cudaErrorNotSupported; }
template <class... A> inline cudaError_t cudaBindTexture2D(A...) { return cudaErrorNotSupported; }
template <class... A> inline cudaError_t cudaBindTextureToArray(A...) { return cudaErrorNotSupported; }
template <class... A> inline cudaError_t cudaUnbindTexture(A...) { return cudaErrorNotSupported; }
template <class... A> inline cudaError_t cudaBindSurfaceToArray(A...) { return cudaErrorNotSupported; }
