// tma_common.cuh -- mbarrier and TMA helpers shared by the staged backprojection kernels
// (bp_tma.cuh, rtk.cu): bounded mbarrier waits, 3-D tile loads, and the driver's tensor-map
// encoder reached through the runtime.
#pragma once
#include <cuda.h>

#include "common.h"

namespace fdk {

constexpr long long kWaitLimit = 1ll << 26;
// Sleep between a producer warp's polls of a stage's empty barrier (tuning macro; 0 = spin).  The
// MIXED staged kernel at 2048^3 measured the same with 256 ns (3167 against 3171 GUPS): try_wait
// already suspends the polling thread for a while before it reports an incomplete phase.
#ifndef FDK_PRODUCER_SLEEP_NS
#define FDK_PRODUCER_SLEEP_NS 0
#endif
constexpr unsigned long long kWaitNs = 10ull * 1000 * 1000 * 1000;  // 10 s
constexpr unsigned kErrTimeout = 1u;
constexpr unsigned kErrFootprint = 2u;  // a tile's footprint did not fit its shared-memory box

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for the phase with the given parity: gives up after limit_ns of wall time
// (default kWaitNs) or kWaitLimit polls; false on timeout.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, unsigned long long limit_ns = kWaitNs) {
    unsigned long long t0 = 0;
    for (long long i = 0; i < kWaitLimit; i++) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 255) == 0) {
            const unsigned long long t = global_ns();
            if (i == 0) t0 = t;
            else if (t - t0 > limit_ns) return false;
        }
    }
    return false;
}
// The same wait for a warp that usually finds the phase incomplete (a producer waiting for
// consumers to free a stage): between polls it sleeps sleep_ns, so its polling does not take
// issue slots from the warps doing the work.
__device__ __forceinline__ bool mbar_wait_backoff(unsigned bar, unsigned parity, unsigned long long limit_ns,
                                                  unsigned sleep_ns) {
    unsigned long long t0 = 0;
    for (long long i = 0; i < kWaitLimit; i++) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (sleep_ns) __nanosleep(sleep_ns);
        if ((i & 15) == 0) {
            const unsigned long long t = global_ns();
            if (i == 0) t0 = t;
            else if (t - t0 > limit_ns) return false;
        }
    }
    return false;
}
__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap *map, int x, int y, int z, unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link, so the
// library still loads on machines without a driver).
inline EncodeTiledFn tensor_map_encoder() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

}  // namespace fdk
