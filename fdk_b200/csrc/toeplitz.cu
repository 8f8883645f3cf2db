// toeplitz.cu -- the FDK row filter as a GEMM on the 5th-generation tensor cores.
//
// The fused filter of filter.cu (pad with edge means, ramp/window by FFT of length W, crop) is a
// linear map of each cosine-weighted row x (nu samples): y = M x.  With the circular kernel
// hc = IDFT(H) (the response of the FFT path, ÷W included),
//   M[u][c] = hc[(u - c) mod W]
//           + [c < pad_n]      (1/pad_n) sum_{k < off}       hc[(off + u - k) mod W]
//           + [c >= nu - pad_n] (1/pad_n) sum_{k >= off + nu} hc[(off + u - k) mod W]
// (off = (W - nu) / 2; the pads are means of the first / last pad_n samples, Filterlib/
// FilterLib.h:26-46 and cudaFftFilter.cu kernelPad).  M is built once in FP64 on the host and
// stored FP16 or BF16; a batch of views is then one GEMM  Y[R][nu] = X[R][nu] . M^T  with R =
// views x nv rows, FP16/BF16 operands and FP32 accumulation (a Toeplitz row-GEMM on the tensor
// cores).  The ramp filter cancels most of its input, so
// 16-bit input rounding shows up ~10x larger in its output; the split mode keeps the operands'
// low parts too, x = x_hi + x_lo and M = M_hi + M_lo, and sums x_hi M_hi + x_lo M_hi + x_hi M_lo
// in the same GEMM with K = 3 nu (three times the FLOPs, close to FP32 accuracy).
//
// GEMM kernel (sm_100a, one CTA per SM, persistent over 128 x 256 output tiles):
//   warp 0  TMA producer: A (128 rows x 64 K) and B (256 rows x 64 K) boxes with 128-byte
//           swizzle into a 4-stage ring, completion by mbarrier expect_tx;
//   warp 1  allocates 512 TMEM columns (two 128 x 256 FP32 accumulators) and one thread issues
//           tcgen05.mma (M 128, N 256, K 16; four per 64-wide K chunk), releasing each stage
//           with tcgen05.commit and handing a finished accumulator to the epilogue the same way;
//   warps 2-5 epilogue: tcgen05.ld of their 32 TMEM lanes (32 columns at a time), FP16 out.
// The accumulators are double-buffered, so the epilogue of one tile overlaps the MMAs of the
// next.  Every mbarrier wait is bounded (10 s of %globaltimer); on timeout the CTA sets the
// device error word, drains what it issued and frees its TMEM before returning.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "common.h"
#include "internal.h"

namespace fdk {
namespace tpz {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4;
constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int THREADS = 192;
constexpr int TMEM_COLS = 512;
constexpr unsigned long long kWaitNs = 10ull * 1000 * 1000 * 1000;
constexpr int XBUF_BYTES = 2 * 4 * 32 * 32 * 2;  // epilogue pair exchange: 2 buffers x 4 warps x 32 x 32 FP16
constexpr size_t SMEM_BYTES = 1024 + STAGES * STAGE_BYTES + 256 + XBUF_BYTES;  // slack, ring, barriers, exchange

__device__ __forceinline__ unsigned su32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long gtime() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void bar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void bar_arrive(unsigned bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// bounded wait for the phase of the given parity; false after kWaitNs
__device__ __forceinline__ bool bar_wait(unsigned bar, unsigned parity) {
    unsigned long long t0 = 0;
    for (long long i = 0;; i++) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 63) == 0) {
            const unsigned long long t = gtime();
            if (i == 0) t0 = t;
            else if (t - t0 > kWaitNs) return false;
        }
    }
}
__device__ __forceinline__ void tma_2d(unsigned dst, const CUtensorMap *map, int x, int y, unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major operand, 128-byte swizzle, rows of 128 bytes in
// 1024-byte 8-row atoms.  Fields: start >> 4 [0,14), leading offset >> 4 [16,30) (1: unused
// for swizzled K-major), stride offset >> 4 [32,46) (1024 B between 8-row groups), version 1
// [46,48), base offset 0 [49,52), layout 2 = SWIZZLE_128B [61,64).
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr) {
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | (1ull << 16) | ((unsigned long long)(1024 >> 4) << 32) |
           (1ull << 46) | (2ull << 61);
}
// Instruction descriptor, kind::f16: D F32 [4,6) = 1, A/B format [7,10)/[10,13) (0 F16, 1 BF16),
// K-major A and B (bits 15, 16 = 0), N >> 3 at [17,23), M >> 4 at [24,29).
__host__ __device__ constexpr unsigned instr_desc(bool bf16) {
    return (1u << 4) | ((bf16 ? 1u : 0u) << 7) | ((bf16 ? 1u : 0u) << 10) | ((unsigned)(BN >> 3) << 17) |
           ((unsigned)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned idesc,
                                     unsigned accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(
            tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(unsigned bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 32 lanes x 32 consecutive FP32 columns of TMEM into registers
__device__ __forceinline__ void tmem_ld32(unsigned taddr, float (&v)[32]) {
    unsigned r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

struct GemmArgs {
    __half *out;        // ROWS: R x N FP16 (row pitch N); MIRROR: views x N x nv FP16 pairs
    int R, N, K;        // rows, output columns (= nu), reduction length (= nu x terms)
    int a_cols;         // stored A columns (nu, or 2 nu for hi | lo); the K segment at 2 nu re-reads hi
    int mirror, nv;     // MIRROR output: each 128-row tile is rows v0..v0+63 and nv-64-v0..nv-1-v0
    float out_scale;
    unsigned *err;      // device error word
    unsigned *overflow; // set when a scaled output leaves the FP16 range
};

template <bool BF16>
__global__ void __launch_bounds__(THREADS, 1) toeplitz_gemm_kernel(const __grid_constant__ CUtensorMap map_a,
                                                                    const __grid_constant__ CUtensorMap map_b,
                                                                    GemmArgs g) {
    extern __shared__ unsigned char smem_raw[];
    const unsigned raw = su32(smem_raw);
    const unsigned base = (raw + 1023u) & ~1023u;  // 128-byte swizzle atoms need 1024-byte alignment
    unsigned char *smem = smem_raw + (base - raw);
    const unsigned bars = base + STAGES * STAGE_BYTES;
    // barriers: full[S], empty[S], acc_full[2], acc_empty[2], fin (8 bytes each); at +128 the
    // TMEM base word and the abort flag
    const unsigned full0 = bars, empty0 = bars + 8 * STAGES, accf0 = bars + 16 * STAGES, acce0 = accf0 + 16;
    const unsigned fin = acce0 + 16;
    static_assert(8 * (2 * STAGES + 5) <= 128, "barrier block");
    unsigned *tmem_word = reinterpret_cast<unsigned *>(smem + STAGES * STAGE_BYTES + 128);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_word + 1);
    unsigned *xbuf = reinterpret_cast<unsigned *>(smem + STAGES * STAGE_BYTES + 256);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n_tiles_n = g.N / BN, n_tiles = (g.R / BM) * n_tiles_n, n_k = g.K / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            bar_init(full0 + 8 * s, 1);
            bar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; b++) {
            bar_init(accf0 + 8 * b, 1);
            bar_init(acce0 + 8 * b, 4);  // one arrival per epilogue warp
        }
        bar_init(fin, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_word)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tmem_word;

    if (warp == 0) {
        // ---------------- TMA producer (one thread)
        if (lane == 0) {
            int it = 0;
            for (int t = blockIdx.x; t < n_tiles && !*abort_flag; t += gridDim.x) {
                const int tm = t / n_tiles_n, tn = t % n_tiles_n;
                for (int kc = 0; kc < n_k; kc++, it++) {
                    const int s = it % STAGES;
                    if (it >= STAGES && !bar_wait(empty0 + 8 * s, ((it / STAGES) + 1) & 1)) {
                        *abort_flag = 1;
                        break;
                    }
                    const unsigned sa = base + s * STAGE_BYTES, sb = sa + A_BYTES;
                    const int xa = (kc * BK) % g.a_cols;
                    int r0 = tm * BM, r1 = r0 + BM / 2;  // two 64-row boxes per A tile
                    if (g.mirror) {
                        const int blocks = g.nv / BM, f = tm / blocks, v0 = (tm % blocks) * (BM / 2);
                        r0 = f * g.nv + v0;
                        r1 = f * g.nv + g.nv - BM / 2 - v0;
                    }
                    bar_expect_tx(full0 + 8 * s, STAGE_BYTES);
                    tma_2d(sa, &map_a, xa, r0, full0 + 8 * s);
                    tma_2d(sa + A_BYTES / 2, &map_a, xa, r1, full0 + 8 * s);
                    tma_2d(sb, &map_b, kc * BK, tn * BN, full0 + 8 * s);
                }
            }
            // drain: every issued stage must have landed before the CTA may exit
            for (int k = (it > STAGES ? it - STAGES : 0); k < it; k++) bar_wait(full0 + 8 * (k % STAGES), (k / STAGES) & 1);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer (one thread)
        if (lane == 0) {
            constexpr unsigned idesc = instr_desc(BF16);
            int it = 0, tile_i = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x, tile_i++) {
                const int b = tile_i & 1;
                if (tile_i >= 2 && !bar_wait(acce0 + 8 * b, ((tile_i >> 1) + 1) & 1)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const unsigned d = tmem + (unsigned)(b * BN);
                for (int kc = 0; kc < n_k; kc++, it++) {
                    const int s = it % STAGES;
                    if (!bar_wait(full0 + 8 * s, (it / STAGES) & 1) || *abort_flag) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const unsigned sa = base + s * STAGE_BYTES, sb = sa + A_BYTES;
#pragma unroll
                    for (int kk = 0; kk < BK / 16; kk++)  // K = 16 per MMA: 32 bytes into the swizzled row
                        umma(d, smem_desc(sa + kk * 32), smem_desc(sb + kk * 32), idesc, (kc | kk) ? 1u : 0u);
                    umma_commit(empty0 + 8 * s);  // stage free once these MMAs have read it
                }
                if (!ok) break;
                umma_commit(accf0 + 8 * b);  // accumulator b complete
            }
            if (!ok) {
                *abort_flag = 1;
                atomicOr(g.err, 1u);
            }
            // every MMA this thread issued must finish before TMEM is released
            umma_commit(fin);
            bar_wait(fin, 0);
        }
    } else {
        // ---------------- epilogue: warps 2..5; TMEM lanes 32 * (warp % 4) ..
        const int q = warp & 3;
        const int row_in_tile = 32 * q + lane;
        int tile_i = 0;
        for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, tile_i++) {
            const int b = tile_i & 1;
            const bool ready = bar_wait(accf0 + 8 * b, (tile_i >> 1) & 1) && !*abort_flag;
            // one decision for all four epilogue warps (they meet at named barrier 1 below, and
            // tcgen05.ld is .sync.aligned): AND-reduction over the 128 epilogue threads
            unsigned all_ready;
            asm volatile(
                "{\n .reg .pred p, r;\n setp.ne.b32 p, %1, 0;\n bar.red.and.pred r, 1, 128, p;\n selp.b32 %0, 1, 0, r;\n}"
                : "=r"(all_ready)
                : "r"((unsigned)ready)
                : "memory");
            if (!all_ready) break;
            tc_fence_after();
            const int tm = t / n_tiles_n, tn = t % n_tiles_n;
            // ROWS: this lane's output row; MIRROR: its detector row vr in view f (TMEM lanes
            // 0..63 hold rows v0 + i, lanes 64..127 rows nv - 64 - v0 + j; lane i pairs with 127 - i)
            __half *orow = g.out + (long long)(tm * BM + row_in_tile) * g.N + tn * BN;
            long long mbase = 0;
            int vr = 0;
            if (g.mirror) {
                const int blocks = g.nv / BM, f = tm / blocks, v0 = (tm % blocks) * (BM / 2);
                vr = row_in_tile < BM / 2 ? v0 + row_in_tile : g.nv - BM - v0 + row_in_tile;
                mbase = (long long)f * g.N * g.nv + (long long)(tn * BN) * g.nv + vr;
            }
#pragma unroll 1
            for (int c = 0; c < BN / 32; c++) {
                float v[32];
                tmem_ld32(tmem + ((unsigned)(32 * q) << 16) + (unsigned)(b * BN + 32 * c), v);
                unsigned packed[16];
                bool over = false;
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const float x0 = v[2 * i] * g.out_scale, x1 = v[2 * i + 1] * g.out_scale;
                    over |= !(fabsf(x0) <= 65504.f) || !(fabsf(x1) <= 65504.f);
                    const __half2 h = __floats2half2_rn(x0, x1);
                    packed[i] = *reinterpret_cast<const unsigned *>(&h);
                }
                if (over && g.overflow) atomicOr(g.overflow, 1u);
                if (!g.mirror) {
                    uint4 *dst = reinterpret_cast<uint4 *>(orow + 32 * c);
#pragma unroll
                    for (int i = 0; i < 4; i++)
                        dst[i] = make_uint4(packed[4 * i], packed[4 * i + 1], packed[4 * i + 2], packed[4 * i + 3]);
                    continue;
                }
                // exchange with the partner row (warp 3 - q, lane 31 - lane) through shared memory
                unsigned *xb = xbuf + (c & 1) * (4 * 32 * 16);
#pragma unroll
                for (int i = 0; i < 16; i++) xb[(q * 32 + lane) * 16 + ((i + lane) & 15)] = packed[i];
                asm volatile("bar.sync 1, 128;" ::: "memory");  // the four epilogue warps
                const unsigned *pb = xb + ((3 - q) * 32 + (31 - lane)) * 16;
                __half2 *dst = reinterpret_cast<__half2 *>(g.out) + mbase + (long long)(32 * c) * g.nv;
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const unsigned o = packed[i], pp = pb[(i + 31 - lane) & 15];
                    const __half2 mine = *reinterpret_cast<const __half2 *>(&o);
                    const __half2 part = *reinterpret_cast<const __half2 *>(&pp);
                    // element (u, vr) = (row vr, row nv-1-vr): consecutive lanes, consecutive vr
                    dst[(long long)(2 * i) * g.nv] = __lows2half2(mine, part);
                    dst[(long long)(2 * i + 1) * g.nv] = __highs2half2(mine, part);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) bar_arrive(acce0 + 8 * b);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

template <typename T>
__device__ __forceinline__ T to16(float x) {
    if constexpr (std::is_same<T, __half>::value) return __float2half_rn(x);
    else return __float2bfloat16_rn(x);
}
template <typename T>
__device__ __forceinline__ float from16(T x) {
    if constexpr (std::is_same<T, __half>::value) return __half2float(x);
    else return __bfloat162float(x);
}

// A operand rows: x = p * cos * in_scale (R rows of nu), stored as [hi] or [hi | lo] (split;
// the GEMM's third K segment reads hi again), hi = round16(x), lo = round16(x - hi); eight
// consecutive samples per thread (nu % 8 == 0), 128-bit loads and stores.
template <typename T>
__global__ void weight_convert_kernel(const float *__restrict__ src, const float *__restrict__ cos, T *__restrict__ dst,
                                      long long n8, int nu, int nv, float in_scale, int split) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n8; g += (long long)gridDim.x * blockDim.x) {
        const long long i = 8 * g, row = i / nu;
        const int c = (int)(i - row * nu), v = (int)(row % nv);
        const float4 *s4 = reinterpret_cast<const float4 *>(src + i);
        const float4 *c4 = reinterpret_cast<const float4 *>(cos + (long long)v * nu + c);
        float x[8];
        {
            const float4 a = s4[0], b = s4[1];
            const float4 ca = cos ? c4[0] : make_float4(1.f, 1.f, 1.f, 1.f);
            const float4 cb = cos ? c4[1] : make_float4(1.f, 1.f, 1.f, 1.f);
            x[0] = a.x * ca.x * in_scale, x[1] = a.y * ca.y * in_scale, x[2] = a.z * ca.z * in_scale;
            x[3] = a.w * ca.w * in_scale, x[4] = b.x * cb.x * in_scale, x[5] = b.y * cb.y * in_scale;
            x[6] = b.z * cb.z * in_scale, x[7] = b.w * cb.w * in_scale;
        }
        T hi[8], lo[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            hi[k] = to16<T>(x[k]);
            lo[k] = to16<T>(x[k] - from16<T>(hi[k]));
        }
        T *d = dst + row * (long long)nu * (split ? 2 : 1) + c;
        *reinterpret_cast<uint4 *>(d) = *reinterpret_cast<const uint4 *>(hi);
        if (split) *reinterpret_cast<uint4 *>(d + nu) = *reinterpret_cast<const uint4 *>(lo);
    }
}

}  // namespace tpz

// --------------------------------------------------------------------------------------------
// host side
// --------------------------------------------------------------------------------------------
namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encoder() {
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

// 2-D map of a row-major [rows][cols] 16-bit matrix, box 64 x box_rows, 128-byte swizzle
int encode_2d(CUtensorMap *map, const void *base, long long rows, long long cols, int box_rows, bool bf16) {
    EncodeTiledFn enc = encoder();
    if (!enc) return fail(FDK_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    const cuuint32_t box[2] = {(cuuint32_t)tpz::BK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                           const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(FDK_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return FDK_OK;
}

}  // namespace

// FP64 filter matrix of the fused FFT filter (see the file header), row-major M[u][c].
void toeplitz_matrix(const double *H, int W, int nu, int pad_n, std::vector<double> &M) {
    // circular kernel hc[n] = (1/W) sum_k H[k] cos(2 pi k n / W)  (H real and even)
    std::vector<double> hc(W);
    for (int n = 0; n < W; n++) {
        double s = 0;
        for (int k = 0; k < W; k++) s += H[k] * std::cos(2.0 * M_PI * (double)((long long)k * n % W) / W);
        hc[n] = s / W;
    }
    const int off = (W - nu) / 2;
    M.assign((size_t)nu * nu, 0.0);
    for (int u = 0; u < nu; u++) {
        double left = 0, right = 0;
        for (int k = 0; k < off; k++) left += hc[((off + u - k) % W + W) % W];
        for (int k = off + nu; k < W; k++) right += hc[((off + u - k) % W + W) % W];
        double *row = &M[(size_t)u * nu];
        for (int c = 0; c < nu; c++) row[c] = hc[((u - c) % W + W) % W];
        for (int c = 0; c < pad_n; c++) row[c] += left / pad_n;
        for (int c = nu - pad_n; c < nu; c++) row[c] += right / pad_n;
    }
}

}  // namespace fdk

using namespace fdk;

struct fdk_toeplitz {
    int device = 0;
    int nu = 0, nv = 0, W = 0, pad = 4;
    bool bf16 = false;
    int terms = 1;              // 1 plain; 3: (x_hi, x_lo, x_hi) . (M_hi, M_hi, M_lo)
    float in_scale = 1.f;
    float m_unscale = 1.f;      // M is stored times 2^e (FP16 normal range); outputs times 2^-e
    float *d_cos = nullptr;
    void *d_M = nullptr;        // nu x nu, 16-bit
    void *d_x = nullptr;        // views x nv x (nu or 2 nu), 16-bit weighted input (hi | lo)
    long long cap_views = 0;
    unsigned *d_err = nullptr;  // [0] device error word, [1] FP16 overflow
    int sms = 0;
};

extern "C" {

int fdk_toeplitz_create(fdk_toeplitz **out, const float *cos_table, const double *H, int64_t nu, int64_t nv,
                        int64_t W, int32_t pad_edge, int32_t bf16, int32_t split, float in_scale, int32_t device) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(out && H, "NULL argument");
    *out = nullptr;
    FDK_CHECK_ARG(nu % tpz::BN == 0 && nu >= tpz::BN && nu <= 8192, "nu must be a multiple of %d (got %lld)", tpz::BN,
                  (long long)nu);
    FDK_CHECK_ARG(nv % tpz::BM == 0, "nv must be a multiple of %d (got %lld)", tpz::BM, (long long)nv);
    FDK_CHECK_ARG(W >= nu && (W & (W - 1)) == 0 && W <= 16384, "bad filter length W");
    FDK_CHECK_ARG(pad_edge >= 1 && pad_edge <= 4, "pad_edge must be 1..4");
    DeviceGuard dg(device);
    FDK_TRY(dg.status);
    int major = 0, minor = 0;
    FDK_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    FDK_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
    if (major != 10) return fail(FDK_ERR_UNSUPPORTED, "the tensor-core filter needs an sm_100 GPU");
    fdk_toeplitz *h = new fdk_toeplitz();
    h->device = device;
    h->nu = (int)nu;
    h->nv = (int)nv;
    h->W = (int)W;
    h->pad = pad_edge;
    h->bf16 = bf16 != 0;
    h->terms = split ? 3 : 1;
    h->in_scale = in_scale;
    std::vector<double> M;
    toeplitz_matrix(H, (int)W, (int)nu, pad_edge, M);
    // FP16: scale M by a power of two so its largest entry sits near 2^14; the kernel's small
    // far-off-diagonal taps (the ramp's low-frequency response) then stay out of the subnormal
    // range.  The output scale divides the same power out exactly.
    double mmax = 0;
    for (double x : M) mmax = std::max(mmax, std::fabs(x));
    int e = 0;
    if (!h->bf16 && mmax > 0) e = 14 - (int)std::ceil(std::log2(mmax));
    h->m_unscale = (float)std::ldexp(1.0, -e);
    // B rows: [M_hi] or [M_hi | M_hi | M_lo] (K = terms * nu)
    const int T = h->terms;
    std::vector<unsigned short> m16((size_t)nu * nu * T);
    auto enc16 = [&](double x, double *back) -> unsigned short {
        if (h->bf16) {
            const __nv_bfloat16 b = __float2bfloat16_rn((float)x);
            *back = (double)__bfloat162float(b);
            return *reinterpret_cast<const unsigned short *>(&b);
        }
        const __half b = __float2half_rn((float)x);
        *back = (double)__half2float(b);
        return *reinterpret_cast<const unsigned short *>(&b);
    };
    for (long long u = 0; u < nu; u++)
        for (long long c = 0; c < nu; c++) {
            const double x = std::ldexp(M[(size_t)u * nu + c], e);
            double hi = 0, lo = 0;
            const unsigned short hb = enc16(x, &hi);
            unsigned short *row = &m16[(size_t)u * nu * T];
            row[c] = hb;
            if (T == 3) {
                row[nu + c] = hb;
                row[2 * nu + c] = enc16(x - hi, &lo);
            }
        }
    int s = FDK_OK;
    auto step = [&](cudaError_t e, const char *what) {
        if (s == FDK_OK && e != cudaSuccess) s = cuda_status(e, what, __FILE__, __LINE__);
    };
    SetupStream ss;  // set-up copies: a private stream, waited for below (no device-wide sync)
    s = ss.open();
    if (s == FDK_OK) step(cudaMalloc(&h->d_M, m16.size() * 2), "cudaMalloc M");
    if (s == FDK_OK)
        step(cudaMemcpyAsync(h->d_M, m16.data(), m16.size() * 2, cudaMemcpyHostToDevice, ss.st), "copy M");
    if (s == FDK_OK && cos_table) {
        step(cudaMalloc(&h->d_cos, sizeof(float) * nu * nv), "cudaMalloc cos");
        if (s == FDK_OK)
            step(cudaMemcpyAsync(h->d_cos, cos_table, sizeof(float) * nu * nv, cudaMemcpyHostToDevice, ss.st),
                 "copy cos");
    }
    if (s == FDK_OK) step(cudaMalloc(&h->d_err, 2 * sizeof(unsigned)), "cudaMalloc err");
    if (s == FDK_OK) step(cudaMemsetAsync(h->d_err, 0, 2 * sizeof(unsigned), ss.st), "memset err");
    if (s == FDK_OK) s = ss.finish("fdk_toeplitz_create");
    if (s == FDK_OK) step(cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    if (s == FDK_OK)
        step(cudaFuncSetAttribute(tpz::toeplitz_gemm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)tpz::SMEM_BYTES),
             "smem attribute");
    if (s == FDK_OK)
        step(cudaFuncSetAttribute(tpz::toeplitz_gemm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)tpz::SMEM_BYTES),
             "smem attribute");
    if (s != FDK_OK) {
        fdk_toeplitz_destroy(h);
        return s;
    }
    *out = h;
    return FDK_OK;
    FDK_ABI_END
}

int fdk_toeplitz_run_device(fdk_toeplitz *h, const float *dev_src, void *dev_dst, int64_t n_views, int32_t layout,
                            float out_scale, void *stream) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && dev_src && dev_dst && n_views > 0, "bad arguments");
    FDK_CHECK_ARG(layout == FDK_LAYOUT_ROWS || layout == FDK_LAYOUT_MIRROR, "layout must be ROWS or MIRROR (FP16)");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    cudaStream_t st = (cudaStream_t)stream;
    const long long frame = (long long)h->nu * h->nv;
    if (n_views > h->cap_views) {
        FDK_CUDA(cudaStreamSynchronize(st));
        if (h->d_x) cudaFree(h->d_x);
        h->d_x = nullptr;
        h->cap_views = 0;
        FDK_CUDA(cudaMalloc(&h->d_x, 2 * frame * n_views * (h->terms > 1 ? 2 : 1)));
        h->cap_views = n_views;
    }
    const long long n8 = frame * n_views / 8;
    FDK_CHECK_ARG(((uintptr_t)dev_src & 15) == 0, "views must start on a 16-byte boundary");
    const int split = h->terms > 1 ? 1 : 0;
    if (h->bf16)
        tpz::weight_convert_kernel<__nv_bfloat16><<<148 * 16, 256, 0, st>>>(
            dev_src, h->d_cos, (__nv_bfloat16 *)h->d_x, n8, h->nu, h->nv, h->in_scale, split);
    else
        tpz::weight_convert_kernel<__half><<<148 * 16, 256, 0, st>>>(dev_src, h->d_cos, (__half *)h->d_x, n8, h->nu,
                                                                     h->nv, h->in_scale, split);
    FDK_CUDA(cudaGetLastError());
    const long long R = (long long)h->nv * n_views;
    FDK_CHECK_ARG(R < (1ll << 31), "too many rows");
    CUtensorMap ma, mb;
    const long long K = (long long)h->nu * h->terms, a_cols = (long long)h->nu * (h->terms > 1 ? 2 : 1);
    FDK_TRY(encode_2d(&ma, h->d_x, R, a_cols, tpz::BM / 2, h->bf16));
    FDK_TRY(encode_2d(&mb, h->d_M, h->nu, K, tpz::BN, h->bf16));
    tpz::GemmArgs g;
    g.out = (__half *)dev_dst;
    g.R = (int)R;
    g.N = h->nu;
    g.K = (int)K;
    g.a_cols = (int)a_cols;
    g.mirror = layout == FDK_LAYOUT_MIRROR ? 1 : 0;
    g.nv = h->nv;
    g.out_scale = out_scale * h->m_unscale;
    g.err = h->d_err;
    g.overflow = h->d_err + 1;
    const long long tiles = (R / tpz::BM) * (h->nu / tpz::BN);
    const int grid = (int)std::min<long long>(tiles, h->sms);
    if (h->bf16)
        tpz::toeplitz_gemm_kernel<true><<<grid, tpz::THREADS, tpz::SMEM_BYTES, st>>>(ma, mb, g);
    else
        tpz::toeplitz_gemm_kernel<false><<<grid, tpz::THREADS, tpz::SMEM_BYTES, st>>>(ma, mb, g);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
    FDK_ABI_END
}

int fdk_toeplitz_check(fdk_toeplitz *h) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(h != nullptr, "NULL handle");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    unsigned e[2] = {0, 0};
    FDK_CUDA(cudaMemcpy(e, h->d_err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e[0]) return fail(FDK_ERR_DEVICE_CHECK, "tensor-core filter: a pipeline wait timed out");
    if (e[1]) return fail(FDK_ERR_DEVICE_CHECK, "tensor-core filter: outputs exceeded the FP16 range");
    return FDK_OK;
    FDK_ABI_END
}

int fdk_toeplitz_matrix(const double *H, int64_t W, int64_t nu, int32_t pad_edge, double *out) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(H && out && nu > 0 && W >= nu && pad_edge >= 1 && pad_edge <= 4, "bad arguments");
    std::vector<double> M;
    toeplitz_matrix(H, (int)W, (int)nu, pad_edge, M);
    std::copy(M.begin(), M.end(), out);
    return FDK_OK;
    FDK_ABI_END
}

int fdk_toeplitz_destroy(fdk_toeplitz *h) {
    if (!h) return FDK_OK;
    DeviceGuard dg(h->device);
    cudaDeviceSynchronize();
    if (h->d_cos) cudaFree(h->d_cos);
    if (h->d_M) cudaFree(h->d_M);
    if (h->d_x) cudaFree(h->d_x);
    if (h->d_err) cudaFree(h->d_err);
    delete h;
    return FDK_OK;
}

}  // extern "C"
