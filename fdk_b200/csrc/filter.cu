// filter.cu -- fused FDK row filter for sm_100a: cosine pre-weight, constant edge pad,
// ramp/window filter by FFT, crop, and the store in the layout the backprojection reads.
//
// Reference semantics: FilterEngine::Filtering (Filterlib/FilterLib.h:167-196) and the cuFFT
// plugin (FilterlibCufft/cudaFftFilter.cu:14-61, 283-392).  One CTA filters two detector rows
// at once -- row r and its mirror row nv-1-r -- as the real and imaginary parts of one complex
// FFT of length W: with a real, even response H the two filtered rows come back as the real
// and imaginary parts of the inverse transform.  Pairing r with nv-1-r is what lets the same
// CTA emit the backprojection's mirror-pair layout directly.
//
// FFT: radix-2 decimation in frequency (natural -> bit-reversed order), pointwise multiply by
// H[bitrev(p)]/W, radix-2 decimation in time (bit-reversed -> natural), in shared memory.
// Three consecutive radix-2 stages run per pass in registers: the stages of a pass touch three
// adjacent index bits, so the 8 elements that differ only in those bits form a closed group.
// Every butterfly is the plain radix-2 one, so the arithmetic is that of the stage-by-stage
// transform, with a third of the shared-memory round trips and barriers.  Twiddles come from
// an FP64-computed table, rearranged per pass so that a group reads its own with vector loads.
//
// The backprojection's MIRROR layout is written by filter_mirror_kernel: a CTA filters G row
// pairs in turn, collects their outputs as an nu x G tile per side in shared memory, and writes
// each detector column's G consecutive elements as one 16-byte store.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "internal.h"

namespace fdk {

struct FilterArgs {
    const float *src;   // views of nv rows x nu, row pitch src_pitch, view stride src_vstride
    void *dst;          // output, layout dependent
    const float *cos;   // nv x nu (pitch cos_pitch) or nullptr
    const float2 *tw;   // W/2 twiddles exp(-2 pi i k / W)
    const float2 *twp;  // per pass and group, the group's twiddles (FilterTables::twp) or nullptr
    const float *hb;    // W: H[bitrev(p)] / W
    int nu, nv, W, log2W, off, pad_n;
    int src_pitch, dst_pitch, cos_pitch;
    long long src_vstride, dst_vstride;
    float out_scale;          // multiplies every output sample (FP16 range control)
    unsigned int *overflow;   // set to 1 when a scaled FP16 output exceeds the format (or NULL)
};

template <typename OUT>
__device__ __forceinline__ OUT to_out(const FilterArgs &a, float y) {
    if constexpr (sizeof(OUT) == 2) {
        const float s = y * a.out_scale;
        if (a.overflow && !(fabsf(s) <= 65504.f)) atomicOr(a.overflow, 1u);
        return __float2half_rn(s);
    } else {
        return y * a.out_scale;
    }
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// Weighted sample of row r at column c of the current view.
__device__ __forceinline__ float row_sample(const FilterArgs &a, const float *view, int r, int c) {
    float x = __ldg(view + (long long)r * a.src_pitch + c);
    if (a.cos) x *= __ldg(a.cos + (long long)r * a.cos_pitch + c);
    return x;
}

// Shared-memory position of element i of an FFT: i ^ ((i >> 4) & 15), a permutation inside each
// block of 16 float2.  Later DIF and early DIT passes read groups 8 or 64 elements apart, which
// in the plain layout fall into the same banks (up to 16-way conflicts); the swizzle spreads
// them, and contiguous runs stay contiguous within their block (about 2.5 wavefronts per warp
// access against 6 for the plain layout, in a model of the passes at W = 512 .. 4096).
__device__ __forceinline__ int fsw(int i) { return i ^ ((i >> 4) & 15); }

// Twiddles of a group.  A DIF pass starting at stage s0 needs, for stage t and butterfly j,
// tw[(g_low + (j mod 2^(NS-1-t)) 2^low) << (s0 + t)], and a DIT pass starting at bit b0
// tw[(g_low + (j mod 2^t) 2^b0) << (log2W - 1 - b0 - t)] (g_low: the group's index bits below
// the pass): 2^NS - 1 distinct values, listed stage by stage and padded to 2^NS.  FilterTables
// keeps every pass's lists as 2^(NS-1) planes of 16-byte pairs, plane k holding pair k of every
// group in group order, so a warp's k-th load covers consecutive 16-byte words; without that
// table (twp == nullptr) the list is gathered from tw.  (One scattered load per butterfly made
// the kernel L1-bound.)

// One pass of NS consecutive radix-2 DIF stages, the first being stage s0 (half = W >> (s0+1)).
// Those stages touch index bits hbit .. hbit-NS+1; a group is the 2^NS elements that differ only
// there.  Butterfly: (x, y) -> (x + y, (x - y) tw[(i & (half-1)) << stage]).  hb_tab (last pass
// only) multiplies the bit-reversed result by H[bitrev(p)] / W.  twp: this pass's group lists.
template <int NS>
__device__ __forceinline__ void dif_pass(float2 *buf0, const float2 *__restrict__ tw, const float2 *__restrict__ twp,
                                         const float *__restrict__ hb_tab, int W, int log2W, int s0, int count) {
    constexpr int GS = 1 << NS;
    const int hbit = log2W - 1 - s0;
    const int low = hbit - NS + 1;
    for (int gg = threadIdx.x; gg < (count << (log2W - NS)); gg += blockDim.x) {
        float2 *buf = buf0 + ((gg >> (log2W - NS)) << log2W);  // FFT gg / (W >> NS) of count
        const int g = gg & ((W >> NS) - 1);
        const int g_low = g & ((1 << low) - 1);
        const int base = ((g >> low) << (hbit + 1)) | g_low;
        float2 v[GS];
#pragma unroll
        for (int j = 0; j < GS; j++) v[j] = buf[fsw(base + (j << low))];
        float2 tq[GS];  // stage t's list starts at GS - (GS >> t)
        if (twp) {
            const float4 *q = reinterpret_cast<const float4 *>(twp) + g_low;
#pragma unroll
            for (int k = 0; k < GS / 2; k++) {
                const float4 f = __ldg(q + (k << low));  // plane k of 2^low groups
                tq[2 * k] = make_float2(f.x, f.y);
                tq[2 * k + 1] = make_float2(f.z, f.w);
            }
        } else {
#pragma unroll
            for (int t = 0; t < NS; t++)
#pragma unroll
                for (int jt = 0; jt < (GS >> (t + 1)); jt++)
                    tq[GS - (GS >> t) + jt] = __ldg(tw + ((g_low + (jt << low)) << (s0 + t)));
        }
#pragma unroll
        for (int t = 0; t < NS; t++) {
            const int hstep = GS >> (t + 1);
#pragma unroll
            for (int j = 0; j < GS; j++) {
                if (j & hstep) continue;
                const float2 w = tq[GS - (GS >> t) + (j & ((1 << (NS - 1 - t)) - 1))];
                const float2 x = v[j], y = v[j + hstep];
                v[j] = make_float2(x.x + y.x, x.y + y.y);
                v[j + hstep] = cmul(make_float2(x.x - y.x, x.y - y.y), w);
            }
        }
        if (hb_tab) {
#pragma unroll
            for (int j = 0; j < GS; j++) {
                const float h = __ldg(hb_tab + base + (j << low));
                v[j] = make_float2(v[j].x * h, v[j].y * h);
            }
        }
#pragma unroll
        for (int j = 0; j < GS; j++) buf[fsw(base + (j << low))] = v[j];
    }
}
template <int NS>
__device__ __forceinline__ void dit_pass(float2 *buf0, const float2 *__restrict__ tw, const float2 *__restrict__ twp,
                                         int W, int log2W, int b0, int count) {
    constexpr int GS = 1 << NS;
    for (int gg = threadIdx.x; gg < (count << (log2W - NS)); gg += blockDim.x) {
        float2 *buf = buf0 + ((gg >> (log2W - NS)) << log2W);
        const int g = gg & ((W >> NS) - 1);
        const int g_low = g & ((1 << b0) - 1);
        const int base = ((g >> b0) << (b0 + NS)) | g_low;
        float2 v[GS];
#pragma unroll
        for (int j = 0; j < GS; j++) v[j] = buf[fsw(base + (j << b0))];
        float2 tq[GS];  // stage t's list starts at 2^t - 1
        if (twp) {
            const float4 *q = reinterpret_cast<const float4 *>(twp) + g_low;
#pragma unroll
            for (int k = 0; k < GS / 2; k++) {
                const float4 f = __ldg(q + (k << b0));  // plane k of 2^b0 groups
                tq[2 * k] = make_float2(f.x, f.y);
                tq[2 * k + 1] = make_float2(f.z, f.w);
            }
        } else {
#pragma unroll
            for (int t = 0; t < NS; t++)
#pragma unroll
                for (int jt = 0; jt < (1 << t); jt++)
                    tq[(1 << t) - 1 + jt] = __ldg(tw + ((g_low + (jt << b0)) << (log2W - 1 - b0 - t)));
        }
#pragma unroll
        for (int t = 0; t < NS; t++) {
            const int hstep = 1 << t;
#pragma unroll
            for (int j = 0; j < GS; j++) {
                if (j & hstep) continue;
                const float2 w = tq[(1 << t) - 1 + (j & ((1 << t) - 1))];
                const float2 x = v[j];
                const float2 u = cmulc(v[j + hstep], w);
                v[j] = make_float2(x.x + u.x, x.y + u.y);
                v[j + hstep] = make_float2(x.x - u.x, x.y - u.y);
            }
        }
#pragma unroll
        for (int j = 0; j < GS; j++) buf[fsw(base + (j << b0))] = v[j];
    }
}

// Forward transform, multiply by H, inverse transform of `count` W-point FFTs stored one after
// the other in buf; ends after a barrier.
__device__ __forceinline__ void filter_fft(float2 *buf, const FilterArgs &a, int count = 1) {
    long long off = 0;  // this pass's group lists in a.twp: the DIF passes', then the DIT passes'
    for (int s = 0; s < a.log2W; s += 3) {
        const int ns = min(3, a.log2W - s);
        const float *h = (s + ns == a.log2W) ? a.hb : nullptr;
        const float2 *twp = a.twp ? a.twp + off : nullptr;
        if (ns == 3) dif_pass<3>(buf, a.tw, twp, h, a.W, a.log2W, s, count);
        else if (ns == 2) dif_pass<2>(buf, a.tw, twp, h, a.W, a.log2W, s, count);
        else dif_pass<1>(buf, a.tw, twp, h, a.W, a.log2W, s, count);
        off += (long long)(1 << ns) << (a.log2W - s - ns);
        __syncthreads();
    }
    for (int b = 0; b < a.log2W; b += 3) {
        const int ns = min(3, a.log2W - b);
        const float2 *twp = a.twp ? a.twp + off : nullptr;
        if (ns == 3) dit_pass<3>(buf, a.tw, twp, a.W, a.log2W, b, count);
        else if (ns == 2) dit_pass<2>(buf, a.tw, twp, a.W, a.log2W, b, count);
        else dit_pass<1>(buf, a.tw, twp, a.W, a.log2W, b, count);
        off += (long long)(1 << ns) << b;
        __syncthreads();
    }
}

// Mean of the first (or last) pad_n weighted samples of row r.
__device__ float edge_mean(const FilterArgs &a, const float *view, int r, bool left) {
    float s = 0.f;
    for (int k = 0; k < a.pad_n; k++) s += row_sample(a, view, r, left ? k : a.nu - 1 - k);
    return s / (float)a.pad_n;
}

// LAYOUT: FDK_LAYOUT_ROWS, FDK_LAYOUT_TRANSPOSED, FDK_LAYOUT_MIRROR; OUT: float or __half
template <int LAYOUT, typename OUT>
__global__ void __launch_bounds__(256) filter_rows_kernel(FilterArgs a) {
    extern __shared__ float2 buf[];
    __shared__ float pads[4];
    const int r1 = blockIdx.x;
    const int r2 = a.nv - 1 - r1;
    const int view = blockIdx.y;
    const float *vsrc = a.src + (long long)view * a.src_vstride;
    const int W = a.W;

    if (threadIdx.x < 4) {
        const int r = (threadIdx.x < 2) ? r1 : r2;
        pads[threadIdx.x] = edge_mean(a, vsrc, r, (threadIdx.x & 1) == 0);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < W; k += blockDim.x) {
        const int c = k - a.off;
        float x1, x2;
        if (c < 0) {
            x1 = pads[0]; x2 = pads[2];
        } else if (c >= a.nu) {
            x1 = pads[1]; x2 = pads[3];
        } else {
            x1 = row_sample(a, vsrc, r1, c);
            x2 = row_sample(a, vsrc, r2, c);
        }
        buf[fsw(k)] = make_float2(x1, x2);
    }
    __syncthreads();

    filter_fft(buf, a);

    OUT *dst = reinterpret_cast<OUT *>(a.dst);
    for (int u = threadIdx.x; u < a.nu; u += blockDim.x) {
        const float2 y = buf[fsw(a.off + u)];
        const OUT o1 = to_out<OUT>(a, y.x), o2 = to_out<OUT>(a, y.y);
        if (LAYOUT == FDK_LAYOUT_ROWS) {
            OUT *d = dst + (long long)view * a.dst_vstride;
            d[(long long)r1 * a.dst_pitch + u] = o1;
            if (r2 != r1) d[(long long)r2 * a.dst_pitch + u] = o2;
        } else if (LAYOUT == FDK_LAYOUT_TRANSPOSED) {
            OUT *d = dst + (long long)view * a.dst_vstride + (long long)u * a.dst_pitch;
            d[r1] = o1;
            if (r2 != r1) d[r2] = o2;
        } else {  // mirror pairs: element (u, v) = (row v, row nv-1-v)
            OUT *d = dst + (long long)view * a.dst_vstride + (long long)u * a.dst_pitch * 2;
            d[2 * r1] = o1;
            d[2 * r1 + 1] = o2;
            if (r2 != r1) {
                d[2 * r2] = o2;
                d[2 * r2 + 1] = o1;
            }
        }
    }
}

template <typename OUT>
struct PairOf;
template <>
struct PairOf<float> {
    using T = float2;
    static __device__ __forceinline__ T make(float a, float b) { return make_float2(a, b); }
};
template <>
struct PairOf<__half> {
    using T = __half2;
    static __device__ __forceinline__ T make(__half a, __half b) { return __halves2half2(a, b); }
};

// MIRROR layout, G row pairs (r, nv-1-r), r = G * blockIdx.x + g, per CTA; G * sizeof(pair) = 16.
// NP = min(G, 4096 / W) pairs are transformed at once, so every 3-stage pass keeps all 512
// threads busy (W / 8 groups per FFT).
template <typename OUT, int G>
__global__ void __launch_bounds__(512, 2) filter_mirror_kernel(FilterArgs a) {
    using P = typename PairOf<OUT>::T;
    static_assert(G * sizeof(P) == 16, "one 16-byte store per column and side");
    extern __shared__ __align__(16) unsigned char fsm[];
    const int NP = min(G, max(1, 4096 >> a.log2W));
    float2 *buf = reinterpret_cast<float2 *>(fsm);                    // NP x W
    P *stg = reinterpret_cast<P *>(fsm + sizeof(float2) * NP * a.W);  // [side][u][G]
    __shared__ float pads[4 * G];
    const int view = blockIdx.y, r0 = blockIdx.x * G;
    const float *vsrc = a.src + (long long)view * a.src_vstride;
    for (int g0 = 0; g0 < G; g0 += NP) {
        if (threadIdx.x < 4 * NP) {
            const int q = threadIdx.x >> 2, j = threadIdx.x & 3, r1 = r0 + g0 + q;
            pads[threadIdx.x] = edge_mean(a, vsrc, j < 2 ? r1 : a.nv - 1 - r1, (j & 1) == 0);
        }
        __syncthreads();  // also ends the previous pairs' reads of buf
        for (int k = threadIdx.x; k < (NP << a.log2W); k += blockDim.x) {
            const int q = k >> a.log2W, c = (k & (a.W - 1)) - a.off;
            const int r1 = r0 + g0 + q, r2 = a.nv - 1 - r1;
            float x1, x2;
            if (c < 0) {
                x1 = pads[4 * q];
                x2 = pads[4 * q + 2];
            } else if (c >= a.nu) {
                x1 = pads[4 * q + 1];
                x2 = pads[4 * q + 3];
            } else {
                x1 = row_sample(a, vsrc, r1, c);
                x2 = row_sample(a, vsrc, r2, c);
            }
            buf[(q << a.log2W) + fsw(k & (a.W - 1))] = make_float2(x1, x2);
        }
        __syncthreads();
        filter_fft(buf, a, NP);
        for (int k = threadIdx.x; k < NP * a.nu; k += blockDim.x) {
            const int q = k / a.nu, u = k - q * a.nu, g = g0 + q;
            const float2 y = buf[(q << a.log2W) + fsw(a.off + u)];
            const OUT o1 = to_out<OUT>(a, y.x), o2 = to_out<OUT>(a, y.y);
            stg[u * G + g] = PairOf<OUT>::make(o1, o2);                     // element (u, r1)
            stg[(a.nu + u) * G + (G - 1 - g)] = PairOf<OUT>::make(o2, o1);  // element (u, r2)
        }
    }
    __syncthreads();
    // side 0: elements v = r0 .. r0+G-1; side 1: v = nv-r0-G .. nv-1-r0 (the mirrors, ascending)
    P *dst = reinterpret_cast<P *>(a.dst) + (long long)view * (a.dst_vstride / 2);
    for (int i = threadIdx.x; i < 2 * a.nu; i += blockDim.x) {
        const int side = i >= a.nu, u = side ? i - a.nu : i;
        const int v0 = side ? a.nv - r0 - G : r0;
        *reinterpret_cast<uint4 *>(dst + (long long)u * a.dst_pitch + v0) = *reinterpret_cast<const uint4 *>(stg + i * G);
    }
}

int FilterTables::create(const double *H, int W_) {
    W = W_;
    log2W = 0;
    while ((1 << log2W) < W) log2W++;
    std::vector<float2> t(W / 2);
    for (int k = 0; k < W / 2; k++) {
        const double ang = -2.0 * 3.14159265358979323846 * k / W;
        t[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    std::vector<float> h(W);
    for (int p = 0; p < W; p++) {
        int r = 0;
        for (int b = 0; b < log2W; b++)
            if (p & (1 << b)) r |= 1 << (log2W - 1 - b);
        h[p] = (float)(H[r] / W);
    }
    // the group lists of every pass, in filter_fft's order (DIF passes, then DIT passes); each
    // group's list padded to 2^ns entries and stored as 2^(ns-1) planes of pairs (pair k of
    // group g at (k * groups + g) * 2)
    std::vector<float2> pt;
    auto put_pass = [&](int groups, int GS, const std::vector<float2> &lists) {  // lists: groups x GS
        for (int k = 0; k < GS / 2; k++)
            for (int g = 0; g < groups; g++) {
                pt.push_back(lists[(size_t)g * GS + 2 * k]);
                pt.push_back(lists[(size_t)g * GS + 2 * k + 1]);
            }
    };
    for (int s0 = 0; s0 < log2W; s0 += 3) {
        const int ns = std::min(3, log2W - s0), GS = 1 << ns, low = log2W - s0 - ns;
        std::vector<float2> lists((size_t)GS << low, make_float2(0.f, 0.f));
        for (int g = 0; g < (1 << low); g++) {
            int e = 0;
            for (int st = 0; st < ns; st++)
                for (int jt = 0; jt < (GS >> (st + 1)); jt++)
                    lists[(size_t)g * GS + e++] = t[(g + (jt << low)) << (s0 + st)];
        }
        put_pass(1 << low, GS, lists);
    }
    for (int b0 = 0; b0 < log2W; b0 += 3) {
        const int ns = std::min(3, log2W - b0), GS = 1 << ns;
        std::vector<float2> lists((size_t)GS << b0, make_float2(0.f, 0.f));
        for (int g = 0; g < (1 << b0); g++) {
            int e = 0;
            for (int st = 0; st < ns; st++)
                for (int jt = 0; jt < (1 << st); jt++)
                    lists[(size_t)g * GS + e++] = t[(g + (jt << b0)) << (log2W - 1 - b0 - st)];
        }
        put_pass(1 << b0, GS, lists);
    }
    FDK_CUDA(cudaMalloc(&tw, sizeof(float2) * (W / 2)));
    FDK_CUDA(cudaMalloc(&hb, sizeof(float) * W));
    FDK_CUDA(cudaMalloc(&twp, sizeof(float2) * pt.size()));
    SetupStream ss;
    FDK_TRY(ss.open());
    FDK_CUDA(cudaMemcpyAsync(tw, t.data(), sizeof(float2) * (W / 2), cudaMemcpyHostToDevice, ss.st));
    FDK_CUDA(cudaMemcpyAsync(hb, h.data(), sizeof(float) * W, cudaMemcpyHostToDevice, ss.st));
    FDK_CUDA(cudaMemcpyAsync(twp, pt.data(), sizeof(float2) * pt.size(), cudaMemcpyHostToDevice, ss.st));
    return ss.finish("filter tables");
}

void FilterTables::release() {
    if (tw) cudaFree(tw);
    if (twp) cudaFree(twp);
    if (hb) cudaFree(hb);
    tw = nullptr;
    twp = nullptr;
    hb = nullptr;
}

template <typename OUT, int G>
static int launch_mirror(const FilterArgs &a, int n_views, cudaStream_t st) {
    using P = typename PairOf<OUT>::T;
    const int np = std::min(G, std::max(1, 4096 >> a.log2W));
    const size_t smem = sizeof(float2) * np * a.W + 2 * sizeof(P) * G * a.nu;
    // per device and size, and needed at 48 KB too (the kernel also has static shared memory):
    // cheap, so set on every launch
    FDK_CUDA(cudaFuncSetAttribute(filter_mirror_kernel<OUT, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    filter_mirror_kernel<OUT, G><<<dim3(a.nv / (2 * G), n_views), 512, smem, st>>>(a);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
}

static int launch_filter(const FilterArgs &a, int n_views, int layout, int dtype, cudaStream_t st) {
    if (layout == FDK_LAYOUT_MIRROR) {
        // grouped kernel when G pairs tile the rows and every 16-byte store is aligned
        const int G = dtype == FDK_DTYPE_F32 ? 2 : 4;
        const size_t pair = dtype == FDK_DTYPE_F32 ? 8 : 4;
        const size_t smem = sizeof(float2) * std::max(a.W, std::min(G, 4096 / a.W) * a.W) + 2 * pair * G * a.nu;
        if (a.nv % (2 * G) == 0 && ((uintptr_t)a.dst & 15) == 0 && (a.dst_pitch * pair) % 16 == 0 &&
            (a.dst_vstride * (pair / 2)) % 16 == 0 && smem <= 200 * 1024) {
            if (dtype == FDK_DTYPE_F32) return launch_mirror<float, 2>(a, n_views, st);
            return launch_mirror<__half, 4>(a, n_views, st);
        }
    }
    const dim3 grid((a.nv + 1) / 2, n_views);
    const size_t smem = sizeof(float2) * a.W;
    if (smem + sizeof(float) * 4 > 48 * 1024) {  // dynamic + static (pads) above the default limit
        // opt in to more than 48 KB of dynamic shared memory (per device: set on every launch)
        FDK_CUDA(cudaFuncSetAttribute(filter_rows_kernel<FDK_LAYOUT_ROWS, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
        FDK_CUDA(cudaFuncSetAttribute(filter_rows_kernel<FDK_LAYOUT_TRANSPOSED, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
        FDK_CUDA(cudaFuncSetAttribute(filter_rows_kernel<FDK_LAYOUT_MIRROR, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
        FDK_CUDA(cudaFuncSetAttribute(filter_rows_kernel<FDK_LAYOUT_ROWS, __half>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
        FDK_CUDA(cudaFuncSetAttribute(filter_rows_kernel<FDK_LAYOUT_TRANSPOSED, __half>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
        FDK_CUDA(cudaFuncSetAttribute(filter_rows_kernel<FDK_LAYOUT_MIRROR, __half>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    }
#define FDK_LAUNCH(L, T) filter_rows_kernel<L, T><<<grid, 256, smem, st>>>(a)
    if (dtype == FDK_DTYPE_F32) {
        if (layout == FDK_LAYOUT_ROWS) FDK_LAUNCH(FDK_LAYOUT_ROWS, float);
        else if (layout == FDK_LAYOUT_TRANSPOSED) FDK_LAUNCH(FDK_LAYOUT_TRANSPOSED, float);
        else FDK_LAUNCH(FDK_LAYOUT_MIRROR, float);
    } else {
        if (layout == FDK_LAYOUT_ROWS) FDK_LAUNCH(FDK_LAYOUT_ROWS, __half);
        else if (layout == FDK_LAYOUT_TRANSPOSED) FDK_LAUNCH(FDK_LAYOUT_TRANSPOSED, __half);
        else FDK_LAUNCH(FDK_LAYOUT_MIRROR, __half);
    }
#undef FDK_LAUNCH
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
}

// Shared by the FilterEngine handle, the cuFFT-plugin entry points and the reconstructor.
int filter_views(const float *src, int src_pitch, long long src_vstride, void *dst, int dst_pitch,
                 long long dst_vstride, const float *cos, int cos_pitch, const FilterTables &t, int nu,
                 int nv, int pad_n, int n_views, int layout, int dtype, cudaStream_t st, float out_scale,
                 unsigned int *overflow) {
    FilterArgs a;
    a.src = src;
    a.dst = dst;
    a.cos = cos;
    a.tw = t.tw;
    a.twp = t.twp;
    a.hb = t.hb;
    a.nu = nu;
    a.nv = nv;
    a.W = t.W;
    a.log2W = t.log2W;
    a.off = (t.W - nu) >> 1;
    a.pad_n = pad_n;
    a.src_pitch = src_pitch;
    a.dst_pitch = dst_pitch;
    a.cos_pitch = cos_pitch;
    a.src_vstride = src_vstride;
    a.dst_vstride = dst_vstride;
    a.out_scale = out_scale;
    a.overflow = overflow;
    return launch_filter(a, n_views, layout, dtype, st);
}

static int check_filter_dims(int64_t nu, int64_t nv, int64_t W, int pad) {
    FDK_CHECK_ARG(nu > 0 && nv > 0, "nu, nv must be positive");
    FDK_CHECK_ARG(W >= nu && W <= 4096 && (W & (W - 1)) == 0, "W=%lld must be a power of two in [nu, 4096]",
                  (long long)W);
    FDK_CHECK_ARG(pad >= 1 && pad <= 4 && pad <= nu, "pad_edge must be 1..4 and <= nu");
    FDK_CHECK_ARG(nv <= 65535 * 2, "nv too large");
    return FDK_OK;
}

// Kernel dst = src * table (kernelCorrect, cudaFftFilter.cu:270-281).
__global__ void correct_kernel(const float *src, float *dst, int pitch, int width, int height, int depth,
                               const float *table, int tpitch) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= width || y >= height || z >= depth) return;
    const long long o = ((long long)z * height + y) * pitch + x;
    dst[o] = src[o] * table[(long long)y * tpitch + x];
}

}  // namespace fdk

struct fdk_filter {
    int device = 0;
    int64_t nu = 0, nv = 0, W = 0;
    int pad = 4;
    float *d_cos = nullptr;
    float *d_src = nullptr;
    float *d_dst = nullptr;
    fdk::FilterTables tables;
    cudaStream_t stream = nullptr;
};

using namespace fdk;

extern "C" {

int fdk_filter_create(fdk_filter **out, const float *cos_table, const float *H, int64_t nu, int64_t nv,
                      int64_t W, int32_t pad_edge, int32_t device) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(out != nullptr && H != nullptr, "out or H is NULL");
    *out = nullptr;
    FDK_TRY(check_filter_dims(nu, nv, W, pad_edge));
    DeviceGuard dg(device);
    FDK_TRY(dg.status);
    fdk_filter *h = new fdk_filter();
    h->device = device;
    h->nu = nu;
    h->nv = nv;
    h->W = W;
    h->pad = pad_edge;
    std::vector<double> Hd(H, H + W);
    int s = h->tables.create(Hd.data(), (int)W);
    if (s == FDK_OK && cos_table) {
        SetupStream ss;
        s = ss.open();
        cudaError_t e = cudaSuccess;
        if (s == FDK_OK) e = cudaMalloc(&h->d_cos, sizeof(float) * nu * nv);
        if (s == FDK_OK && e == cudaSuccess)
            e = cudaMemcpyAsync(h->d_cos, cos_table, sizeof(float) * nu * nv, cudaMemcpyHostToDevice, ss.st);
        if (e != cudaSuccess) s = cuda_status(e, "filter cos table", __FILE__, __LINE__);
        if (s == FDK_OK) s = ss.finish("filter cos table");
    }
    if (s == FDK_OK) {
        cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) s = cuda_status(e, "cudaStreamCreate", __FILE__, __LINE__);
    }
    if (s != FDK_OK) {
        fdk_filter_destroy(h);
        return s;
    }
    *out = h;
    return FDK_OK;
    FDK_ABI_END
}

int fdk_filter_filtering(fdk_filter *h, float *src_host, float *dst_host, int32_t transpose) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && src_host && dst_host, "NULL argument");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    const size_t n = (size_t)h->nu * h->nv;
    // FilterCosCorrect (FilterLib.h:8-13): src *= cos, in place on the caller's buffer, in FP32.
    if (h->d_cos) {
        std::vector<float> cos(n);
        FDK_CUDA(cudaMemcpy(cos.data(), h->d_cos, sizeof(float) * n, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; i++) src_host[i] = src_host[i] * cos[i];
    }
    if (!h->d_src) {
        FDK_CUDA(cudaMalloc(&h->d_src, sizeof(float) * n));
        FDK_CUDA(cudaMalloc(&h->d_dst, sizeof(float) * n));
    }
    FDK_CUDA(cudaMemcpyAsync(h->d_src, src_host, sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
    const int layout = transpose ? FDK_LAYOUT_TRANSPOSED : FDK_LAYOUT_ROWS;
    const int dpitch = transpose ? (int)h->nv : (int)h->nu;
    FDK_TRY(filter_views(h->d_src, (int)h->nu, (long long)n, h->d_dst, dpitch, (long long)n, nullptr, 0,
                         h->tables, (int)h->nu, (int)h->nv, h->pad, 1, layout, FDK_DTYPE_F32, h->stream));
    FDK_CUDA(cudaMemcpyAsync(dst_host, h->d_dst, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
    FDK_CUDA(cudaStreamSynchronize(h->stream));
    return FDK_OK;
    FDK_ABI_END
}

int fdk_filter_run_device(fdk_filter *h, const float *src_dev, void *dst_dev, int64_t n_views, int32_t layout,
                          int32_t out_dtype, float out_scale, void *stream) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && src_dev && dst_dev, "NULL argument");
    FDK_CHECK_ARG(n_views > 0 && n_views <= 65535, "n_views out of range");
    FDK_CHECK_ARG(layout >= FDK_LAYOUT_ROWS && layout <= FDK_LAYOUT_MIRROR, "bad layout");
    FDK_CHECK_ARG(out_dtype == FDK_DTYPE_F32 || out_dtype == FDK_DTYPE_F16, "bad dtype");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    const long long n = (long long)h->nu * h->nv;
    const int dpitch = layout == FDK_LAYOUT_ROWS ? (int)h->nu : (int)h->nv;
    const long long dstride = layout == FDK_LAYOUT_MIRROR ? 2 * n : n;
    return filter_views(src_dev, (int)h->nu, n, dst_dev, dpitch, dstride, h->d_cos, (int)h->nu, h->tables,
                        (int)h->nu, (int)h->nv, h->pad, (int)n_views, layout, out_dtype,
                        (cudaStream_t)stream, out_scale, nullptr);
    FDK_ABI_END
}

int fdk_filter_destroy(fdk_filter *h) {
    if (!h) return FDK_OK;
    {
        DeviceGuard dg(h->device);
        if (h->stream) cudaStreamSynchronize(h->stream);
        h->tables.release();
        if (h->d_cos) cudaFree(h->d_cos);
        if (h->d_src) cudaFree(h->d_src);
        if (h->d_dst) cudaFree(h->d_dst);
        if (h->stream) cudaStreamDestroy(h->stream);
    }
    delete h;
    return FDK_OK;
}

int fdk_correct_image_real32(const fdk_dataref *src, const fdk_dataref *table, fdk_dataref *dst) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(src && table && dst && src->data && table->data && dst->data, "NULL argument");
    FDK_CHECK_ARG(src->pitch == dst->pitch && src->width == dst->width && src->height == dst->height &&
                      src->depth <= dst->depth,
                  "src/dst shapes differ (CorrectImage, cudaFftFilter.cu:286-289)");
    FDK_CHECK_ARG(src->width > 0 && src->height > 0 && src->depth > 0 && src->pitch >= src->width, "bad shape");
    FDK_CHECK_ARG(src->height <= 65535 && src->depth <= 65535, "shape too large");
    const dim3 grid((unsigned)ceil_div(src->width, 128), src->height, src->depth);
    correct_kernel<<<grid, 128, 0, cudaStreamLegacy>>>(src->data, dst->data, src->pitch, src->width, src->height,
                                                       src->depth, table->data, table->pitch);
    FDK_CUDA(cudaGetLastError());
    FDK_CUDA(cudaStreamSynchronize(cudaStreamLegacy));  // synchronous, as the reference
    return FDK_OK;
    FDK_ABI_END
}

int fdk_filter_row_real32(const fdk_dataref *src, fdk_dataref *dst, const fdk_dataref *filter) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(src && dst && filter && src->data && dst->data && filter->data, "NULL argument");
    FDK_CHECK_ARG(src->width == dst->width && src->height == dst->height && src->depth <= dst->depth,
                  "src/dst shapes differ (FilterRow, cudaFftFilter.cu:302-305)");
    FDK_CHECK_ARG(filter->height == 1 || filter->height == 0, "filter must be one row");
    const int W = filter->width;
    FDK_TRY(check_filter_dims(src->width, src->height, W, 3));
    std::vector<float> Hf(W);
    FDK_CUDA(cudaMemcpy(Hf.data(), filter->data, sizeof(float) * W, cudaMemcpyDeviceToHost));
    std::vector<double> Hd(Hf.begin(), Hf.end());
    FilterTables t;
    int s = t.create(Hd.data(), W);
    if (s == FDK_OK)
        s = filter_views(src->data, src->pitch, (long long)src->pitch * src->height, dst->data, dst->pitch,
                         (long long)dst->pitch * dst->height, nullptr, 0, t, src->width, src->height, 3,
                         src->depth, FDK_LAYOUT_ROWS, FDK_DTYPE_F32, cudaStreamLegacy);
    if (s == FDK_OK) {
        cudaError_t e = cudaStreamSynchronize(cudaStreamLegacy);  // synchronous, as the reference
        if (e != cudaSuccess) s = cuda_status(e, "FilterRow sync", __FILE__, __LINE__);
    }
    t.release();
    return s;
    FDK_ABI_END
}

}  // extern "C"
