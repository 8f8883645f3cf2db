// learn.cu -- the learned residual row filter and what training it needs (no reference
// counterpart): a small 1D residual network (3 conv layers, 32 channels, kernel 9) refines each
// ramp-filtered row; it is trained on phantoms that this library's own ray-marching forward
// projector generates, with the loss backpropagated through the exact adjoint of BP.
//
// Network, per detector row x (length L = nu), s = the row scale (1 / (SOD^2 AAF): line-integral
// units):
//   a1 = relu(W1 * (s x) + b1)      1 -> 32 channels, kernel 9, zero 'same' padding
//   a2 = relu(W2 * a1 + b2)         32 -> 32
//   o  = W3 * a2 + b3               32 -> 1
//   y  = x + o / s                  residual: zero W3, b3 give plain FDK
// Parameters FP32 (layout W1[32][9], b1[32], W2[32][32][9], b2[32], W3[32][9], b3); activations
// are kept in shared memory as BF16 (forward) and recomputed in the backward pass, so no
// activation tensor touches HBM.
//
// Training kernels: exact adjoint of the staged backprojection (scatter with the gather's
// bilinear weights and bounds, accumulated per view in a shared-memory box), the volume MSE
// and its gradient, Adam, Poisson transmission noise, an ellipsoid voxelizer, and the
// ROWS -> MIRROR layout change that feeds the backprojection.
#include <cuda_bf16.h>

#include <mutex>
#include <vector>

#include "common.h"
#include "internal.h"

namespace fdk {

constexpr int kCh = 32, kK = 9, kHalo = 4;
constexpr int kW1 = 0, kB1 = kW1 + kCh * kK, kW2 = kB1 + kCh, kB2 = kW2 + kCh * kCh * kK, kW3 = kB2 + kCh,
              kB3 = kW3 + kCh * kK, kNParam = kB3 + 1;
constexpr int kMaxLen = 256;  // row length limit (the backward kernel holds ~176 KB of shared memory)

// --------------------------------------------------------------------------------------------
// Network kernels.  One CTA of 256 threads works on one row at a time (persistent over rows).
// The convolutions are register-blocked: in the channel phases thread t owns 4 consecutive
// positions (pg = t % 64) x 8 channels (q = t / 64, uniform within a warp), so each float4
// weight load (a warp-wide broadcast) feeds 16 FMAs and one 12-value activation window feeds
// all 9 taps.  Activation rows carry a zero halo: buffer index = position + 4, and every entry
// past the row's end stays zero, so no tap needs a bounds test.
// --------------------------------------------------------------------------------------------
constexpr int kThreads = 256;
constexpr int kBuf = kMaxLen + 2 * kHalo + 8;  // 272 f32 per scalar row buffer (x, d3)
constexpr int kPitchA = 268;                    // bf16 per activation row (8-byte aligned rows)
constexpr int kPitchD = 268;                    // f32 per dz2 row (16-byte aligned rows)
constexpr int kPitchZ = 260;                    // f32 per dz1 row (16-byte aligned rows)

struct NnWeights {
    float w2f[kCh * kK * kCh];  // W2 as [ci][k][c]: the 8 output channels of one (ci, k) are contiguous
    float w1[kCh * kK], b1[kCh], b2[kCh], w3[kCh * kK], b3[4];
};

struct NnFwdShared {
    NnWeights w;
    float x[kBuf];                        // s * x with halo
    float part[4][kMaxLen];               // layer-3 partial sums of the 4 channel groups
    __nv_bfloat16 a1[kCh][kPitchA];       // relu(layer 1), BF16
    __nv_bfloat16 a2[kCh][kPitchA];       // relu(layer 2), BF16
};

__device__ __forceinline__ float bf_lo(unsigned u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf_hi(unsigned u) { return __uint_as_float(u & 0xFFFF0000u); }

// 12 consecutive f32 from a 16-byte aligned address
__device__ __forceinline__ void ld_f12(const float *p, float (&v)[12]) {
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const float4 t = reinterpret_cast<const float4 *>(p)[i];
        v[4 * i] = t.x;
        v[4 * i + 1] = t.y;
        v[4 * i + 2] = t.z;
        v[4 * i + 3] = t.w;
    }
}

// 4n consecutive BF16 (as f32) from an 8-byte aligned address
template <int N>
__device__ __forceinline__ void ld_bf(const __nv_bfloat16 *p, float (&v)[N]) {
    static_assert(N % 4 == 0, "groups of 4");
#pragma unroll
    for (int i = 0; i < N / 4; i++) {
        const uint2 u = reinterpret_cast<const uint2 *>(p)[i];
        v[4 * i] = bf_lo(u.x);
        v[4 * i + 1] = bf_hi(u.x);
        v[4 * i + 2] = bf_lo(u.y);
        v[4 * i + 3] = bf_hi(u.y);
    }
}

// 4 values -> BF16 (round to nearest even) at an 8-byte aligned address
__device__ __forceinline__ void st_bf4(__nv_bfloat16 *p, const float (&v)[4]) {
    const __nv_bfloat162 lo = __floats2bfloat162_rn(v[0], v[1]), hi = __floats2bfloat162_rn(v[2], v[3]);
    uint2 u;
    u.x = *reinterpret_cast<const unsigned *>(&lo);
    u.y = *reinterpret_cast<const unsigned *>(&hi);
    *reinterpret_cast<uint2 *>(p) = u;
}

__device__ void nn_load_weights(NnWeights &w, float *w2b, const float *params) {
    for (int i = threadIdx.x; i < kCh * kCh * kK; i += kThreads) {
        const int c = i / (kCh * kK), ci = (i / kK) % kCh, k = i % kK;  // params W2[c][ci][k]
        const float v = params[kW2 + i];
        w.w2f[(ci * kK + k) * kCh + c] = v;
        if (w2b) w2b[(c * kK + k) * kCh + ci] = v;
    }
    for (int i = threadIdx.x; i < kCh * kK; i += kThreads) {
        w.w1[i] = params[kW1 + i];
        w.w3[i] = params[kW3 + i];
    }
    for (int i = threadIdx.x; i < kCh; i += kThreads) {
        w.b1[i] = params[kB1 + i];
        w.b2[i] = params[kB2 + i];
    }
    if (threadIdx.x == 0) w.b3[0] = params[kB3];
}

// a1[c][p] = relu(b1[c] + sum_k W1[c][k] xs[p + k - 4]) for this thread's 4 positions x 8 channels
__device__ __forceinline__ void nn_layer1(const NnWeights &w, const float *xb, __nv_bfloat16 (*a1)[kPitchA], int pg,
                                          int q, int L) {
    const int p0 = 4 * pg;
    float xw[12];
    ld_f12(xb + p0, xw);  // positions p0 - 4 .. p0 + 7
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int c = 8 * q + i;
        float z[4];
#pragma unroll
        for (int j = 0; j < 4; j++) z[j] = w.b1[c];
#pragma unroll
        for (int k = 0; k < kK; k++) {
            const float wk = w.w1[c * kK + k];
#pragma unroll
            for (int j = 0; j < 4; j++) z[j] = fmaf(wk, xw[j + k], z[j]);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) z[j] = (p0 + j < L) ? fmaxf(z[j], 0.f) : 0.f;
        st_bf4(&a1[c][p0 + kHalo], z);
    }
}

// a2[c][p] = relu(b2[c] + sum_ci sum_k W2[c][ci][k] a1[ci][p + k - 4])
__device__ __forceinline__ void nn_layer2(const NnWeights &w, const __nv_bfloat16 (*a1)[kPitchA],
                                          __nv_bfloat16 (*a2)[kPitchA], int pg, int q, int L) {
    const int p0 = 4 * pg;
    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = w.b2[8 * q + i];
#pragma unroll 2
    for (int ci = 0; ci < kCh; ci++) {
        float a[12];
        ld_bf<12>(&a1[ci][p0], a);
#pragma unroll
        for (int k = 0; k < kK; k++) {
            const float4 wa = *reinterpret_cast<const float4 *>(&w.w2f[(ci * kK + k) * kCh + 8 * q]);
            const float4 wb = *reinterpret_cast<const float4 *>(&w.w2f[(ci * kK + k) * kCh + 8 * q + 4]);
            const float wv[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(wv[i], a[j + k], acc[i][j]);
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        float r[4];
#pragma unroll
        for (int j = 0; j < 4; j++) r[j] = (p0 + j < L) ? fmaxf(acc[i][j], 0.f) : 0.f;
        st_bf4(&a2[8 * q + i][p0 + kHalo], r);
    }
}

__global__ void __launch_bounds__(kThreads, 2) nn_forward_kernel(const float *__restrict__ params, const float *x,
                                                                float *y, int L, long long rows, float s) {
    extern __shared__ __align__(16) unsigned char smraw[];
    NnFwdShared &sm = *reinterpret_cast<NnFwdShared *>(smraw);
    const int t = threadIdx.x, pg = t % 64, q = t / 64;
    nn_load_weights(sm.w, nullptr, params);
    for (int i = t; i < kCh * kPitchA; i += kThreads) {
        (&sm.a1[0][0])[i] = __float2bfloat16(0.f);
        (&sm.a2[0][0])[i] = __float2bfloat16(0.f);
    }
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        __syncthreads();
        for (int i = t; i < kBuf; i += kThreads) {
            const int p = i - kHalo;
            sm.x[i] = (p >= 0 && p < L) ? x[r * L + p] * s : 0.f;
        }
        __syncthreads();
        nn_layer1(sm.w, sm.x, sm.a1, pg, q, L);
        __syncthreads();
        nn_layer2(sm.w, sm.a1, sm.a2, pg, q, L);
        __syncthreads();
        {  // layer 3, partial over this thread's 8 channels
            float o[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int c = 8 * q + i;
                float a[12];
                ld_bf<12>(&sm.a2[c][4 * pg], a);
#pragma unroll
                for (int k = 0; k < kK; k++) {
                    const float wk = sm.w.w3[c * kK + k];
#pragma unroll
                    for (int j = 0; j < 4; j++) o[j] = fmaf(wk, a[j + k], o[j]);
                }
            }
            *reinterpret_cast<float4 *>(&sm.part[q][4 * pg]) = make_float4(o[0], o[1], o[2], o[3]);
        }
        __syncthreads();
        if (t < L) {
            const float o = sm.w.b3[0] + ((sm.part[0][t] + sm.part[1][t]) + (sm.part[2][t] + sm.part[3][t]));
            y[r * L + t] = x[r * L + t] + o / s;
        }
    }
}

// --------------------------------------------------------------------------------------------
// backward: persistent CTAs (one per SM); each row's activations are recomputed in shared
// memory, and the parameter gradients stay in registers for the CTA's whole life:
//   dW2[c][ci][k]  thread (warp w: c = 4w..4w+3, lane: ci), 36 accumulators
//   dW3[c][k], dW1[ci][k]  lane = channel, warp = a 32-position range, 9 accumulators each
//   db1, db2 (8 per thread, its channel group), db3
// and are added to global memory once at the end.
// --------------------------------------------------------------------------------------------
struct NnBackShared {
    NnWeights w;
    float w2b[kCh * kK * kCh];        // W2 as [c][k][ci]: the 8 input channels of one (c, k) are contiguous
    float x[kBuf];                    // s * x with halo
    float d3[kBuf];                   // dL/do = dL/dy / s with halo
    float dz2[kCh][kPitchD];          // dL/dz2 with halo
    float dz1[kCh][kPitchZ];          // dL/dz1, positions 0 .. 255
    __nv_bfloat16 a1[kCh][kPitchA];
    __nv_bfloat16 a2[kCh][kPitchA];
};

__global__ void __launch_bounds__(kThreads, 1) nn_backward_kernel(const float *__restrict__ params, const float *x,
                                                                 const float *dy, float *dparams, int L,
                                                                 long long rows, float s) {
    extern __shared__ __align__(16) unsigned char smraw[];
    NnBackShared &sm = *reinterpret_cast<NnBackShared *>(smraw);
    const int t = threadIdx.x, pg = t % 64, q = t / 64, p0 = 4 * pg, lane = t & 31, wp = t >> 5;
    nn_load_weights(sm.w, sm.w2b, params);
    for (int i = t; i < kCh * kPitchA; i += kThreads) {
        (&sm.a1[0][0])[i] = __float2bfloat16(0.f);
        (&sm.a2[0][0])[i] = __float2bfloat16(0.f);
    }
    for (int i = t; i < kCh * kPitchD; i += kThreads) (&sm.dz2[0][0])[i] = 0.f;

    float gw2[4][kK], gw3[kK], gw1[kK], gb1[8], gb2[8], gb3 = 0.f;
#pragma unroll
    for (int k = 0; k < kK; k++) {
        gw3[k] = gw1[k] = 0.f;
#pragma unroll
        for (int i = 0; i < 4; i++) gw2[i][k] = 0.f;
    }
#pragma unroll
    for (int i = 0; i < 8; i++) gb1[i] = gb2[i] = 0.f;

    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        __syncthreads();
        for (int i = t; i < kBuf; i += kThreads) {
            const int p = i - kHalo;
            const bool in = p >= 0 && p < L;
            sm.x[i] = in ? x[r * L + p] * s : 0.f;
            const float d = in ? dy[r * L + p] / s : 0.f;  // y = x + o / s
            sm.d3[i] = d;
            gb3 += d;
        }
        __syncthreads();
        nn_layer1(sm.w, sm.x, sm.a1, pg, q, L);
        __syncthreads();
        nn_layer2(sm.w, sm.a1, sm.a2, pg, q, L);
        __syncthreads();
        {  // dz2[c][p] = [a2 > 0] sum_k W3[c][k] d3[p - k + 4]
            float dw[12];
            ld_f12(sm.d3 + p0, dw);  // positions p0 - 4 .. p0 + 7
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int c = 8 * q + i;
                float m[4];
                ld_bf<4>(&sm.a2[c][p0 + kHalo], m);
                float g[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int k = 0; k < kK; k++) {
                    const float wk = sm.w.w3[c * kK + k];
#pragma unroll
                    for (int j = 0; j < 4; j++) g[j] = fmaf(wk, dw[j - k + 8], g[j]);
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    g[j] = m[j] > 0.f ? g[j] : 0.f;
                    gb2[i] += g[j];
                }
                *reinterpret_cast<float4 *>(&sm.dz2[c][p0 + kHalo]) = make_float4(g[0], g[1], g[2], g[3]);
            }
        }
        // dW3[c][k] += sum_p d3[p] a2[c][p + k - 4]   (lane = c, warp = positions 32 wp ..)
#pragma unroll 1
        for (int m = 0; m < 4; m++) {
            const int pb = 32 * wp + 8 * m;
            if (pb >= L) break;
            float a[16];
            ld_bf<16>(&sm.a2[lane][pb], a);
            const float4 d0 = *reinterpret_cast<const float4 *>(&sm.d3[pb + kHalo]);
            const float4 d1 = *reinterpret_cast<const float4 *>(&sm.d3[pb + kHalo + 4]);
            const float d[8] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w};
#pragma unroll
            for (int j = 0; j < 8; j++)
#pragma unroll
                for (int k = 0; k < kK; k++) gw3[k] = fmaf(d[j], a[j + k], gw3[k]);
        }
        __syncthreads();
        {  // dz1[ci][p] = [a1 > 0] sum_c sum_k W2[c][ci][k] dz2[c][p - k + 4]
            float acc[8][4];
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
#pragma unroll 2
            for (int c = 0; c < kCh; c++) {
                float dw[12];
                ld_f12(&sm.dz2[c][p0], dw);
#pragma unroll
                for (int k = 0; k < kK; k++) {
                    const float4 wa = *reinterpret_cast<const float4 *>(&sm.w2b[(c * kK + k) * kCh + 8 * q]);
                    const float4 wb = *reinterpret_cast<const float4 *>(&sm.w2b[(c * kK + k) * kCh + 8 * q + 4]);
                    const float wv[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
                    for (int i = 0; i < 8; i++)
#pragma unroll
                        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(wv[i], dw[j - k + 8], acc[i][j]);
                }
            }
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int ci = 8 * q + i;
                float m[4];
                ld_bf<4>(&sm.a1[ci][p0 + kHalo], m);
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    acc[i][j] = m[j] > 0.f ? acc[i][j] : 0.f;
                    gb1[i] += acc[i][j];
                }
                *reinterpret_cast<float4 *>(&sm.dz1[ci][p0]) = make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
            }
        }
        // dW2[c][ci][k] += sum_p dz2[c][p] a1[ci][p + k - 4]   (c = 4 wp + i, lane = ci)
#pragma unroll 1
        for (int pb = 0; pb < L; pb += 8) {
            float a[16];
            ld_bf<16>(&sm.a1[lane][pb], a);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float4 d0 = *reinterpret_cast<const float4 *>(&sm.dz2[4 * wp + i][pb + kHalo]);
                const float4 d1 = *reinterpret_cast<const float4 *>(&sm.dz2[4 * wp + i][pb + kHalo + 4]);
                const float d[8] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w};
#pragma unroll
                for (int j = 0; j < 8; j++)
#pragma unroll
                    for (int k = 0; k < kK; k++) gw2[i][k] = fmaf(d[j], a[j + k], gw2[i][k]);
            }
        }
        __syncthreads();
        // dW1[ci][k] += sum_p dz1[ci][p] xs[p + k - 4]   (lane = ci, warp = positions 32 wp ..)
#pragma unroll 1
        for (int m = 0; m < 4; m++) {
            const int pb = 32 * wp + 8 * m;
            if (pb >= L) break;
            float xw[16];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float4 v = *reinterpret_cast<const float4 *>(&sm.x[pb + 4 * i]);
                xw[4 * i] = v.x;
                xw[4 * i + 1] = v.y;
                xw[4 * i + 2] = v.z;
                xw[4 * i + 3] = v.w;
            }
            const float4 g0 = *reinterpret_cast<const float4 *>(&sm.dz1[lane][pb]);
            const float4 g1 = *reinterpret_cast<const float4 *>(&sm.dz1[lane][pb + 4]);
            const float g[8] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
#pragma unroll
            for (int j = 0; j < 8; j++)
#pragma unroll
                for (int k = 0; k < kK; k++) gw1[k] = fmaf(g[j], xw[j + k], gw1[k]);
        }
    }

    // one global add per accumulator (db sums reduced over the warp's lanes first)
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int k = 0; k < kK; k++) atomicAdd(dparams + kW2 + ((4 * wp + i) * kCh + lane) * kK + k, gw2[i][k]);
#pragma unroll
    for (int k = 0; k < kK; k++) {
        atomicAdd(dparams + kW3 + lane * kK + k, gw3[k]);
        atomicAdd(dparams + kW1 + lane * kK + k, gw1[k]);
    }
#pragma unroll
    for (int i = 0; i < 8; i++)
        for (int o = 16; o; o >>= 1) {
            gb1[i] += __shfl_xor_sync(0xFFFFFFFFu, gb1[i], o);
            gb2[i] += __shfl_xor_sync(0xFFFFFFFFu, gb2[i], o);
        }
    for (int o = 16; o; o >>= 1) gb3 += __shfl_xor_sync(0xFFFFFFFFu, gb3, o);
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            atomicAdd(dparams + kB1 + 8 * q + i, gb1[i]);
            atomicAdd(dparams + kB2 + 8 * q + i, gb2[i]);
        }
        atomicAdd(dparams + kB3, gb3);
    }
}

// --------------------------------------------------------------------------------------------
// Adam (Kingma & Ba), bias-corrected
// --------------------------------------------------------------------------------------------
__global__ void adam_kernel(float *w, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// --------------------------------------------------------------------------------------------
// transmission noise: p -> -log(max(Poisson(I0 exp(-mu p)), 1) / I0) / mu
// --------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    // splitmix64 finaliser
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double uniform01(unsigned long long &state) {
    state = mix64(state);
    return ((state >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
// Poisson sample: inversion by sequential search for lambda < 64, otherwise the normal
// approximation with continuity correction (relative error of the variance < 1% there).
__device__ double poisson(double lam, unsigned long long &st) {
    if (lam <= 0.0) return 0.0;
    if (lam < 64.0) {
        const double L = exp(-lam);
        double p = 1.0;
        int k = 0;
        do {
            k++;
            p *= uniform01(st);
        } while (p > L && k < 1000);
        return (double)(k - 1);
    }
    const double u1 = uniform01(st), u2 = uniform01(st);
    const double n = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    return fmax(0.0, floor(lam + sqrt(lam) * n + 0.5));
}

__global__ void noise_kernel(float *p, long long n, double i0, double mu, unsigned long long seed) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long st = mix64(seed ^ mix64((unsigned long long)i));
        const double lam = i0 * exp(-mu * (double)p[i]);
        const double cnt = fmax(poisson(lam, st), 1.0);
        p[i] = (float)(-log(cnt / i0) / mu);
    }
}

// --------------------------------------------------------------------------------------------
// ellipsoid voxelizer (value at voxel centres), [z][y][x]
// --------------------------------------------------------------------------------------------
struct EllipsoidSet {  // passed by value: no device allocation or copy per call
    double e[64 * 16];
};

__global__ void voxelize_kernel(const __grid_constant__ EllipsoidSet ell, int n_ell, int nx, int ny, int nz, double dx,
                                double dy, double dz, float *out) {
    __shared__ double se[64 * 16];
    for (int i = threadIdx.x; i < n_ell * 16; i += blockDim.x) se[i] = ell.e[i];
    __syncthreads();
    const long long total = (long long)nx * ny * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const int y = (int)((i / nx) % ny);
        const int z = (int)(i / ((long long)nx * ny));
        const double P[3] = {(x - (nx - 1) / 2.0) * dx, -(y - (ny - 1) / 2.0) * dy, -(z - (nz - 1) / 2.0) * dz};
        double v = 0;
        for (int k = 0; k < n_ell; k++) {
            const double *e = se + 16 * k;
            double q = 0;
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const double l = e[6 + r] * (P[0] - e[0]) + e[9 + r] * (P[1] - e[1]) + e[12 + r] * (P[2] - e[2]);
                q += l * l / (e[3 + r] * e[3 + r]);
            }
            if (q <= 1.0) v += e[15];
        }
        out[i] = (float)v;
    }
}

// --------------------------------------------------------------------------------------------
// ROWS (views x nv rows x nu) -> MIRROR pairs (views x nu x nv, element (u, v) = (P[v][u], P[nv-1-v][u]))
// --------------------------------------------------------------------------------------------
__global__ void rows_to_mirror_kernel(const float *__restrict__ src, float2 *__restrict__ dst, int nu, int nv) {
    __shared__ float tile[32][33];
    __shared__ float tilem[32][33];
    const long long f = blockIdx.z;
    const float *s = src + f * (long long)nu * nv;
    float2 *d = dst + f * (long long)nu * nv;
    const int u0 = blockIdx.x * 32, v0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int v = v0 + r, u = u0 + threadIdx.x;
        if (u < nu && v < nv) {
            tile[r][threadIdx.x] = s[(long long)v * nu + u];
            tilem[r][threadIdx.x] = s[(long long)(nv - 1 - v) * nu + u];
        }
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int u = u0 + r, v = v0 + threadIdx.x;
        if (u < nu && v < nv) d[(long long)u * nv + v] = make_float2(tile[threadIdx.x][r], tilem[threadIdx.x][r]);
    }
}

// --------------------------------------------------------------------------------------------
// volume MSE: vol in the backprojection's [x][y][z] layout, truth [z][y][x];
// res[z][y][x] = 2 (vol - truth) / N, sum of squared errors in *sse
// --------------------------------------------------------------------------------------------
__device__ double g_sse;  // fdk_volume_mse's accumulator

__global__ void mse_kernel(const float *__restrict__ vol, const float *__restrict__ truth, float *res, int nx, int ny,
                           int nz, double *sse) {
    const long long total = (long long)nx * ny * nz;
    double acc = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const int y = (int)((i / nx) % ny);
        const int z = (int)(i / ((long long)nx * ny));
        const float d = vol[((long long)x * ny + y) * nz + z] - truth[i];
        if (res) res[i] = 2.0f * d / (float)total;
        acc += (double)d * d;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sse, acc);
}

// --------------------------------------------------------------------------------------------
// exact adjoint of the staged backprojection (FDK_BP_FP32 semantics): for every voxel pair
// (z, nz-1-z) and view, the residual is scattered with the gather's weights -- bilinear, the
// 1/w^2 factor, SUBPIXEL's bounds -- into the view's ROWS-layout gradient.  One CTA: 16 x 16
// columns x 8 top slices and their mirrors; per view, two shared-memory boxes (main rows and
// mirror rows) collect the contributions before they are added to global memory.
//
// Contention: a warp covers 16 x 2 columns.  Per view the 16-wide side is laid along the
// volume axis whose neighbours land on different detector columns (the larger |dU|), so the
// lanes of one shared-memory atomic rarely hit the same address; both thread -> column
// mappings keep their residuals in registers.  The boxes are double-buffered and zeroed by the
// flush that reads them, so each view costs one barrier.
//
// Shared-memory float atomics run as load + compare-and-swap loops, so the boxes hold 32-bit
// fixed point and take native integer atomics: per view every contribution w g is scaled by a
// power of two S with |w g| S <= 2^19 for all voxels of the tile (the tile's largest |residual|
// times the largest 1/w^2, found at its corners).  An entry sums at most one term per voxel, so
// it stays below 2048 * 2^19 = 2^30; each term is rounded to the nearest 1/S.  The box is laid
// out u-fastest, so the lanes of one atomic (consecutive detector columns) hit consecutive banks.
// --------------------------------------------------------------------------------------------
constexpr int kAdjR = 8, kAdjBU = 48, kAdjBV = 24;  // box: u extent (fastest) x v extent

struct AdjArgs {
    const float *res;   // [z][y][x]
    float *grad;        // views x nv x nu (ROWS)
    const float *mats;  // 12 per view
    int n, nx, ny, nz, nu, nv;
};

__global__ void __launch_bounds__(256, 3) bp_adjoint_kernel(AdjArgs a) {
    __shared__ int box[2][2][kAdjBV * kAdjBU];  // [buffer][main, mirror], fixed point
    __shared__ float warp_max[8];
    const int tid = threadIdx.x, lx = tid & 15, ly = tid >> 4;
    const int zt = blockIdx.z * kAdjR, nzz = a.nz / 2;
    // residuals of column (x0 + lx, y0 + ly) [mapping 0] and (x0 + ly, y0 + lx) [mapping 1]
    float rm[2][kAdjR], rr[2][kAdjR];
    bool col_ok[2];
#pragma unroll
    for (int mp = 0; mp < 2; mp++) {
        const int xi = blockIdx.x * 16 + (mp ? ly : lx), yi = blockIdx.y * 16 + (mp ? lx : ly);
        col_ok[mp] = xi < a.nx && yi < a.ny;
#pragma unroll
        for (int k = 0; k < kAdjR; k++) {
            const int z = zt + k;
            const bool ok = col_ok[mp] && z < nzz;
            rm[mp][k] = ok ? a.res[((long long)z * a.ny + yi) * a.nx + xi] : 0.f;
            rr[mp][k] = ok ? a.res[((long long)(a.nz - 1 - z) * a.ny + yi) * a.nx + xi] : 0.f;
        }
    }
    // largest |residual| of the tile: the fixed-point range
    float gmax = 0.f;
#pragma unroll
    for (int k = 0; k < kAdjR; k++) gmax = fmaxf(gmax, fmaxf(fabsf(rm[0][k]), fabsf(rr[0][k])));
#pragma unroll
    for (int o = 16; o; o >>= 1) gmax = fmaxf(gmax, __shfl_xor_sync(0xFFFFFFFFu, gmax, o));
    if ((tid & 31) == 0) warp_max[tid >> 5] = gmax;
    for (int i = tid; i < 2 * 2 * kAdjBV * kAdjBU; i += 256) (&box[0][0][0])[i] = 0;
    __syncthreads();
    gmax = warp_max[0];
#pragma unroll
    for (int i = 1; i < 8; i++) gmax = fmaxf(gmax, warp_max[i]);
    if (!(gmax > 0.f)) return;  // the tile adds nothing (the whole CTA leaves together)
    const float zf0 = (float)zt;
    const int corner = tid & 3;
    const float cx = blockIdx.x * 16 + ((corner & 1) ? 15 : 0), cy = blockIdx.y * 16 + ((corner & 2) ? 15 : 0);
    for (int s = 0; s < a.n; s++) {
        const float *m = a.mats + 12 * s;
        const int cur = s & 1;
        // footprint of the tile: lanes 4j .. 4j+3 evaluate one corner each (as the gather kernels)
        float umin, umax, vmin, vmax, du_x, du_y, wtmax;
        {
            const float rw = 1.f / fmaf(m[8], cx, fmaf(m[9], cy, m[11]));
            const float U = fmaf(m[0], cx, fmaf(m[1], cy, m[3])) * rw;
            const float vw = fmaf(m[4], cx, fmaf(m[5], cy, m[7]));
            const float va = fmaf(m[6], zf0, vw) * rw, vb = fmaf(m[6], zf0 + kAdjR - 1, vw) * rw;
            umin = umax = U;
            vmin = fminf(va, vb);
            vmax = fmaxf(va, vb);
            wtmax = rw * rw;  // 1/w is largest at a corner (w is linear in x, y)
            const int base = tid & 28;  // lane of this group's corner 0
            const float u0c = __shfl_sync(0xFFFFFFFFu, U, base);
            du_x = __shfl_sync(0xFFFFFFFFu, U, base | 1) - u0c;
            du_y = __shfl_sync(0xFFFFFFFFu, U, base | 2) - u0c;
#pragma unroll
            for (int o = 1; o <= 2; o <<= 1) {
                umin = fminf(umin, __shfl_xor_sync(0xFFFFFFFFu, umin, o));
                umax = fmaxf(umax, __shfl_xor_sync(0xFFFFFFFFu, umax, o));
                vmin = fminf(vmin, __shfl_xor_sync(0xFFFFFFFFu, vmin, o));
                vmax = fmaxf(vmax, __shfl_xor_sync(0xFFFFFFFFu, vmax, o));
                wtmax = fmaxf(wtmax, __shfl_xor_sync(0xFFFFFFFFu, wtmax, o));
            }
        }
        const int u_lo = (int)floorf(umin) - 1, v_lo = (int)floorf(vmin) - 1;
        const int rows = (int)floorf(umax) + 3 - u_lo, cols = (int)floorf(vmax) + 3 - v_lo;  // u, v extents
        const bool boxed = rows <= kAdjBU && cols <= kAdjBV;
        const int mp = fabsf(du_y) > fabsf(du_x) ? 1 : 0;  // 16 lanes along the axis with the larger |dU|
        int ex;
        frexpf(gmax * wtmax * 1.0001f, &ex);  // |w g| <= gmax * wtmax < 2^ex
        const int e = min(19 - ex, 126);
        const float S = ldexpf(1.f, e), inv_s = ldexpf(1.f, -e);
        int *boxm = box[cur][0], *boxr = box[cur][1];
        float *gv = a.grad + (long long)s * a.nu * a.nv;
        if (mp ? col_ok[1] : col_ok[0]) {
            const float x = (float)(blockIdx.x * 16 + (mp ? ly : lx)), y = (float)(blockIdx.y * 16 + (mp ? lx : ly));
            const float rw = 1.f / fmaf(m[8], x, fmaf(m[9], y, m[11]));
            const float U = fmaf(m[0], x, fmaf(m[1], y, m[3])) * rw;
            const float A = fmaf(m[4], x, fmaf(m[5], y, fmaf(m[6], zf0, m[7]))) * rw;
            const float B = m[6] * rw;
            const float wt = rw * rw;
            if (U >= 0.f && U < (float)(a.nu - 1)) {
                const float fuf = floorf(U);
                const float fu = U - fuf;
                const int u0 = (int)fuf;
#pragma unroll
                for (int k = 0; k < kAdjR; k++) {
                    const float v = fmaf(B, (float)k, A);
                    const float vr = (float)(a.nv - 1) - v;
                    const bool mv = v >= 0.f && v < (float)(a.nv - 1);
                    const bool rv = vr >= 0.f && vr < (float)(a.nv - 1);
                    if (!(mv || rv)) continue;
                    const float vf = fminf(floorf(v), (float)(a.nv - 2));
                    const int vi = (int)vf;
                    const float fv = v - vf;
                    const float w00 = (1 - fu) * (1 - fv) * wt, w10 = fu * (1 - fv) * wt;
                    const float w01 = (1 - fu) * fv * wt, w11 = fu * fv * wt;
                    const float gm = mp ? rm[1][k] : rm[0][k];  // selects, not a dynamic register index
                    const float gr = mp ? rr[1][k] : rr[0][k];
                    if (mv && gm != 0.f) {
                        // main voxel: P[u0][vi], P[u0+1][vi], P[u0][vi+1], P[u0+1][vi+1]
                        const float g = gm;
                        if (boxed) {
                            const float gs = g * S;
                            const int b = (vi - v_lo) * kAdjBU + (u0 - u_lo);
                            atomicAdd(&boxm[b], __float2int_rn(w00 * gs));
                            atomicAdd(&boxm[b + 1], __float2int_rn(w10 * gs));
                            atomicAdd(&boxm[b + kAdjBU], __float2int_rn(w01 * gs));
                            atomicAdd(&boxm[b + kAdjBU + 1], __float2int_rn(w11 * gs));
                        } else {
                            atomicAdd(&gv[(long long)vi * a.nu + u0], w00 * g);
                            atomicAdd(&gv[(long long)vi * a.nu + u0 + 1], w10 * g);
                            atomicAdd(&gv[(long long)(vi + 1) * a.nu + u0], w01 * g);
                            atomicAdd(&gv[(long long)(vi + 1) * a.nu + u0 + 1], w11 * g);
                        }
                    }
                    if (rv && gr != 0.f) {
                        // mirror voxel: weight (1-fv) on row nv-1-vi, fv on row nv-2-vi; box index by vi
                        const float g = gr;
                        if (boxed) {
                            const float gs = g * S;
                            const int b = (vi - v_lo) * kAdjBU + (u0 - u_lo);
                            atomicAdd(&boxr[b], __float2int_rn(w00 * gs));
                            atomicAdd(&boxr[b + 1], __float2int_rn(w10 * gs));
                            atomicAdd(&boxr[b + kAdjBU], __float2int_rn(w01 * gs));
                            atomicAdd(&boxr[b + kAdjBU + 1], __float2int_rn(w11 * gs));
                        } else {
                            const long long r0 = a.nv - 1 - vi, r1 = a.nv - 2 - vi;
                            atomicAdd(&gv[r0 * a.nu + u0], w00 * g);
                            atomicAdd(&gv[r0 * a.nu + u0 + 1], w10 * g);
                            atomicAdd(&gv[r1 * a.nu + u0], w01 * g);
                            atomicAdd(&gv[r1 * a.nu + u0 + 1], w11 * g);
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (boxed) {
            // flush: entry (c, ru) = (v - v_lo, u - u_lo) holds row v (main) / row nv-1-v (mirror),
            // column u; each entry is zeroed as it is read, ready for view s + 2
            for (int i = tid; i < rows * cols; i += 256) {
                const int c = i / rows, ru = i - c * rows;
                const int bi = c * kAdjBU + ru;
                const int qm = boxm[bi], qr = boxr[bi];
                boxm[bi] = 0;
                boxr[bi] = 0;
                const int u = u_lo + ru, v = v_lo + c;
                if (u < 0 || u >= a.nu || v < 0 || v >= a.nv) continue;
                if (qm != 0) atomicAdd(&gv[(long long)v * a.nu + u], (float)qm * inv_s);
                if (qr != 0) atomicAdd(&gv[(long long)(a.nv - 1 - v) * a.nu + u], (float)qr * inv_s);
            }
        }
    }
}

}  // namespace fdk

using namespace fdk;

extern "C" {

int fdk_nn_param_count(void) { return kNParam; }

int fdk_nn_forward(const float *params, const float *x, float *y, int64_t rows, int32_t len, float scale, void *stream) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(params && x && y, "NULL argument");
    FDK_CHECK_ARG(len >= kK && len <= kMaxLen && rows > 0, "row length must be 9..%d", kMaxLen);
    const size_t smem = sizeof(NnFwdShared);
    FDK_CUDA(cudaFuncSetAttribute(nn_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int sms = 0, dev = 0;
    FDK_CUDA(cudaGetDevice(&dev));
    FDK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = (int)std::min<long long>(rows, 2 * sms);  // two resident CTAs per SM
    nn_forward_kernel<<<blocks, kThreads, smem, (cudaStream_t)stream>>>(params, x, y, len, rows, scale);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
    FDK_ABI_END
}

int fdk_nn_backward(const float *params, const float *x, const float *dy, float *dparams, int64_t rows, int32_t len,
                    float scale, void *stream) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(params && x && dy && dparams, "NULL argument");
    FDK_CHECK_ARG(len >= kK && len <= kMaxLen && rows > 0, "row length must be 9..%d", kMaxLen);
    const size_t smem = sizeof(NnBackShared);
    FDK_CUDA(cudaFuncSetAttribute(nn_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int sms = 0, dev = 0;
    FDK_CUDA(cudaGetDevice(&dev));
    FDK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = (int)std::min<long long>(rows, sms);
    FDK_CUDA(cudaMemsetAsync(dparams, 0, sizeof(float) * kNParam, (cudaStream_t)stream));
    nn_backward_kernel<<<blocks, kThreads, smem, (cudaStream_t)stream>>>(params, x, dy, dparams, len, rows, scale);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
    FDK_ABI_END
}

int fdk_adam_step(float *params, const float *grads, float *m, float *v, int64_t n, float lr, float beta1, float beta2,
                  float eps, int64_t t, void *stream) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(params && grads && m && v && n > 0 && t > 0, "bad arguments");
    const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
    adam_kernel<<<(int)ceil_div(n, 256), 256, 0, (cudaStream_t)stream>>>(params, grads, m, v, (int)n, lr, beta1, beta2,
                                                                         eps, c1, c2);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
    FDK_ABI_END
}

int fdk_transmission_noise(float *dev_views, int64_t n, double i0, double mu, uint64_t seed, void *stream) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(dev_views && n > 0 && i0 > 0 && mu > 0, "bad arguments");
    noise_kernel<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(dev_views, n, i0, mu, seed);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
    FDK_ABI_END
}

int fdk_voxelize(const fdk_geometry *g, const double *ell, int32_t n_ell, float *dev_vol, void *stream) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(g && ell && dev_vol && n_ell >= 0 && n_ell <= 64, "bad arguments");
    EllipsoidSet set;
    for (int i = 0; i < 16 * n_ell; i++) set.e[i] = ell[i];
    voxelize_kernel<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(set, n_ell, (int)g->nx, (int)g->ny, (int)g->nz, g->dx,
                                                               g->dy, g->dz, dev_vol);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
    FDK_ABI_END
}

int fdk_rows_to_mirror(const float *dev_rows, void *dev_mirror, int64_t n_views, int32_t nu, int32_t nv, void *stream) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(dev_rows && dev_mirror && n_views > 0 && n_views <= 65535 && nu > 0 && nv > 0, "bad arguments");
    const dim3 grid((unsigned)ceil_div(nu, 32), (unsigned)ceil_div(nv, 32), (unsigned)n_views);
    rows_to_mirror_kernel<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(dev_rows, (float2 *)dev_mirror, nu, nv);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
    FDK_ABI_END
}

int fdk_volume_mse(const float *dev_vol_xyz, const float *dev_truth, float *dev_res, int32_t nx, int32_t ny, int32_t nz,
                   double *sse_host, void *stream) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(dev_vol_xyz && dev_truth && sse_host && nx > 0 && ny > 0 && nz > 0, "bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    // one accumulator per device (a module global), shared by the callers of that device in turn
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    double *d_sse = nullptr;
    FDK_CUDA(cudaGetSymbolAddress((void **)&d_sse, g_sse));
    FDK_CUDA(cudaMemsetAsync(d_sse, 0, sizeof(double), st));
    mse_kernel<<<148 * 8, 256, 0, st>>>(dev_vol_xyz, dev_truth, dev_res, nx, ny, nz, d_sse);
    FDK_CUDA(cudaGetLastError());
    FDK_CUDA(cudaMemcpyAsync(sse_host, d_sse, sizeof(double), cudaMemcpyDeviceToHost, st));
    FDK_CUDA(cudaStreamSynchronize(st));
    return FDK_OK;
    FDK_ABI_END
}

int fdk_bp_adjoint(const fdk_geometry *g, const float *dev_res, const float *dev_mats, int32_t n_views, float *dev_grad,
                   void *stream) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(g && dev_res && dev_mats && dev_grad && n_views > 0, "NULL argument");
    FDK_CHECK_ARG(g->nz % 2 == 0, "the slab-pair adjoint needs an even nz");
    AdjArgs a;
    a.res = dev_res;
    a.grad = dev_grad;
    a.mats = dev_mats;
    a.n = n_views;
    a.nx = (int)g->nx;
    a.ny = (int)g->ny;
    a.nz = (int)g->nz;
    a.nu = (int)g->nu;
    a.nv = (int)g->nv;
    const dim3 grid((unsigned)ceil_div(a.nx, 16), (unsigned)ceil_div(a.ny, 16), (unsigned)ceil_div(a.nz / 2, kAdjR));
    bp_adjoint_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(a);
    FDK_CUDA(cudaGetLastError());
    return FDK_OK;
    FDK_ABI_END
}

}  // extern "C"
