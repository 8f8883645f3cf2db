// learn.cu -- the learned residual row filter and what training it needs (no reference
// counterpart: "a small 1D residual filter network (3 conv layers, 32
// channels, kernel 9) refines each ramp-filtered row ... trained on phantoms the project's own
// ray-marching forward projector generates, and backpropagates through BP").
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

#include <vector>

#include "common.h"
#include "internal.h"

namespace fdk {

constexpr int kCh = 32, kK = 9, kHalo = 4;
constexpr int kW1 = 0, kB1 = kW1 + kCh * kK, kW2 = kB1 + kCh, kB2 = kW2 + kCh * kCh * kK, kW3 = kB2 + kCh,
              kB3 = kW3 + kCh * kK, kNParam = kB3 + 1;
constexpr int kMaxLen = 256;  // row length limit (threads per CTA = row length; smem ~180 KB backward)

// --------------------------------------------------------------------------------------------
// fused forward (inference): one CTA per row, thread = position
// --------------------------------------------------------------------------------------------
struct NnShared {
    float w[kNParam];                            // all parameters
    __nv_bfloat16 a1[kCh][kMaxLen + 2 * kHalo];  // layer-1 activations, zero halo
    float x[kMaxLen + 2 * kHalo];
};

__device__ __forceinline__ void nn_load(NnShared &sm, const float *params, const float *xrow, int L, float s) {
    for (int i = threadIdx.x; i < kNParam; i += blockDim.x) sm.w[i] = params[i];
    for (int i = threadIdx.x; i < L + 2 * kHalo; i += blockDim.x) {
        const int p = i - kHalo;
        sm.x[i] = (p >= 0 && p < L) ? xrow[p] * s : 0.f;
        if (i < kHalo || i >= L + kHalo)
            for (int c = 0; c < kCh; c++) sm.a1[c][i] = __float2bfloat16(0.f);
    }
}

// a1 for this thread's position (pre-activation returned in z1 when requested)
__device__ __forceinline__ void nn_layer1(NnShared &sm, int p, int L) {
    if (p >= L) return;
#pragma unroll 4
    for (int c = 0; c < kCh; c++) {
        float z = sm.w[kB1 + c];
#pragma unroll
        for (int k = 0; k < kK; k++) z = fmaf(sm.w[kW1 + c * kK + k], sm.x[p + k], z);
        sm.a1[c][p + kHalo] = __float2bfloat16(fmaxf(z, 0.f));
    }
}

// z2[c] for all 32 output channels of this position
__device__ __forceinline__ void nn_layer2(const NnShared &sm, int p, float (&z2)[kCh]) {
#pragma unroll
    for (int c = 0; c < kCh; c++) z2[c] = sm.w[kB2 + c];
    for (int ci = 0; ci < kCh; ci++) {
#pragma unroll
        for (int k = 0; k < kK; k++) {
            const float a = __bfloat162float(sm.a1[ci][p + k]);
#pragma unroll
            for (int c = 0; c < kCh; c++) z2[c] = fmaf(sm.w[kW2 + (c * kCh + ci) * kK + k], a, z2[c]);
        }
    }
}

__global__ void __launch_bounds__(kMaxLen) nn_forward_kernel(const float *__restrict__ params, const float *x, float *y,
                                                            int L, long long rows, float s) {
    extern __shared__ __align__(16) unsigned char smraw[];
    NnShared &sm = *reinterpret_cast<NnShared *>(smraw);
    __shared__ __nv_bfloat16 a2s[kCh][kMaxLen + 2 * kHalo];
    const int p = threadIdx.x;
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        __syncthreads();
        nn_load(sm, params, x + r * L, L, s);
        if (p < kCh)
            for (int i = 0; i < kHalo; i++) {
                a2s[p][i] = __float2bfloat16(0.f);
                a2s[p][L + kHalo + i] = __float2bfloat16(0.f);
            }
        __syncthreads();
        nn_layer1(sm, p, L);
        __syncthreads();
        if (p < L) {
            float z2[kCh];
            nn_layer2(sm, p, z2);
#pragma unroll
            for (int c = 0; c < kCh; c++) a2s[c][p + kHalo] = __float2bfloat16(fmaxf(z2[c], 0.f));
        }
        __syncthreads();
        if (p < L) {
            float o = sm.w[kB3];
            for (int c = 0; c < kCh; c++)
#pragma unroll
                for (int k = 0; k < kK; k++) o = fmaf(sm.w[kW3 + c * kK + k], __bfloat162float(a2s[c][p + k]), o);
            y[r * L + p] = x[r * L + p] + o / s;
        }
    }
}

// --------------------------------------------------------------------------------------------
// backward: persistent CTAs, rows recomputed, parameter gradients accumulated per CTA
// --------------------------------------------------------------------------------------------
struct NnBackShared {
    NnShared f;
    __nv_bfloat16 a2[kCh][kMaxLen + 2 * kHalo];
    float dz2[kCh][kMaxLen + 2 * kHalo];  // gradient of layer-2 pre-activation, zero halo
    float dz1[kCh][kMaxLen];               // gradient of layer-1 pre-activation
    float d3[kMaxLen + 2 * kHalo];         // dL/do (output gradient, scaled), zero halo
    float gw[kNParam];                     // this CTA's parameter gradients
};

__global__ void __launch_bounds__(kMaxLen) nn_backward_kernel(const float *__restrict__ params, const float *x,
                                                             const float *dy, float *dparams, int L, long long rows,
                                                             float s) {
    extern __shared__ __align__(16) unsigned char smraw[];
    NnBackShared &sm = *reinterpret_cast<NnBackShared *>(smraw);
    const int p = threadIdx.x;
    for (int i = p; i < kNParam; i += blockDim.x) sm.gw[i] = 0.f;
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        __syncthreads();
        nn_load(sm.f, params, x + r * L, L, s);
        for (int i = p; i < L + 2 * kHalo; i += blockDim.x) {
            const int q = i - kHalo;
            // y = x + o / s  ->  dL/do = dL/dy / s
            sm.d3[i] = (q >= 0 && q < L) ? dy[r * L + q] / s : 0.f;
            if (i < kHalo || i >= L + kHalo)
                for (int c = 0; c < kCh; c++) {
                    sm.a2[c][i] = __float2bfloat16(0.f);
                    sm.dz2[c][i] = 0.f;
                }
        }
        __syncthreads();
        nn_layer1(sm.f, p, L);
        __syncthreads();
        float z2[kCh];
        if (p < L) {
            nn_layer2(sm.f, p, z2);
#pragma unroll
            for (int c = 0; c < kCh; c++) sm.a2[c][p + kHalo] = __float2bfloat16(fmaxf(z2[c], 0.f));
        }
        __syncthreads();
        if (p < L) {
            // dz2[c][p] = relu'(z2) * sum_k W3[c][k] d3[p - k + 4]   (transpose conv)
#pragma unroll
            for (int c = 0; c < kCh; c++) {
                float g = 0.f;
#pragma unroll
                for (int k = 0; k < kK; k++) g = fmaf(sm.f.w[kW3 + c * kK + k], sm.d3[p + 2 * kHalo - k], g);
                sm.dz2[c][p + kHalo] = z2[c] > 0.f ? g : 0.f;
            }
        }
        __syncthreads();
        if (p < L) {
            // dz1[ci][p] = relu'(z1) * sum_c sum_k W2[c][ci][k] dz2[c][p - k + 4]
            for (int ci = 0; ci < kCh; ci++) {
                if (__bfloat162float(sm.f.a1[ci][p + kHalo]) <= 0.f) {
                    sm.dz1[ci][p] = 0.f;
                    continue;
                }
                float g = 0.f;
                for (int c = 0; c < kCh; c++)
#pragma unroll
                    for (int k = 0; k < kK; k++)
                        g = fmaf(sm.f.w[kW2 + (c * kCh + ci) * kK + k], sm.dz2[c][p + 2 * kHalo - k], g);
                sm.dz1[ci][p] = g;
            }
        }
        __syncthreads();
        // parameter gradients of this row, summed over positions; thread t owns parameters t, t+B, ...
        for (int i = p; i < kNParam; i += blockDim.x) {
            float g = 0.f;
            if (i < kB1) {  // W1[c][k]: sum_q dz1[c][q] * (s x)[q + k - 4]
                const int c = i / kK, k = i % kK;
                for (int q = 0; q < L; q++) g = fmaf(sm.dz1[c][q], sm.f.x[q + k], g);
            } else if (i < kW2) {  // b1
                const int c = i - kB1;
                for (int q = 0; q < L; q++) g += sm.dz1[c][q];
            } else if (i < kB2) {  // W2[c][ci][k]: sum_q dz2[c][q] * a1[ci][q + k - 4]
                const int j = i - kW2, c = j / (kCh * kK), ci = (j / kK) % kCh, k = j % kK;
                for (int q = 0; q < L; q++) g = fmaf(sm.dz2[c][q + kHalo], __bfloat162float(sm.f.a1[ci][q + k]), g);
            } else if (i < kW3) {  // b2
                const int c = i - kB2;
                for (int q = 0; q < L; q++) g += sm.dz2[c][q + kHalo];
            } else if (i < kB3) {  // W3[c][k]: sum_q d3[q] * a2[c][q + k - 4]
                const int j = i - kW3, c = j / kK, k = j % kK;
                for (int q = 0; q < L; q++) g = fmaf(sm.d3[q + kHalo], __bfloat162float(sm.a2[c][q + k]), g);
            } else {  // b3
                for (int q = 0; q < L; q++) g += sm.d3[q + kHalo];
            }
            sm.gw[i] += g;
        }
    }
    __syncthreads();
    for (int i = p; i < kNParam; i += blockDim.x) atomicAdd(dparams + i, sm.gw[i]);
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
__global__ void voxelize_kernel(const double *__restrict__ ell, int n_ell, int nx, int ny, int nz, double dx, double dy,
                                double dz, float *out) {
    __shared__ double se[64 * 16];
    for (int i = threadIdx.x; i < n_ell * 16; i += blockDim.x) se[i] = ell[i];
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
// --------------------------------------------------------------------------------------------
constexpr int kAdjR = 8, kAdjBH = 48, kAdjBW = 24;  // box: u rows x v columns

struct AdjArgs {
    const float *res;   // [z][y][x]
    float *grad;        // views x nv x nu (ROWS)
    const float *mats;  // 12 per view
    int n, nx, ny, nz, nu, nv;
};

__global__ void __launch_bounds__(256) bp_adjoint_kernel(AdjArgs a) {
    __shared__ float boxm[kAdjBH * kAdjBW], boxr[kAdjBH * kAdjBW];
    __shared__ int meta[6];
    const int tid = threadIdx.x, lx = tid & 15, ly = tid >> 4;
    const int xi = blockIdx.x * 16 + lx, yi = blockIdx.y * 16 + ly, zt = blockIdx.z * kAdjR;
    const bool col_ok = xi < a.nx && yi < a.ny;
    const int nzz = a.nz / 2;
    float rm[kAdjR], rr[kAdjR];
#pragma unroll
    for (int k = 0; k < kAdjR; k++) {
        const int z = zt + k;
        const bool ok = col_ok && z < nzz;
        rm[k] = ok ? a.res[((long long)z * a.ny + yi) * a.nx + xi] : 0.f;
        rr[k] = ok ? a.res[((long long)(a.nz - 1 - z) * a.ny + yi) * a.nx + xi] : 0.f;
    }
    const float x = (float)xi, y = (float)yi, zf0 = (float)zt;
    for (int s = 0; s < a.n; s++) {
        const float *m = a.mats + 12 * s;
        if (tid == 0) {
            // footprint of the block: corners of 16 x 16 columns x 8 slices (as the gather kernels)
            float umin = 3e38f, umax = -3e38f, vmin = 3e38f, vmax = -3e38f;
            for (int c = 0; c < 4; c++) {
                const float cx = blockIdx.x * 16 + ((c & 1) ? 15 : 0), cy = blockIdx.y * 16 + ((c & 2) ? 15 : 0);
                const float rw = 1.f / fmaf(m[8], cx, fmaf(m[9], cy, m[11]));
                const float U = fmaf(m[0], cx, fmaf(m[1], cy, m[3])) * rw;
                const float vw = fmaf(m[4], cx, fmaf(m[5], cy, m[7]));
                const float va = fmaf(m[6], zf0, vw) * rw, vb = fmaf(m[6], zf0 + kAdjR - 1, vw) * rw;
                umin = fminf(umin, U);
                umax = fmaxf(umax, U);
                vmin = fminf(vmin, fminf(va, vb));
                vmax = fmaxf(vmax, fmaxf(va, vb));
            }
            const int u_lo = (int)floorf(umin) - 1, v_lo = (int)floorf(vmin) - 1;
            const int rows = (int)floorf(umax) + 3 - u_lo, cols = (int)floorf(vmax) + 3 - v_lo;
            meta[0] = u_lo;
            meta[1] = v_lo;
            meta[2] = rows;
            meta[3] = cols;
            meta[4] = (rows <= kAdjBH && cols <= kAdjBW) ? 1 : 0;
        }
        for (int i = tid; i < kAdjBH * kAdjBW; i += 256) boxm[i] = boxr[i] = 0.f;
        __syncthreads();
        const int u_lo = meta[0], v_lo = meta[1], rows = meta[2], cols = meta[3];
        const bool boxed = meta[4] != 0;
        float *gv = a.grad + (long long)s * a.nu * a.nv;
        if (col_ok) {
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
                    if (mv && rm[k] != 0.f) {
                        // main voxel: P[u0][vi], P[u0+1][vi], P[u0][vi+1], P[u0+1][vi+1]
                        const float g = rm[k];
                        if (boxed) {
                            const int b = (u0 - u_lo) * kAdjBW + (vi - v_lo);
                            atomicAdd(&boxm[b], w00 * g);
                            atomicAdd(&boxm[b + kAdjBW], w10 * g);
                            atomicAdd(&boxm[b + 1], w01 * g);
                            atomicAdd(&boxm[b + kAdjBW + 1], w11 * g);
                        } else {
                            atomicAdd(&gv[(long long)vi * a.nu + u0], w00 * g);
                            atomicAdd(&gv[(long long)vi * a.nu + u0 + 1], w10 * g);
                            atomicAdd(&gv[(long long)(vi + 1) * a.nu + u0], w01 * g);
                            atomicAdd(&gv[(long long)(vi + 1) * a.nu + u0 + 1], w11 * g);
                        }
                    }
                    if (rv && rr[k] != 0.f) {
                        // mirror voxel: weight (1-fv) on row nv-1-vi, fv on row nv-2-vi; box index by vi
                        const float g = rr[k];
                        if (boxed) {
                            const int b = (u0 - u_lo) * kAdjBW + (vi - v_lo);
                            atomicAdd(&boxr[b], w00 * g);
                            atomicAdd(&boxr[b + kAdjBW], w10 * g);
                            atomicAdd(&boxr[b + 1], w01 * g);
                            atomicAdd(&boxr[b + kAdjBW + 1], w11 * g);
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
            // flush: box (u, c) with c = v - v_lo holds row v (main) / row nv-1-v (mirror), column u
            for (int i = tid; i < rows * cols; i += 256) {
                const int ru = i / cols, c = i - ru * cols;
                const int u = u_lo + ru, v = v_lo + c;
                if (u < 0 || u >= a.nu || v < 0 || v >= a.nv) continue;
                const float gm = boxm[ru * kAdjBW + c], gr = boxr[ru * kAdjBW + c];
                if (gm != 0.f) atomicAdd(&gv[(long long)v * a.nu + u], gm);
                if (gr != 0.f) atomicAdd(&gv[(long long)(a.nv - 1 - v) * a.nu + u], gr);
            }
        }
        __syncthreads();
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
    const size_t smem = sizeof(NnShared);
    FDK_CUDA(cudaFuncSetAttribute(nn_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int blocks = (int)std::min<long long>(rows, 148 * 8);
    nn_forward_kernel<<<blocks, len, smem, (cudaStream_t)stream>>>(params, x, y, len, rows, scale);
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
    nn_backward_kernel<<<blocks, len, smem, (cudaStream_t)stream>>>(params, x, dy, dparams, len, rows, scale);
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
    cudaStream_t st = (cudaStream_t)stream;
    double *d_ell = nullptr;
    FDK_CUDA(cudaMallocAsync((void **)&d_ell, sizeof(double) * 16 * (n_ell > 0 ? n_ell : 1), st));
    if (n_ell > 0) FDK_CUDA(cudaMemcpyAsync(d_ell, ell, sizeof(double) * 16 * n_ell, cudaMemcpyHostToDevice, st));
    voxelize_kernel<<<148 * 8, 256, 0, st>>>(d_ell, n_ell, (int)g->nx, (int)g->ny, (int)g->nz, g->dx, g->dy, g->dz,
                                             dev_vol);
    FDK_CUDA(cudaGetLastError());
    FDK_CUDA(cudaFreeAsync(d_ell, st));
    FDK_CUDA(cudaStreamSynchronize(st));
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
    double *d_sse = nullptr;
    FDK_CUDA(cudaMallocAsync((void **)&d_sse, sizeof(double), st));
    FDK_CUDA(cudaMemsetAsync(d_sse, 0, sizeof(double), st));
    mse_kernel<<<148 * 8, 256, 0, st>>>(dev_vol_xyz, dev_truth, dev_res, nx, ny, nz, d_sse);
    FDK_CUDA(cudaGetLastError());
    FDK_CUDA(cudaMemcpyAsync(sse_host, d_sse, sizeof(double), cudaMemcpyDeviceToHost, st));
    FDK_CUDA(cudaFreeAsync(d_sse, st));
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
