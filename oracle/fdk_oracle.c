/*
 * fdk_oracle.c -- CPU restatement of the reference FDK hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (fdk_b200/, include/) links,
 * loads or calls this file; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py use it, and only as the checker.
 *
 * Every function restates one piece of the reference (peng-ac/fdk) and cites the
 * file:line it follows.  Two arithmetic flavours are provided:
 *   - "ref32": bit-level emulation of the reference GPU kernel cudaFdkBP, including
 *     its `mad.rz.ftz.f32` fused multiply-adds (cudaBP/cudaBpLib.cuh:5-13), so the
 *     product's parity kernel can be compared bit for bit;
 *   - "f64": the same algorithm in double precision, the accuracy yardstick.
 *
 * Parity pin: the reference ships no golden vectors or known-answer tests
 * (Test/TestTests.cpp is an empty googletest demo).  This oracle is pinned against
 * the reference's own code compiled from its sources (oracle/build_ref.sh):
 * the CPU pieces (filter(), CalculateCosTable, 3dct BackProjection) here, and the
 * GPU kernel cudaFdkBP on a B200 (tests/test_gpu_parity.py).
 */
#include <math.h>
#include <float.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
/* common/type.h uses its own PI literal; the value below is the one it defines. */
#define REF_PI 3.14159265358979323846

/* ------------------------------------------------------------------------- */
/* geometry                                                                   */
/* ------------------------------------------------------------------------- */

/* nextpow2: common/type.h:4418-4425.  Returns 2^(bit length of n), i.e. exact
 * powers of two are doubled (256 -> 512). */
int orc_nextpow2(int n)
{
    unsigned m = (unsigned)n;
    int i = 0;
    for (i = 0; m > 0; i++) m >>= 1;
    return 1 << i;
}

/* filter(strType, len, d): common/type.h:4427-4475 (double version).
 * type: 0 none, 1 ram-lak, 2 shepp-logan, 3 cosine, 4 hamming, 5 hann
 * (s_FILTER_TYPE order, common/type.h:4619-4626).  out has nextpow2(len) entries.
 * Quirks kept: shepp-logan multiplies by sin(w)/(2d)/(w/(2d)) (:4443), hamming
 * divides only the cosine by d (:4457), the `> PI*d` clamp (:4470-4472). */
int orc_filter_design(int type, int len, int d, double *out)
{
    const int order = orc_nextpow2(len);
    const int nf = order / 2 + 1;
    double *filt = (double *)malloc(sizeof(double) * nf);
    if (!filt) return -1;
    for (int i = 0; i < nf; i++) filt[i] = i * 1.0 * 2 / order;
    for (int i = 1; i < nf; i++) {
        const double w = 2 * REF_PI * i / order;
        switch (type) {
        case 0: case 1: break;
        case 2: filt[i] *= sin(w) / (2 * d) / (w / (2 * d)); break;
        case 3: filt[i] *= cos(w / (2.0 * d)); break;
        case 4: filt[i] *= (0.54 + 0.46 * cos(w) / d); break;
        case 5: filt[i] *= (1.0 + cos(w / d)) / 2.0; break;
        default: free(filt); return -2;
        }
    }
    /* vec = [filt, filt[nf-2 .. 1]] (:4467-4469) */
    for (int i = 0; i < nf; i++) out[i] = filt[i];
    for (int j = 0, i = nf; i < order; i++, j++) out[i] = filt[nf - 2 - j];
    for (int i = 0; i < order; i++)
        if (out[i] > REF_PI * d) out[i] = 0;
    free(filt);
    return order;
}

/* AngularAndrampFactor: common/type.h:4736. */
double orc_angular_ramp_factor(double du, long n_proj, double sid, double sod)
{
    return 1.0 / 2.0 / du * (2.0 * REF_PI / (double)n_proj) / 2.0 * (sid / sod);
}

/* cos_sigma table: common/type.h:4756-4783 with DetectorCoor<float>
 * (common/type.h:4019-4051).  Arithmetic follows the reference's types: the
 * detector coordinates are float, the distance is formed in double because
 * para.SID is double, the weight is stored as float.  out is nv rows of nu. */
void orc_cos_table(long nu, long nv, double du, double dv, double offset_nu, double offset_nv,
                   double sid, double sod, double aaf, float *out)
{
    const float fdu = (float)du, fdv = (float)dv, fnu = (float)nu, fnv = (float)nv;
    const float centerX = (float)((fnu - 1) / 2.0 + (float)offset_nu);
    const float centerY = (float)((fnv - 1) / 2.0 + (float)offset_nv);
    for (long i = 0; i < nv; i++) {
        for (long j = 0; j < nu; j++) {
            const float u = (float)j - centerX;
            const float v = centerY - (float)i;
            const float uMM = u * fdu;
            const float vMM = v * fdv;
            const float dis = (float)sqrt((double)(uMM * uMM + vMM * vMM) + sid * sid);
            float w = (float)(sid / dis);
            w = (float)(w * (sod * sod * aaf));
            out[i * nu + j] = w;
        }
    }
}

/* 4x4 products of CalculateProjMat (common/type.h:4898-4944) in double.
 * out receives the first three rows (12 values, row major): the 3x4 matrix the
 * GPU kernels use (vec_rot_mat_ijk3x4, common/type.h:4821-4831).  It maps the
 * voxel index (x, y, z, 1) to (u*w, v*w, w) in detector pixels. */
static void mat_mul4(const double *a, const double *b, double *c)
{
    double t[16];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            double s = 0;
            for (int k = 0; k < 4; k++) s += a[i * 4 + k] * b[k * 4 + j];
            t[i * 4 + j] = s;
        }
    memcpy(c, t, sizeof(t));
}

void orc_proj_matrix(long nx, long ny, long nz, double dx, double dy, double dz,
                     long nu, long nv, double du, double dv, double sid, double sod,
                     double angle_rad, double *out12)
{
    const double c = cos(angle_rad), s = sin(angle_rad);
    const double m0[16] = {1, 0, 0, -(nx - 1) / 2.0, 0, -1, 0, (ny - 1) / 2.0,
                           0, 0, -1, (nz - 1) / 2.0, 0, 0, 0, 1};
    const double m1[16] = {dx, 0, 0, 0, 0, dy, 0, 0, 0, 0, dz, 0, 0, 0, 0, 1};
    const double m2[16] = {c, -s, 0, 0, s, c, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    const double m3[16] = {1, 0, 0, 0, 0, 0, -1, 0, 0, 1, 0, sod, 0, 0, 0, 1};
    const double m4[16] = {sid, 0, (nu - 1) / 2.0 * du, 0, 0, sid, (nv - 1) / 2.0 * dv, 0,
                           0, 0, 1, 0, 0, 0, 0, 1};
    const double m5[16] = {1.0 / du, 0, 0, 0, 0, 1.0 / dv, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    double r[16];
    mat_mul4(m5, m4, r);
    mat_mul4(r, m3, r);
    mat_mul4(r, m2, r);
    mat_mul4(r, m1, r);
    mat_mul4(r, m0, r);
    memcpy(out12, r, sizeof(double) * 12);
}

/* ------------------------------------------------------------------------- */
/* ramp filter (rows)                                                         */
/* ------------------------------------------------------------------------- */

static void fft64(double complex *x, int n, int inverse)
{
    /* iterative radix-2, in place; inverse is unscaled */
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { double complex t = x[i]; x[i] = x[j]; x[j] = t; }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const double ang = 2 * M_PI / len * (inverse ? 1 : -1);
        for (int i = 0; i < n; i += len)
            for (int k = 0; k < len / 2; k++) {
                const double complex w = cos(ang * k) + I * sin(ang * k);
                const double complex a = x[i + k], b = x[i + k + len / 2] * w;
                x[i + k] = a + b;
                x[i + k + len / 2] = a - b;
            }
    }
}

/* Row filter of one view, double precision.
 * Follows FilterEngine::Filtering (Filterlib/FilterLib.h:167-196):
 *   p *= cos_table                                  (FilterCosCorrect, :8-13)
 *   each row: place at offset (W-nu)>>1, left pad = mean of the first `pad_n`
 *   samples, right pad = mean of the last `pad_n`   (FilterImageRow, :21-47)
 *   FFT, multiply by H, inverse FFT / W, crop       (:49-56, IppLib.h:76)
 *   optional transpose to (nu rows x nv columns)    (:188-189)
 * pad_n = 4 is the IPP plugin (FilterLib.h:38,44); pad_n = 3 is the cuFFT plugin
 * (FilterlibCufft/cudaFftFilter.cu:25,29) and the Bourke CPU path (type.h:4202-4203).
 * cos_table may be NULL (no weighting).  src/dst are float, math is double. */
int orc_filter_view(const float *src, float *dst, long nu, long nv, const float *cos_table,
                    const double *H, int W, int pad_n, int transpose)
{
    if (W < nu || pad_n < 1 || pad_n > nu) return -1;
    double complex *buf = (double complex *)malloc(sizeof(double complex) * W);
    if (!buf) return -2;
    const long off = (W - nu) >> 1;
    for (long r = 0; r < nv; r++) {
        double *row = (double *)malloc(sizeof(double) * nu);
        for (long c = 0; c < nu; c++) {
            double p = src[r * nu + c];
            if (cos_table) p *= (double)cos_table[r * nu + c];
            row[c] = p;
        }
        double lv = 0, rv = 0;
        for (int k = 0; k < pad_n; k++) { lv += row[k]; rv += row[nu - 1 - k]; }
        lv /= pad_n; rv /= pad_n;
        for (long k = 0; k < W; k++) {
            double val;
            if (k < off) val = lv;
            else if (k < off + nu) val = row[k - off];
            else val = rv;
            buf[k] = val;
        }
        fft64(buf, W, 0);
        for (long k = 0; k < W; k++) buf[k] *= H[k];
        fft64(buf, W, 1);
        for (long c = 0; c < nu; c++) {
            const double y = creal(buf[off + c]) / W;
            if (transpose) dst[c * nv + r] = (float)y;
            else dst[r * nu + c] = (float)y;
        }
        free(row);
    }
    free(buf);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* backprojection                                                             */
/* ------------------------------------------------------------------------- */

/* mad.rz.ftz.f32 (cudaBP/cudaBpLib.cuh:5-13): a*b+c rounded once toward zero,
 * subnormal inputs and results flushed to zero.  a*b is exact in double; the
 * double sum s and its TwoSum error e represent a*b+c exactly; the float nearest
 * to s is stepped one ulp toward zero when it lies beyond the exact value. */
static inline float ftz(float x) { return (fabsf(x) < FLT_MIN) ? copysignf(0.0f, x) : x; }

float orc_fma_rz(float a, float b, float c)
{
    a = ftz(a); b = ftz(b); c = ftz(c);
    const double p = (double)a * (double)b;
    const double s = p + (double)c;
    const double bb = s - p;
    const double e = (p - (s - bb)) + ((double)c - bb);
    if (s == 0.0 && e == 0.0) {
        /* exact zero: sign as IEEE fma in round-toward-zero mode */
        const int neg_p = signbit(p) != 0, neg_c = signbit((double)c) != 0;
        return (neg_p && neg_c) ? -0.0f : 0.0f;
    }
    float f = (float)s;
    if (isinf(f)) return ftz(nextafterf(f, 0.0f));
    const double d = (double)f - s; /* exact: f and s are within one float ulp */
    const double diff = d - e;      /* sign of (f - exact) */
    if (s > 0 || (s == 0 && e > 0)) {
        if (diff > 0) f = nextafterf(f, 0.0f);
    } else {
        if (diff < 0) f = nextafterf(f, 0.0f);
    }
    return ftz(f);
}

static inline float dot_ijkw_rz(const float *m4, float k, float j, float i)
{
    /* dotIJKW: cudaBP/cudaBpLib.cuh:31-44 */
    float sum = m4[3];
    sum = orc_fma_rz(m4[0], k, sum);
    sum = orc_fma_rz(m4[1], j, sum);
    sum = orc_fma_rz(m4[2], i, sum);
    return sum;
}

/* SUBPIXEL: cudaBP/backprojectionFDK.cu:15-48 (bilinear, zero outside
 * [0, width-1) x [0, height-1), mad.rz blends). */
static inline float subpixel_rz(const float *proj, long pitch, int width, int height, float u, float v)
{
    if (u >= 0 && u < width - 1 && v >= 0 && v < height - 1) {
        const float iu = floorf(u), iv = floorf(v);
        const int nu = (int)iu, nv = (int)iv;
        const float du = u - iu, dv = v - iv;
        const float _du = (float)(1.0 - du), _dv = (float)(1.0 - dv);
        const float *p0 = proj + (long)nv * pitch + nu;
        const float *p1 = p0 + pitch;
        float x0 = p0[0], x1 = p0[1], x2 = p1[0], x3 = p1[1];
        x0 = orc_fma_rz(x0, _du, x1 * du);
        x2 = orc_fma_rz(x2, _du, x3 * du);
        return orc_fma_rz(x0, _dv, x2 * dv);
    }
    return 0.0f;
}

/* One launch of cudaFdkBP<TRANSPOSE=1, false, bSymmetric>
 * (cudaBP/backprojectionFDK.cu:50-129) as issued by BackProjectionFDK::inBP
 * (:240-276).  Views are transposed: view s is `height` rows (detector columns u)
 * of `width` values (detector rows v), pitch == width.  vol is the device volume
 * layout [x][y][zs] with zs = top slab then (if symmetric) bottom slab, i.e.
 * offset = (kk*ny_sub + jj)*depth_total + ii.  mats: 12 floats per view.
 * top = {x, y, z, width, height, depth}, depth_bottom > 0 selects bSymmetric. */
void orc_bp_ref32(float *vol, const long top[6], long depth_bottom, long nz,
                  const float *proj, int width, int height, const float *mats, int n_proj)
{
    const long D = top[5] + depth_bottom;
    const int sym = depth_bottom > 0;
    const long nzz = sym ? D / 2 : top[5];
    const long fsize = (long)width * height;
#pragma omp parallel for collapse(2) schedule(static)
    for (long kk = 0; kk < top[3]; kk++) {
        for (long jj = 0; jj < top[4]; jj++) {
            for (long ii = 0; ii < nzz; ii++) {
                const float k = (float)(kk + top[0]);
                const float j = (float)(jj + top[1]);
                const float i = (float)(ii + top[2]);
                float sum = 0, _sum = 0;
                for (int s = 0; s < n_proj; s++) {
                    const float *m = mats + 12 * s;
                    const float Z = 1.f / dot_ijkw_rz(m + 8, k, j, i);
                    const float U = dot_ijkw_rz(m + 0, k, j, i) * Z;
                    const float f = Z;
                    const float f2 = f * f;
                    const float v = dot_ijkw_rz(m + 4, k, j, i) * f;
                    const float *p = proj + fsize * s;
                    sum = orc_fma_rz(subpixel_rz(p, width, width, height, v, U), f2, sum);
                    if (sym) {
                        const float _v = (float)(width - 1) - v;
                        _sum = orc_fma_rz(subpixel_rz(p, width, width, height, _v, U), f2, _sum);
                    }
                }
                float *out = vol + (kk * top[4] + jj) * D;
                out[ii] += sum;
                if (sym) out[D - 1 - ii] += _sum;
            }
        }
    }
}

/* The same backprojection in double precision (accuracy yardstick).  Views are
 * float (they are the filtered data), matrices double, all arithmetic double.
 * Same bounds rule as SUBPIXEL.  Output layout as orc_bp_ref32. */
void orc_bp_f64(double *vol, const long top[6], long depth_bottom, long nz,
                const float *proj, int width, int height, const double *mats, int n_proj)
{
    const long D = top[5] + depth_bottom;
    const int sym = depth_bottom > 0;
    const long nzz = sym ? D / 2 : top[5];
    const long fsize = (long)width * height;
    (void)nz;
#pragma omp parallel for collapse(2) schedule(static)
    for (long kk = 0; kk < top[3]; kk++) {
        for (long jj = 0; jj < top[4]; jj++) {
            for (long ii = 0; ii < nzz; ii++) {
                const double k = (double)(kk + top[0]);
                const double j = (double)(jj + top[1]);
                const double i = (double)(ii + top[2]);
                double sum = 0, _sum = 0;
                for (int s = 0; s < n_proj; s++) {
                    const double *m = mats + 12 * s;
                    const double Z = 1.0 / (m[8] * k + m[9] * j + m[10] * i + m[11]);
                    const double U = (m[0] * k + m[1] * j + m[2] * i + m[3]) * Z;
                    const double v = (m[4] * k + m[5] * j + m[6] * i + m[7]) * Z;
                    const float *p = proj + fsize * s;
                    for (int pass = 0; pass < (sym ? 2 : 1); pass++) {
                        const double vv = pass ? (width - 1) - v : v;
                        double val = 0;
                        if (vv >= 0 && vv < width - 1 && U >= 0 && U < height - 1) {
                            const double fv = floor(vv), fu = floor(U);
                            const double a = vv - fv, b = U - fu;
                            const float *p0 = p + (long)fu * width + (long)fv;
                            const float *p1 = p0 + width;
                            val = (p0[0] * (1 - a) + p0[1] * a) * (1 - b) + (p1[0] * (1 - a) + p1[1] * a) * b;
                        }
                        if (pass) _sum += val * Z * Z; else sum += val * Z * Z;
                    }
                }
                double *out = vol + (kk * top[4] + jj) * D;
                out[ii] += sum;
                if (sym) out[D - 1 - ii] += _sum;
            }
        }
    }
}

/* ------------------------------------------------------------------------- */
/* FP64 FDK at sampled voxels (accuracy yardstick at full size)                */
/* ------------------------------------------------------------------------- */

/* In-place radix-2 FFT of length W with a precomputed table tw[k] = exp(-2 pi i k / W),
 * k < W/2 (the inverse uses the conjugates and is unscaled). */
static void fft64_tab(double complex *x, int W, const double complex *tw, int inverse)
{
    for (int i = 1, j = 0; i < W; i++) {
        int bit = W >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { double complex t = x[i]; x[i] = x[j]; x[j] = t; }
    }
    for (int len = 2; len <= W; len <<= 1) {
        const int step = W / len;
        for (int i = 0; i < W; i += len)
            for (int k = 0; k < len / 2; k++) {
                const double complex w = inverse ? conj(tw[k * step]) : tw[k * step];
                const double complex a = x[i + k], b = x[i + k + len / 2] * w;
                x[i + k] = a + b;
                x[i + k + len / 2] = a - b;
            }
    }
}

/* FDK in double precision at a list of voxels.  Backprojection is independent per voxel, so a
 * full-size reconstruction can be checked on sampled voxels and whole slices without holding
 * the volume.  For each of the n raw views (nv rows of nu, FP32, consecutive, with their FP64
 * 3x4 matrices):
 *   - the row filter of FilterEngine::Filtering (Filterlib/FilterLib.h:167-196), as
 *     orc_filter_view: optional cosine weight, edge pads of the mean of pad_n samples at offset
 *     (W-nu)>>1, FFT x H, inverse FFT / W, crop -- kept in double (two rows per complex
 *     transform: H is real and even, so the real and imaginary parts filter independently);
 *   - for every listed voxel (x, y, z) (vox: int32 triples, volume index coordinates) the
 *     sample of orc_bp_f64 / cudaFdkBP (cudaBP/backprojectionFDK.cu:80-114): Z = 1/(m2.X),
 *     U = (m0.X) Z, v = (m1.X) Z, bilinear over (U, v) with SUBPIXEL's bounds (0 <= v < nv-1,
 *     0 <= U < nu-1; backprojectionFDK.cu:18), times Z^2, added to out[i] (out accumulates, so
 *     views may come in several calls).
 * edge (optional, n_vox bytes) is set to 1 where some view puts the voxel within 1e-3 px of a
 * border of the bounds rule (the knife-edge voxels, where the rule is discontinuous and a
 * different FP32 rounding switches a whole sample on or off).  Returns 0, or < 0 on bad input. */
int orc_fdk_sampled(const float *views, int n, long nu, long nv, const float *cos_table, const double *H, int W,
                    int pad_n, const double *mats, const int32_t *vox, long n_vox, double *out, uint8_t *edge)
{
    if (W < nu || pad_n < 1 || pad_n > nu || n < 0 || n_vox < 0) return -1;
    double complex *tw = (double complex *)malloc(sizeof(double complex) * (W / 2 > 0 ? W / 2 : 1));
    double *fd = (double *)malloc(sizeof(double) * nu * nv);
    if (!tw || !fd) { free(tw); free(fd); return -2; }
    for (int k = 0; k < W / 2; k++) tw[k] = cos(-2 * M_PI * k / W) + I * sin(-2 * M_PI * k / W);
    const long off = (W - nu) >> 1;
    const long pairs = (nv + 1) / 2;
    for (int s = 0; s < n; s++) {
        const float *src = views + (long)s * nu * nv;
#pragma omp parallel
        {
            double complex *buf = (double complex *)malloc(sizeof(double complex) * W);
            double *row = (double *)malloc(sizeof(double) * 2 * nu);
#pragma omp for schedule(static)
            for (long q = 0; q < pairs; q++) {
                const long r0 = 2 * q, r1 = 2 * q + 1 < nv ? 2 * q + 1 : -1;
                double pad[4] = {0, 0, 0, 0};
                for (int h = 0; h < 2; h++) {
                    const long r = h ? r1 : r0;
                    double *rw = row + h * nu;
                    for (long c = 0; c < nu; c++) {
                        double p = r >= 0 ? src[r * nu + c] : 0.0;
                        if (cos_table && r >= 0) p *= (double)cos_table[r * nu + c];
                        rw[c] = p;
                    }
                    double lv = 0, rv = 0;
                    for (int k = 0; k < pad_n; k++) { lv += rw[k]; rv += rw[nu - 1 - k]; }
                    pad[2 * h] = lv / pad_n;
                    pad[2 * h + 1] = rv / pad_n;
                }
                for (long k = 0; k < W; k++) {
                    double a, b;
                    if (k < off) { a = pad[0]; b = pad[2]; }
                    else if (k < off + nu) { a = row[k - off]; b = row[nu + k - off]; }
                    else { a = pad[1]; b = pad[3]; }
                    buf[k] = a + I * b;
                }
                fft64_tab(buf, W, tw, 0);
                for (long k = 0; k < W; k++) buf[k] *= H[k];
                fft64_tab(buf, W, tw, 1);
                for (long c = 0; c < nu; c++) {
                    fd[c * nv + r0] = creal(buf[off + c]) / W;
                    if (r1 >= 0) fd[c * nv + r1] = cimag(buf[off + c]) / W;
                }
            }
            free(buf);
            free(row);
        }
        const double *m = mats + 12 * (long)s;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n_vox; i++) {
            const double x = vox[3 * i], y = vox[3 * i + 1], z = vox[3 * i + 2];
            const double Z = 1.0 / (m[8] * x + m[9] * y + m[10] * z + m[11]);
            const double U = (m[0] * x + m[1] * y + m[2] * z + m[3]) * Z;
            const double v = (m[4] * x + m[5] * y + m[6] * z + m[7]) * Z;
            if (edge) {
                const double e = 1e-3;
                if (fabs(v) < e || fabs(v - (nv - 1)) < e || fabs(U) < e || fabs(U - (nu - 1)) < e) edge[i] = 1;
            }
            if (v >= 0 && v < nv - 1 && U >= 0 && U < nu - 1) {
                const double fv = floor(v), fu = floor(U);
                const double a = v - fv, b = U - fu;
                const double *p0 = fd + (long)fu * nv + (long)fv;
                const double *p1 = p0 + nv;
                const double val = (p0[0] * (1 - a) + p0[1] * a) * (1 - b) + (p1[0] * (1 - a) + p1[1] * a) * b;
                out[i] += val * Z * Z;
            }
        }
    }
    free(tw);
    free(fd);
    return 0;
}

/* GetVolumeData (cudaBP/backprojectionFDK.cu:278-302 with kernelTransformVolume
 * :131-148): [x][y][zs] -> [zs][y][x] (x fastest).  zs keeps the storage order
 * (top slab ascending, then bottom slab ascending). */
void orc_transform_volume(const float *src, float *dst, long nxs, long nys, long D)
{
    for (long x = 0; x < nxs; x++)
        for (long y = 0; y < nys; y++)
            for (long z = 0; z < D; z++)
                dst[(z * nys + y) * nxs + x] = src[(x * nys + y) * D + z];
}

/* RTK kernel_fdk_3Dgrid + RtkSUBPIXEL
 * (cudaBP/rtkCudaFDKBackProjectionImageFilter.cu:83-112, 156-191), double math.
 * proj: n_proj views of (proj_size[1] rows x proj_size[0] columns), u fastest.
 * vol_out[i + (j + k*ny)*nx] = vol_in[...] + sum_p bilinear(p; u, v) * (1/w)^2.
 * Bilinear is zero outside [0, W-1) x [0, H-1). */
void orc_rtk_bp(const int proj_size[3], const int vol_size[3], const float *mats,
                const float *vol_in, float *vol_out, const float *proj)
{
    const int W = proj_size[0], H = proj_size[1], NP = proj_size[2];
    const long nx = vol_size[0], ny = vol_size[1], nz = vol_size[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (long k = 0; k < nz; k++)
        for (long j = 0; j < ny; j++)
            for (long i = 0; i < nx; i++) {
                double acc = 0;
                for (int p = 0; p < NP; p++) {
                    const float *m = mats + 12 * p;
                    const double x = (double)m[0] * i + (double)m[1] * j + (double)m[2] * k + m[3];
                    const double y = (double)m[4] * i + (double)m[5] * j + (double)m[6] * k + m[7];
                    const double w = 1.0 / ((double)m[8] * i + (double)m[9] * j + (double)m[10] * k + m[11]);
                    const double u = x * w, v = y * w;
                    double s = 0;
                    if (u >= 0 && u < W - 1 && v >= 0 && v < H - 1) {
                        const double iu = floor(u), iv = floor(v);
                        const double du = u - iu, dv = v - iv;
                        const float *p0 = proj + (long)p * W * H + (long)iv * W + (long)iu;
                        const float *p1 = p0 + W;
                        s = (p0[0] * (1 - du) + p0[1] * du) * (1 - dv) + (p1[0] * (1 - du) + p1[1] * du) * dv;
                    }
                    acc += s * w * w;
                }
                const long idx = i + (j + k * ny) * nx;
                vol_out[idx] = (float)((double)vol_in[idx] + acc);
            }
}

/* ------------------------------------------------------------------------- */
/* analytic phantom                                                           */
/* ------------------------------------------------------------------------- */

/* Ellipsoid record: centre (cx,cy,cz) mm, semi-axes (a,b,c) mm, rotation matrix
 * R (9, row major, world = R * local), density rho.  16 doubles per ellipsoid:
 * [cx cy cz a b c R00..R22 rho].  World frame: X = (x - (nx-1)/2)*dx,
 * Y = -(y - (ny-1)/2)*dy, Z = -(z - (nz-1)/2)*dz -- the frame of
 * CalculateProjMat's mat1*mat0 (common/type.h:4906-4917). */
static double chord_len(const double *e, const double o[3], const double d[3])
{
    double po[3] = {o[0] - e[0], o[1] - e[1], o[2] - e[2]};
    const double *R = e + 6;
    /* local = R^T * (p - c) */
    double lo[3], ld[3];
    for (int r = 0; r < 3; r++) {
        lo[r] = R[0 * 3 + r] * po[0] + R[1 * 3 + r] * po[1] + R[2 * 3 + r] * po[2];
        ld[r] = R[0 * 3 + r] * d[0] + R[1 * 3 + r] * d[1] + R[2 * 3 + r] * d[2];
    }
    const double ax[3] = {e[3], e[4], e[5]};
    double A = 0, B = 0, C = -1;
    for (int r = 0; r < 3; r++) {
        const double q = 1.0 / (ax[r] * ax[r]);
        A += ld[r] * ld[r] * q;
        B += 2 * lo[r] * ld[r] * q;
        C += lo[r] * lo[r] * q;
    }
    const double disc = B * B - 4 * A * C;
    if (disc <= 0 || A <= 0) return 0;
    const double dl = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    return sqrt(disc) / A * dl;
}

/* Exact line integrals sum_e rho_e * chord_e for view angle `angle_rad` (the
 * angle CalculateProjMat receives), detector nv rows x nu columns, u fastest.
 * The ray through detector pixel (u, v) is the preimage of the projection
 * matrix: camera origin = source, direction ((u-cu)du, (v-cv)dv, SID) in
 * camera axes; camera -> rotated world: X_r = Xc, Y_r = Zc - SOD, Z_r = -Yc;
 * world = Rz(angle)^T * rotated (inverse of mat3 * mat2, common/type.h:4918-4929). */
void orc_ellipsoid_projection(const double *ell, int n_ell, long nu, long nv, double du, double dv,
                              double sid, double sod, double angle_rad, float *out)
{
    const double c = cos(angle_rad), s = sin(angle_rad);
    const double cu = (nu - 1) / 2.0, cv = (nv - 1) / 2.0;
    /* source in rotated frame (0, -SOD, 0) -> world */
    const double o[3] = {c * 0 + s * (-sod), -s * 0 + c * (-sod), 0};
#pragma omp parallel for schedule(static)
    for (long r = 0; r < nv; r++) {
        for (long q = 0; q < nu; q++) {
            const double xc = (q - cu) * du, yc = (r - cv) * dv, zc = sid;
            const double xr = xc, yr = zc, zr = -yc; /* direction, rotated frame */
            const double d[3] = {c * xr + s * yr, -s * xr + c * yr, zr};
            double sum = 0;
            for (int k = 0; k < n_ell; k++) sum += ell[16 * k + 15] * chord_len(ell + 16 * k, o, d);
            out[r * nu + q] = (float)sum;
        }
    }
}

/* Voxelised phantom (value at voxel centres), volume layout [z][y][x]. */
void orc_ellipsoid_volume(const double *ell, int n_ell, long nx, long ny, long nz,
                          double dx, double dy, double dz, float *out)
{
#pragma omp parallel for collapse(2) schedule(static)
    for (long z = 0; z < nz; z++)
        for (long y = 0; y < ny; y++)
            for (long x = 0; x < nx; x++) {
                const double p[3] = {(x - (nx - 1) / 2.0) * dx, -(y - (ny - 1) / 2.0) * dy,
                                     -(z - (nz - 1) / 2.0) * dz};
                double v = 0;
                for (int k = 0; k < n_ell; k++) {
                    const double *e = ell + 16 * k;
                    const double *R = e + 6;
                    double q = 0;
                    for (int rr = 0; rr < 3; rr++) {
                        const double l = R[0 * 3 + rr] * (p[0] - e[0]) + R[1 * 3 + rr] * (p[1] - e[1]) +
                                         R[2 * 3 + rr] * (p[2] - e[2]);
                        q += l * l / (e[3 + rr] * e[3 + rr]);
                    }
                    if (q <= 1.0) v += e[15];
                }
                out[(z * ny + y) * nx + x] = (float)v;
            }
}

/* ------------------------------------------------------------------------- */
/* ray-marching forward projector                                            */
/* ------------------------------------------------------------------------- */

static inline float vox_clamp(const float *vol, long nx, long ny, long nz, long x, long y, long z)
{
    x = x < 0 ? 0 : (x >= nx ? nx - 1 : x);
    y = y < 0 ? 0 : (y >= ny ? ny - 1 : y);
    z = z < 0 ? 0 : (z >= nz ? nz - 1 : z);
    return vol[(z * ny + y) * nx + x];
}

/* kernel_forwardProject (genProj/cudaForwardProjection.cu:174-254) for one view, FP32 as the
 * reference: the projector rotates by -angle (:426), cuRotate (x c - y s, x s + y c); ray from the
 * source (0, -SOD, 0) to the pixel (u_mm, SID-SOD, v_mm), normalised (:216); cuIntersectBox with the
 * voxel-centre box (:28-48, cudaIterType.cuh:189-199); samples every min(dx,dy,dz) from t_near while
 * t < t_far (:240); Text3DLinear: int3 truncation, texels clamped to the volume, blend z, then y,
 * then x (cudaIterType.cuh:256-270); value = sum * step (:249).  vol [z][y][x]; out nv x nu. */
void orc_forward_project(const float *vol, long nx, long ny, long nz, float dx, float dy, float dz, long nu,
                         long nv, float du, float dv, float sid, float sod, double angle_bp, float *out)
{
    const double ang = -angle_bp;
    const float c = (float)cos(ang), s = (float)sin(ang);
    const float src_y = -sod, det_y = sid - sod;
    const float ox = -src_y * s, oy = src_y * c, oz = 0.f;
    const float cu = (nu - 1) / 2.0f, cv = (nv - 1) / 2.0f;
    const float bx = (nx - 1) / 2.0f * dx, by = (ny - 1) / 2.0f * dy, bz = (nz - 1) / 2.0f * dz;
    const float step = fminf(fminf(dx, dy), dz);
#pragma omp parallel for schedule(static)
    for (long j = 0; j < nv; j++)
        for (long i = 0; i < nu; i++) {
            const float umm = ((float)i - cu) * du, vmm = (cv - (float)j) * dv;
            const float px = umm * c - det_y * s, py = umm * s + det_y * c, pz = vmm;
            float dxr = px - ox, dyr = py - oy, dzr = pz - oz;
            const float inv = 1.0f / sqrtf(dxr * dxr + dyr * dyr + dzr * dzr);
            dxr *= inv;
            dyr *= inv;
            dzr *= inv;
            const float tx0 = (-bx - ox) / dxr, tx1 = (bx - ox) / dxr;
            const float ty0 = (-by - oy) / dyr, ty1 = (by - oy) / dyr;
            const float tz0 = (-bz - oz) / dzr, tz1 = (bz - oz) / dzr;
            const float tnear = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fminf(tz0, tz1));
            const float tfar = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1));
            float sum = 0.f;
            if (tfar > tnear) {
                const float si = ox / dx + (nx - 1) / 2.0f, sj = (ny - 1) / 2.0f - oy / dy,
                            sk = (nz - 1) / 2.0f - oz / dz;
                const float vi = dxr / dx, vj = -dyr / dy, vk = -dzr / dz;
                for (float t = tnear; t < tfar; t += step) {
                    const float pi = si + vi * t, pj = sj + vj * t, pk = sk + vk * t;
                    const long ai = (long)pi, aj = (long)pj, ak = (long)pk;
                    const float fi = pi - ai, fj = pj - aj, fk = pk - ak;
#define V(a, b, cc) vox_clamp(vol, nx, ny, nz, a, b, cc)
                    const float c00 = V(ai, aj, ak) * (1 - fk) + V(ai, aj, ak + 1) * fk;
                    const float c10 = V(ai + 1, aj, ak) * (1 - fk) + V(ai + 1, aj, ak + 1) * fk;
                    const float c01 = V(ai, aj + 1, ak) * (1 - fk) + V(ai, aj + 1, ak + 1) * fk;
                    const float c11 = V(ai + 1, aj + 1, ak) * (1 - fk) + V(ai + 1, aj + 1, ak + 1) * fk;
#undef V
                    const float f0 = c00 * (1 - fj) + c01 * fj, f1 = c10 * (1 - fj) + c11 * fj;
                    sum += f0 * (1 - fi) + f1 * fi;
                }
            }
            out[j * nu + i] = sum * step;
        }
}
