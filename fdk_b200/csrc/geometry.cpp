// geometry.cpp -- FP64 host geometry: the FDK Parameter core (filter response, cosine
// pre-weight table, per-view 3x4 projection matrices) behind the C ABI.
//
// Reference: common/type.h Parameter (4627-4895).  The formulas are the reference's; the
// arithmetic is FP64 throughout and rounded to FP32 only where the GPU consumes FP32.
#include <cmath>
#include <cstring>
#include <new>
#include <stdexcept>
#include <vector>

#include "common.h"

namespace fdk {

namespace {
thread_local std::string g_last_error;
constexpr double kPi = 3.14159265358979323846;
}  // namespace

void set_error(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}
void clear_error() { g_last_error.clear(); }
const char *last_error() { return g_last_error.c_str(); }

static int check_geometry(const fdk_geometry *g) {
    FDK_CHECK_ARG(g != nullptr, "geometry is NULL");
    FDK_CHECK_ARG(g->nx > 0 && g->ny > 0 && g->nz > 0, "volume size must be positive");
    FDK_CHECK_ARG(g->nu > 0 && g->nv > 0, "detector size must be positive");
    FDK_CHECK_ARG(g->dx > 0 && g->dy > 0 && g->dz > 0 && g->du > 0 && g->dv > 0, "pitches must be positive");
    FDK_CHECK_ARG(g->sod > 0 && g->sid > g->sod, "need 0 < SOD < SID");
    FDK_CHECK_ARG(g->n_proj > 0, "n_proj must be positive");
    FDK_CHECK_ARG(g->filter_type >= FDK_FILTER_NONE && g->filter_type <= FDK_FILTER_HANN, "bad filter_type");
    return FDK_OK;
}

// 3x4 matrix mapping the voxel index (x, y, z, 1) to (u*w, v*w, w) for view angle `a`.
// Closed form of S * K * E * R(a) * D * C of CalculateProjMat (common/type.h:4898-4944):
//   C: centre, flip y and z       world X = dx(x-cx), Y = -dy(y-cy), Z = -dz(z-cz)
//   R: rotation about z           Xr = cX - sY, Yr = sX + cY
//   E: camera                     Xc = Xr, Yc = -Z, Zc = Yr + SOD   (source at the origin)
//   K, S: pinhole at SID, pixels  u*w = (SID/du) Xc + cu Zc,  v*w = (SID/dv) Yc + cv Zc,  w = Zc
void projection_matrix(const fdk_geometry &g, double a, double *m) {
    const double c = std::cos(a), s = std::sin(a);
    const double cx = (g.nx - 1) / 2.0, cy = (g.ny - 1) / 2.0, cz = (g.nz - 1) / 2.0;
    const double cu = (g.nu - 1) / 2.0, cv = (g.nv - 1) / 2.0;
    const double ku = g.sid / g.du, kv = g.sid / g.dv;
    // rotated-frame coordinates as affine forms in (x, y, z, 1)
    const double Xr[4] = {c * g.dx, s * g.dy, 0.0, -c * g.dx * cx - s * g.dy * cy};
    const double Zc[4] = {s * g.dx, -c * g.dy, 0.0, -s * g.dx * cx + c * g.dy * cy + g.sod};
    const double Yc[4] = {0.0, 0.0, g.dz, -g.dz * cz};
    for (int k = 0; k < 4; k++) {
        m[0 + k] = ku * Xr[k] + cu * Zc[k];
        m[4 + k] = kv * Yc[k] + cv * Zc[k];
        m[8 + k] = Zc[k];
    }
}

}  // namespace fdk

using namespace fdk;

extern "C" {

const char *fdk_last_error(void) { return fdk::last_error(); }
int fdk_abi_version(void) { return FDK_ABI_VERSION; }

int fdk_device_count(int *count) {
    FDK_CHECK_ARG(count != nullptr, "count is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return FDK_OK;
}

// Parameter::Parameter() defaults (common/type.h:4628-4662).
void fdk_geometry_default(fdk_geometry *g) {
    if (!g) return;
    std::memset(g, 0, sizeof(*g));
    g->nx = g->ny = g->nz = 512;
    g->dx = g->dy = 0.157;
    g->dz = 0.146;
    g->nu = 608;
    g->nv = 616;
    g->du = g->dv = 0.2;
    g->sod = 468;
    g->sid = 700.0;
    g->direction = -1;
    g->scan_angle = 360;
    g->n_proj = 512;
    g->offset_nu = g->offset_nv = 0;
    g->volume_position_angle = -kPi * 48.8671875 / 180.0;
    g->filter_type = FDK_FILTER_SHEPP_LOGAN;
}

// nextpow2 (common/type.h:4418-4425): 2^(bit length of n).
int64_t fdk_filter_length(int64_t nu) {
    if (nu <= 0) return 0;
    int bits = 0;
    for (uint64_t m = (uint64_t)nu; m; m >>= 1) bits++;
    return int64_t(1) << bits;
}

// filter() (common/type.h:4427-4475): ramp 2k/W up to k = W/2, windowed, mirrored.
// The window formulas keep the reference's exact expressions (including the shepp-logan
// and hamming quirks) so that the response is identical.
int fdk_filter_design(int32_t type, int64_t len, int32_t d, double *out, int64_t out_len) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(out != nullptr, "out is NULL");
    FDK_CHECK_ARG(len > 0 && d > 0, "len and d must be positive");
    FDK_CHECK_ARG(type >= FDK_FILTER_NONE && type <= FDK_FILTER_HANN, "bad filter type %d", type);
    const int64_t W = fdk_filter_length(len);
    FDK_CHECK_ARG(out_len >= W, "out_len %lld < W %lld", (long long)out_len, (long long)W);
    const int64_t half = W / 2;
    for (int64_t k = 0; k <= half; k++) {
        double r = k * 1.0 * 2 / W;
        if (k > 0) {
            const double w = 2 * kPi * k / W;
            switch (type) {
            case FDK_FILTER_SHEPP_LOGAN: r *= std::sin(w) / (2 * d) / (w / (2 * d)); break;
            case FDK_FILTER_COSINE: r *= std::cos(w / (2.0 * d)); break;
            case FDK_FILTER_HAMMING: r *= (0.54 + 0.46 * std::cos(w) / d); break;
            case FDK_FILTER_HANN: r *= (1.0 + std::cos(w / d)) / 2.0; break;
            default: break;
            }
        }
        out[k] = r;
        if (k > 0 && k < half) out[W - k] = r;  // even extension
    }
    for (int64_t k = 0; k < W; k++)
        if (out[k] > kPi * d) out[k] = 0;
    return FDK_OK;
    FDK_ABI_END
}

int fdk_angular_ramp_factor(const fdk_geometry *g, double *out) {
    FDK_ABI_BEGIN
    FDK_TRY(check_geometry(g));
    FDK_CHECK_ARG(out != nullptr, "out is NULL");
    // 1/(2 du) * (2 pi / N) / 2 * (SID / SOD)   (common/type.h:4736)
    *out = 1.0 / 2.0 / g->du * (2.0 * kPi / (double)g->n_proj) / 2.0 * (g->sid / g->sod);
    return FDK_OK;
    FDK_ABI_END
}

// cos_sigma(u, v) = SID / sqrt(u_mm^2 + v_mm^2 + SID^2) * SOD^2 * AAF   (common/type.h:4756-4783),
// pixel centre (nu-1)/2 + offset_nu, rows counted downward from (nv-1)/2 + offset_nv (4019-4051).
int fdk_cos_table(const fdk_geometry *g, float *out) {
    FDK_ABI_BEGIN
    FDK_TRY(check_geometry(g));
    FDK_CHECK_ARG(out != nullptr, "out is NULL");
    double aaf = 0;
    FDK_TRY(fdk_angular_ramp_factor(g, &aaf));
    const double cu = (g->nu - 1) / 2.0 + g->offset_nu;
    const double cv = (g->nv - 1) / 2.0 + g->offset_nv;
    const double scale = g->sod * g->sod * aaf;
    for (int64_t r = 0; r < g->nv; r++) {
        const double vmm = (cv - r) * g->dv;
        for (int64_t q = 0; q < g->nu; q++) {
            const double umm = (q - cu) * g->du;
            const double w = g->sid / std::sqrt(umm * umm + vmm * vmm + g->sid * g->sid);
            out[r * g->nu + q] = (float)(w * scale);
        }
    }
    return FDK_OK;
    FDK_ABI_END
}

// csc_sigma = 1 / cos_sigma, taken of the stored FP32 value in FP64 (common/type.h:4784).
int fdk_csc_table(const fdk_geometry *g, float *out) {
    FDK_ABI_BEGIN
    FDK_TRY(fdk_cos_table(g, out));
    const int64_t n = g->nu * g->nv;
    for (int64_t i = 0; i < n; i++) out[i] = (float)(1.0 / (double)out[i]);
    return FDK_OK;
    FDK_ABI_END
}

int fdk_view_angles(const fdk_geometry *g, double *out) {
    FDK_ABI_BEGIN
    FDK_TRY(check_geometry(g));
    FDK_CHECK_ARG(out != nullptr, "out is NULL");
    for (int64_t i = 0; i < g->n_proj; i++) {
        const double deg = i * g->scan_angle / double(g->n_proj);
        out[i] = g->direction * deg / 180.0 * kPi + g->volume_position_angle;
    }
    return FDK_OK;
    FDK_ABI_END
}

int fdk_projection_matrices(const fdk_geometry *g, double *out_f64, float *out_f32) {
    FDK_ABI_BEGIN
    FDK_TRY(check_geometry(g));
    FDK_CHECK_ARG(out_f64 || out_f32, "both outputs are NULL");
    std::vector<double> ang(g->n_proj);
    FDK_TRY(fdk_view_angles(g, ang.data()));
    double m[12];
    for (int64_t i = 0; i < g->n_proj; i++) {
        projection_matrix(*g, ang[i], m);
        for (int k = 0; k < 12; k++) {
            if (out_f64) out_f64[12 * i + k] = m[k];
            if (out_f32) out_f32[12 * i + k] = (float)m[k];
        }
    }
    return FDK_OK;
    FDK_ABI_END
}

}  // extern "C"
