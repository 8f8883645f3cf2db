// ref_cpu_harness.cpp -- extern "C" entry points around the reference's own CPU
// code, compiled in place from the reference tree by oracle/build_ref.sh.
// TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline), never the product.
//
//   refc_parameter        Parameter::init        common/type.h:4719-4754
//                         (filter() 4427-4475, CalculateCosTable 4756-4833,
//                          CalculateProjMat 4898-4944)
//   refc_filter_rows      filterImageRow         common/type.h:4169-4239 (Bourke FFT, pad 3, double)
//   refc_cpu_fdk          BackProjection<float>  3dct/3dct.cpp:3-241 (cos*AAF, filter, BP) per view,
//                         the angle as CTBackProjection forms it (3dct/3dct.cpp:275)
//   refc_forward_projection  ForwardProjection<float>  3dct/3dct.cpp:430-573, one view, the angle as
//                         CTForwardProjection forms it (3dct/3dct.cpp:594)
#define main ref3dct_main_unused
#include "3dct/3dct.cpp"
#undef main
#include <omp.h>

static void fill_param(Parameter& p, long nx, long ny, long nz, double dx, double dy, double dz,
                       long nu, long nv, double du, double dv, double offset_nu, double offset_nv,
                       double sid, double sod, long direction, double scan_angle, long nproj,
                       double vpa, int filter_type) {
    p.nx = nx; p.ny = ny; p.nz = nz; p.dx = dx; p.dy = dy; p.dz = dz;
    p.nu = nu; p.nv = nv; p.du = du; p.dv = dv;
    p.offset_nu = offset_nu; p.offset_nv = offset_nv;
    p.SID = sid; p.SOD = sod; p.direction = direction; p.scan_angle = scan_angle;
    p.nProj = nproj; p.volume_postion_angle = vpa;
    p.str_filter = s_FILTER_TYPE[filter_type];
    p.init();
}

extern "C" int refc_parameter(long nx, long ny, long nz, double dx, double dy, double dz,
                              long nu, long nv, double du, double dv, double offset_nu, double offset_nv,
                              double sid, double sod, long direction, double scan_angle, long nproj,
                              double vpa, int filter_type,
                              double* out_filter, int out_filter_cap, float* out_cos, float* out_mats,
                              double* out_aaf) {
    try {
        Parameter p;
        fill_param(p, nx, ny, nz, dx, dy, dz, nu, nv, du, dv, offset_nu, offset_nv, sid, sod,
                   direction, scan_angle, nproj, vpa, filter_type);
        const int W = (int)p.fft_kernel_real.size();
        if (out_filter) {
            if (W > out_filter_cap) return -2;
            for (int i = 0; i < W; i++) out_filter[i] = p.fft_kernel_real[i];
        }
        if (out_cos) memcpy(out_cos, p.cos_image_table.cos_sigma.buffer, sizeof(float) * nu * nv);
        if (out_mats) memcpy(out_mats, &p.vec_rot_mat_ijk3x4[0], sizeof(float) * 12 * nproj);
        if (out_aaf) *out_aaf = p.AngularAndrampFactor;
        return W;
    } catch (...) {
        return -1;
    }
}

extern "C" int refc_filter_rows(const double* H, int W, const float* src, float* dst, int width, int height) {
    try {
        std::vector<double> filt(H, H + W);
        filterImageRow(filt, src, dst, width, height);
        return 0;
    } catch (...) {
        return -1;
    }
}

// Full CPU FDK of views [first, first+count) into vol ([z][y][x], accumulated).
// proj holds `count` raw (unfiltered) views, nv rows of nu.  threads <= 0: all.
extern "C" int refc_cpu_fdk(long nx, long ny, long nz, double dx, double dy, double dz,
                            long nu, long nv, double du, double dv, double sid, double sod,
                            long direction, double scan_angle, long nproj, double vpa, int filter_type,
                            const float* proj, int first, int count, float* vol, int threads) {
    try {
        if (threads > 0) omp_set_num_threads(threads);
        Parameter p;
        fill_param(p, nx, ny, nz, dx, dy, dz, nu, nv, du, dv, 0, 0, sid, sod, direction, scan_angle,
                   nproj, vpa, filter_type);
        Volume v(nx, ny, nz);
        memcpy(v.buffer, vol, sizeof(float) * nx * ny * nz);
        VolumeT<ushort> cnt(nx, ny, nz);
        for (int s = 0; s < count; s++) {
            const int idx = first + s;
            FrameT<float> fr(const_cast<float*>(proj) + (size_t)s * nu * nv, (int)nu, (int)nv, idx);
            const double angle_rad = p.direction * p.vec_deg[idx] / 180.0 * PI + p.volume_postion_angle;
            if (!BackProjection<float>(fr, p, angle_rad, v, cnt)) return -3;
        }
        memcpy(vol, v.buffer, sizeof(float) * nx * ny * nz);
        return 0;
    } catch (...) {
        return -1;
    }
}

// Persistent form for timing: the Parameter (init() builds every table) and the volume and
// count buffers are set up once, outside the timed calls.
struct RefFdk {
    Parameter p;
    Volume *vol = nullptr;
    VolumeT<ushort> *cnt = nullptr;
};

extern "C" void* refc_fdk_create(long nx, long ny, long nz, double dx, double dy, double dz,
                                 long nu, long nv, double du, double dv, double sid, double sod,
                                 long direction, double scan_angle, long nproj, double vpa, int filter_type) {
    try {
        RefFdk* h = new RefFdk();
        fill_param(h->p, nx, ny, nz, dx, dy, dz, nu, nv, du, dv, 0, 0, sid, sod, direction, scan_angle,
                   nproj, vpa, filter_type);
        h->vol = new Volume(nx, ny, nz);
        h->cnt = new VolumeT<ushort>(nx, ny, nz);
        return h;
    } catch (...) {
        return nullptr;
    }
}

// Backproject (with cos weighting and filtering, as BackProjection does) views
// [first, first+count) from `proj`; threads <= 0: all.
extern "C" int refc_fdk_run(void* hv, const float* proj, int first, int count, int threads) {
    try {
        RefFdk* h = static_cast<RefFdk*>(hv);
        if (threads > 0) omp_set_num_threads(threads);
        const long nu = h->p.nu, nv = h->p.nv;
        for (int s = 0; s < count; s++) {
            const int idx = first + s;
            FrameT<float> fr(const_cast<float*>(proj) + (size_t)s * nu * nv, (int)nu, (int)nv, idx);
            const double angle_rad = h->p.direction * h->p.vec_deg[idx] / 180.0 * PI + h->p.volume_postion_angle;
            if (!BackProjection<float>(fr, h->p, angle_rad, *h->vol, *h->cnt)) return -3;
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

extern "C" void refc_fdk_destroy(void* hv) {
    RefFdk* h = static_cast<RefFdk*>(hv);
    if (!h) return;
    delete h->vol;
    delete h->cnt;
    delete h;
}

// ForwardProjection<float> (3dct/3dct.cpp:430-573) of a [z][y][x] FP32 volume for view `view`
// of the scan: ray-marched sums of the volume's own trilinear samples x min(dx, dy, dz), nv rows
// of nu into out.  The angle is CTForwardProjection's, -(direction * deg / 180 * PI +
// volume_postion_angle) (3dct/3dct.cpp:594).  threads <= 0: all.
extern "C" int refc_forward_projection(long nx, long ny, long nz, double dx, double dy, double dz,
                                       long nu, long nv, double du, double dv, double sid, double sod,
                                       long direction, double scan_angle, long nproj, double vpa,
                                       const float* vol, int view, float* out, int threads) {
    try {
        if (threads > 0) omp_set_num_threads(threads);
        Parameter p;
        fill_param(p, nx, ny, nz, dx, dy, dz, nu, nv, du, dv, 0, 0, sid, sod, direction, scan_angle,
                   nproj, vpa, 0);
        if (view < 0 || view >= p.nProj) return -2;
        Volume v(nx, ny, nz);
        memcpy(v.buffer, vol, sizeof(float) * nx * ny * nz);
        ImageT<float> image((int)nu, (int)nv);
        ImageT<float> frm((int)nu, (int)nv);
        image.Clear();
        const double angle_rad = -(p.direction * p.vec_deg[view] / 180.0 * PI + p.volume_postion_angle);
        if (!ForwardProjection(p, angle_rad, v, frm.GetFrame(), image)) return -3;
        memcpy(out, image.buffer, sizeof(float) * nu * nv);
        return 0;
    } catch (...) {
        return -1;
    }
}
