// drop_in.cpp -- the reference pipeline's single-GPU call sequence written against fdk.hpp:
// Parameter tables, FilterEngine::Filtering(src, dst, transpose=true) per view (as
// FilterThread::OnProc, cuFDK/mpiFDK.cpp:122-126), BackProjectionFDK::BP every 32 views (as
// BpThread::PushBpData, :167-203), GetVolumeData at the end (:302).
//   drop_in <views.f32> <out.f32> <n> <nu> <nv> <n_views> <precision>
// views.f32: n_views raw views (nv x nu floats); out: the n^3 volume [z][y][x].
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "fdk.hpp"

int main(int argc, char **argv) {
    if (argc < 8) {
        std::fprintf(stderr, "usage: drop_in views out n nu nv n_views precision\n");
        return 2;
    }
    const int n = atoi(argv[3]), nu = atoi(argv[4]), nv = atoi(argv[5]), nviews = atoi(argv[6]);
    const int precision = atoi(argv[7]);
    fdk_geometry g;
    fdk_geometry_default(&g);
    g.nx = g.ny = g.nz = n;
    g.dx = g.dy = g.dz = 256.0 / n;
    g.nu = nu;
    g.nv = nv;
    g.du = g.dv = 384.0 / nu;
    g.sod = 1000;
    g.sid = 1500;
    g.n_proj = nviews;
    g.volume_position_angle = 0;
    g.filter_type = FDK_FILTER_HANN;
    try {
        const int64_t W = fdk_filter_length(nu);
        std::vector<double> Hd(W);
        fdk::check(fdk_filter_design(g.filter_type, nu, 1, Hd.data(), W));
        std::vector<float> H(Hd.begin(), Hd.end()), cos((size_t)nu * nv), mats((size_t)12 * nviews);
        fdk::check(fdk_cos_table(&g, cos.data()));
        fdk::check(fdk_projection_matrices(&g, nullptr, mats.data()));
        std::vector<float> views((size_t)nviews * nu * nv);
        FILE *f = std::fopen(argv[1], "rb");
        if (!f || std::fread(views.data(), sizeof(float), views.size(), f) != views.size()) return 3;
        std::fclose(f);

        fdk::FilterEngine engine(cos.data(), nu, nv, H);
        fdk::BackProjectionFDK bp(nv, nu, fdk::BackProjectionFDK::MAX_PROJ, n, n, n, fdk::BoxT(0, 0, 0, n, n, n / 2),
                                  fdk::BoxT(0, 0, n / 2, n, n, n / 2), precision);
        std::vector<float> batch((size_t)32 * nu * nv), bmats(12 * 32);
        int count = 0;
        for (int s = 0; s < nviews; s++) {
            engine.Filtering(views.data() + (size_t)s * nu * nv, batch.data() + (size_t)count * nu * nv, true);
            std::copy(mats.begin() + 12 * s, mats.begin() + 12 * s + 12, bmats.begin() + 12 * count);
            if (++count == 32 || s == nviews - 1) {
                bp.BP(1, batch.data(), nv, nu, bmats.data(), count);
                count = 0;
            }
        }
        std::vector<float> vol((size_t)n * n * n);
        bp.GetVolumeData(vol.data(), (int64_t)vol.size());
        std::printf("nBpCount=%lld fKernelTime=%.3f ms\n", (long long)bp.nBpCount(), bp.fKernelTime());
        FILE *o = std::fopen(argv[2], "wb");
        if (!o) return 4;
        std::fwrite(vol.data(), sizeof(float), vol.size(), o);
        std::fclose(o);
    } catch (const fdk::Error &e) {
        std::fprintf(stderr, "%s (code %d)\n", e.what(), e.code);
        return 1;
    }
    return 0;
}
