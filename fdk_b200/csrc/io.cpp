// io.cpp -- the reference's on-disk formats on the reconstruction path.
//
// Projections: one raw little-endian FP32 file per view, nu x nv, u fastest, named
// "<folder>img%04d.raw"; view v lives in file v * step + start (Parameter::GetProjPath,
// common/type.h:4847-4851; LoadProjectionImageFolder, 1797-1828, which refuses the whole folder
// when any file's size is not nu * nv * 4; ProjectionImageT::SaveToFolder, 3848-3861).
// Volumes: ".vol" = three int32 (nx, ny, nz) and then the FP32 voxels, x fastest, z slowest
// (VolumeT::Save / Load, common/type.h:3256-3313); per-slice raw FP32 files of nx * ny voxels
// named by the global slice index (the slice writer of cuFDK/mpiFDK.cpp:548-576, whose name
// also encodes its MPI grid; here "<folder>%06d.raw").
//
// Several files are read or written at once by a few host threads (the reference uses an
// OpenMP loop of 4 threads); the caller's buffer may be pinned memory, which is what
// fdk_recon_push_folder feeds to the device.
#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "common.h"
#include "internal.h"

namespace fdk {

std::string proj_file_path(const char *folder, long long file_index) {
    char name[32];
    std::snprintf(name, sizeof(name), "img%04lld.raw", file_index);
    return std::string(folder) + name;
}

namespace {

long long file_size(const std::string &path) {
    struct stat st;
    if (::stat(path.c_str(), &st) != 0) return -1;
    return (long long)st.st_size;
}

// mkdir -p of the directory part of `path` (MakePathDirIfNeed, common/type.h)
int make_parent_dirs(const std::string &path) {
    for (size_t pos = path.find('/', 1); pos != std::string::npos; pos = path.find('/', pos + 1)) {
        const std::string dir = path.substr(0, pos);
        if (::mkdir(dir.c_str(), 0755) != 0 && errno != EEXIST) {
            set_error("cannot create directory %s: %s", dir.c_str(), std::strerror(errno));
            return FDK_ERR_IO;
        }
    }
    return FDK_OK;
}

int read_exact(const std::string &path, void *dst, size_t bytes) {
    FILE *fp = std::fopen(path.c_str(), "rb");
    if (!fp) {
        set_error("cannot open %s: %s", path.c_str(), std::strerror(errno));
        return FDK_ERR_IO;
    }
    const size_t got = std::fread(dst, 1, bytes, fp);
    std::fclose(fp);
    if (got != bytes) {
        set_error("short read of %s: %zu of %zu bytes", path.c_str(), got, bytes);
        return FDK_ERR_IO;
    }
    return FDK_OK;
}

int write_exact(const std::string &path, const void *const *parts, const size_t *sizes, int n_parts) {
    FDK_TRY(make_parent_dirs(path));
    FILE *fp = std::fopen(path.c_str(), "wb");
    if (!fp) {
        set_error("cannot create %s: %s", path.c_str(), std::strerror(errno));
        return FDK_ERR_IO;
    }
    bool ok = true;
    for (int i = 0; i < n_parts && ok; i++) ok = std::fwrite(parts[i], 1, sizes[i], fp) == sizes[i];
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) {
        set_error("write to %s failed", path.c_str());
        return FDK_ERR_IO;
    }
    return FDK_OK;
}

// run job(i) for i in [0, n) on up to `threads` host threads; first failing status wins
template <typename Job>
int parallel_files(long long n, int threads, Job job) {
    if (threads <= 0) threads = (int)std::min(8u, std::max(1u, std::thread::hardware_concurrency()));
    threads = (int)std::max(1LL, std::min<long long>(threads, n));
    std::atomic<long long> next{0};
    std::atomic<int> status{FDK_OK};
    std::string first_error;
    std::atomic<bool> have_error{false};
    auto worker = [&]() {
        for (long long i; (i = next.fetch_add(1)) < n && status.load() == FDK_OK;) {
            const int rc = job(i);
            if (rc != FDK_OK) {
                int expect = FDK_OK;
                if (status.compare_exchange_strong(expect, rc)) {
                    first_error = fdk_last_error();  // the message of this thread's failure
                    have_error = true;
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; t++) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
    if (have_error) set_error("%s", first_error.c_str());
    return status.load();
}

}  // namespace

int read_views(const char *folder, int nu, int nv, long long first, long long count, int step, int start, float *dst,
               int threads) {
    const size_t frame = (size_t)nu * nv;
    // every file is checked before any is read, as the reference's loader does
    for (long long i = 0; i < count; i++) {
        const std::string p = proj_file_path(folder, (first + i) * step + start);
        const long long sz = file_size(p);
        if (sz != (long long)(frame * sizeof(float))) {
            set_error("%s: %s (expected %zu bytes of FP32, %d x %d)", p.c_str(),
                      sz < 0 ? "missing" : "wrong size", frame * sizeof(float), nu, nv);
            return FDK_ERR_IO;
        }
    }
    return parallel_files(count, threads, [&](long long i) {
        return read_exact(proj_file_path(folder, (first + i) * step + start), dst + i * frame, frame * sizeof(float));
    });
}

}  // namespace fdk

using namespace fdk;

extern "C" {

int fdk_proj_path(const char *folder, int64_t view, int32_t step, int32_t start, char *out, int32_t capacity) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(folder && out && view >= 0 && step >= 1 && start >= 0, "bad arguments");
    const std::string p = proj_file_path(folder, (long long)view * step + start);
    FDK_CHECK_ARG((int64_t)p.size() < capacity, "path needs %zu bytes, capacity %d", p.size() + 1, capacity);
    std::memcpy(out, p.c_str(), p.size() + 1);
    return FDK_OK;
    FDK_ABI_END
}

int fdk_load_proj_folder(const char *folder, int32_t nu, int32_t nv, int64_t first, int64_t count, int32_t step,
                         int32_t start, float *host_views, int32_t threads) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(folder && host_views, "NULL argument");
    FDK_CHECK_ARG(nu > 0 && nv > 0 && first >= 0 && count > 0 && step >= 1 && start >= 0, "bad sizes");
    return read_views(folder, nu, nv, first, count, step, start, host_views, threads);
    FDK_ABI_END
}

int fdk_save_proj_folder(const char *folder, const float *host_views, int32_t nu, int32_t nv, int64_t first,
                         int64_t count, int32_t step, int32_t threads) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(folder && host_views, "NULL argument");
    FDK_CHECK_ARG(nu > 0 && nv > 0 && first >= 0 && count > 0 && step >= 1, "bad sizes");
    const size_t frame = (size_t)nu * nv;
    FDK_TRY(make_parent_dirs(std::string(folder) + "x"));
    return parallel_files(count, threads, [&](long long i) {
        const void *parts[1] = {host_views + i * frame};
        const size_t sizes[1] = {frame * sizeof(float)};
        return write_exact(proj_file_path(folder, (first + i) * step), parts, sizes, 1);
    });
    FDK_ABI_END
}

int fdk_save_volume(const char *path, const float *host_vol, int32_t nx, int32_t ny, int32_t nz) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(path && host_vol && nx > 0 && ny > 0 && nz > 0, "bad arguments");
    const int32_t hdr[3] = {nx, ny, nz};
    const void *parts[2] = {hdr, host_vol};
    const size_t sizes[2] = {sizeof(hdr), sizeof(float) * (size_t)nx * ny * nz};
    return write_exact(path, parts, sizes, 2);
    FDK_ABI_END
}

int fdk_load_volume(const char *path, float *host_vol, int64_t capacity, int32_t *nx, int32_t *ny, int32_t *nz) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(path && nx && ny && nz, "NULL argument");
    int32_t hdr[3];
    FILE *fp = std::fopen(path, "rb");
    if (!fp) {
        set_error("cannot open %s: %s", path, std::strerror(errno));
        return FDK_ERR_IO;
    }
    const bool hdr_ok = std::fread(hdr, sizeof(int32_t), 3, fp) == 3 && hdr[0] > 0 && hdr[1] > 0 && hdr[2] > 0;
    std::fclose(fp);
    if (!hdr_ok) {
        set_error("%s: no valid .vol header", path);
        return FDK_ERR_IO;
    }
    *nx = hdr[0];
    *ny = hdr[1];
    *nz = hdr[2];
    const long long n = (long long)hdr[0] * hdr[1] * hdr[2];
    if (!host_vol) return FDK_OK;  // size query
    FDK_CHECK_ARG(capacity >= n, "capacity %lld < %lld voxels", (long long)capacity, n);
    if (file_size(path) != (long long)(sizeof(hdr) + sizeof(float) * n)) {
        set_error("%s: size does not match its header %d x %d x %d", path, hdr[0], hdr[1], hdr[2]);
        return FDK_ERR_IO;
    }
    fp = std::fopen(path, "rb");
    if (!fp) {
        set_error("cannot open %s: %s", path, std::strerror(errno));
        return FDK_ERR_IO;
    }
    const bool ok = std::fseek(fp, (long)sizeof(hdr), SEEK_SET) == 0 &&
                    std::fread(host_vol, sizeof(float), (size_t)n, fp) == (size_t)n;
    std::fclose(fp);
    if (!ok) {
        set_error("short read of %s", path);
        return FDK_ERR_IO;
    }
    return FDK_OK;
    FDK_ABI_END
}

int fdk_save_volume_slices(const char *folder, const float *host_vol, int32_t nx, int32_t ny, int32_t z0,
                           int32_t depth, int32_t threads) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(folder && host_vol && nx > 0 && ny > 0 && z0 >= 0 && depth > 0, "bad arguments");
    const size_t slice = (size_t)nx * ny;
    FDK_TRY(make_parent_dirs(std::string(folder) + "x"));
    return parallel_files(depth, threads, [&](long long k) {
        char name[32];
        std::snprintf(name, sizeof(name), "%06lld.raw", (long long)z0 + k);
        const void *parts[1] = {host_vol + k * slice};
        const size_t sizes[1] = {slice * sizeof(float)};
        return write_exact(std::string(folder) + name, parts, sizes, 1);
    });
    FDK_ABI_END
}

}  // extern "C"
