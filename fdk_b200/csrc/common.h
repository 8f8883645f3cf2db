// common.h -- internal helpers shared by the libfdk_b200 translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/fdk.h"

namespace fdk {

// Thread-local last-error message behind fdk_last_error().
void set_error(const char *fmt, ...);
void clear_error();

// Status carried through the host code; converted to the ABI's int at the boundary.
struct Status {
    int code = FDK_OK;
    bool ok() const { return code == FDK_OK; }
};

inline int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_error("%s", buf);
    return code;
}

inline int cuda_status(cudaError_t e, const char *what, const char *file, int line) {
    if (e == cudaSuccess) return FDK_OK;
    if (e == cudaErrorMemoryAllocation)
        return fail(FDK_ERR_OUT_OF_MEMORY, "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return fail(FDK_ERR_NO_DEVICE, "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    return fail(FDK_ERR_CUDA, "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}

}  // namespace fdk

// Evaluate a CUDA call; on failure record the message and return the status code.
#define FDK_CUDA(call)                                                             \
    do {                                                                           \
        cudaError_t fdk_e_ = (call);                                               \
        if (fdk_e_ != cudaSuccess) return ::fdk::cuda_status(fdk_e_, #call, __FILE__, __LINE__); \
    } while (0)

// Propagate a non-zero int status.
#define FDK_TRY(expr)                 \
    do {                                \
        int fdk_s_ = (expr);            \
        if (fdk_s_ != FDK_OK) return fdk_s_; \
    } while (0)

#define FDK_CHECK_ARG(cond, ...)                                  \
    do {                                                          \
        if (!(cond)) return ::fdk::fail(FDK_ERR_INVALID_ARG, __VA_ARGS__); \
    } while (0)

// ABI guard: no C++ exception crosses extern "C".
#define FDK_ABI_BEGIN try {
#define FDK_ABI_END                                                               \
    }                                                                             \
    catch (const std::bad_alloc &) {                                              \
        return ::fdk::fail(FDK_ERR_OUT_OF_MEMORY, "host allocation failed");      \
    }                                                                             \
    catch (const std::exception &ex) {                                            \
        return ::fdk::fail(FDK_ERR_INVALID_ARG, "exception: %s", ex.what());      \
    }                                                                             \
    catch (...) {                                                                 \
        return ::fdk::fail(FDK_ERR_INVALID_ARG, "unknown exception");             \
    }

namespace fdk {

// Scoped current-device switch (restores the caller's device).
struct DeviceGuard {
    int prev = -1;
    int status = FDK_OK;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        cudaError_t e = cudaSetDevice(dev);
        if (e != cudaSuccess) status = cuda_status(e, "cudaSetDevice", __FILE__, __LINE__);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace fdk
