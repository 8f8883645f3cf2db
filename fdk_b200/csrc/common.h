// common.h -- internal helpers shared by the libfdk_b200 translation units.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <thread>

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

// Limit of the library's host waits in milliseconds: FDK_WAIT_TIMEOUT_MS, default 10 minutes
// (a whole 2048^3 batch takes about two seconds).
inline long long wait_limit_ms() {
    static const long long ms = [] {
        const char *e = std::getenv("FDK_WAIT_TIMEOUT_MS");
        const long long v = e ? std::atoll(e) : 0;
        return v > 0 ? v : 600000ll;
    }();
    return ms;
}

// Bounded host wait for an event: polls it (yielding for the first millisecond, then sleeping
// 50 us between polls) and returns FDK_ERR_TIMEOUT after timeout_ms (<= 0: wait_limit_ms())
// instead of blocking for good.  Waits for that event only, never for the whole device.
inline int wait_event(cudaEvent_t e, const char *what, long long timeout_ms = 0) {
    const long long limit = timeout_ms > 0 ? timeout_ms : wait_limit_ms();
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t r = cudaEventQuery(e);
        if (r == cudaSuccess) return FDK_OK;
        if (r != cudaErrorNotReady) return cuda_status(r, what, __FILE__, __LINE__);
        const auto us =
            std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count();
        if (us > limit * 1000) return fail(FDK_ERR_TIMEOUT, "%s: not finished after %lld ms", what, limit);
        if (us < 1000) std::this_thread::yield();
        else std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

// Bounded wait for the work queued on a stream so far (an event recorded on it).
inline int wait_stream(cudaStream_t st, cudaEvent_t scratch, const char *what, long long timeout_ms = 0) {
    FDK_CUDA(cudaEventRecord(scratch, st));
    return wait_event(scratch, what, timeout_ms);
}

// Private stream for the one-time copies and memsets of a create call: they are queued on it
// and finish() waits for them (bounded), so kernels on any other stream see the data without a
// device-wide synchronisation.  (A pageable cudaMemcpy may return before its DMA has landed,
// and non-blocking streams do not order after the legacy default stream.)
struct SetupStream {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    int open() {
        FDK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        FDK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        return FDK_OK;
    }
    int finish(const char *what) { return wait_stream(st, ev, what); }
    ~SetupStream() {
        if (st) {
            cudaStreamSynchronize(st);  // error paths: nothing queued may outlive its sources
            cudaStreamDestroy(st);
        }
        if (ev) cudaEventDestroy(ev);
    }
};

}  // namespace fdk
