// Shared host helpers for the C ABI: thread-local error reporting, CUDA
// checks and NVTX ranges (one named range per entry point, visible in
// Nsight Systems / ncu range filters; a no-op when no tool is attached).
#pragma once

#include <cstdarg>
#include <cstdio>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "acoustic_rt.h"

namespace ac {

struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

std::string &last_error_slot();

inline int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list args;
    va_start(args, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, args);
    va_end(args);
    last_error_slot() = buf;
    return code;
}

}  // namespace ac

#define AC_CUDA_TRY(expr)                                                                      \
    do {                                                                                       \
        cudaError_t ac_err_ = (expr);                                                          \
        if (ac_err_ != cudaSuccess)                                                            \
            return ac::fail(AC_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,                       \
                            cudaGetErrorString(ac_err_), __FILE__, __LINE__);                  \
    } while (0)
