// Shared helpers for the fml_b200 CUDA library (libfmlb.so).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>

#include "../../include/fmlb.h"

namespace fmlb {

// Records a formatted message retrievable through fmlb_last_error_string().
void set_error(const char *fmt, ...);

inline int cuda_status(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return FMLB_ECUDA;
    }
    return FMLB_OK;
}

inline int launch_status(const char *what) {
    return cuda_status(cudaGetLastError(), what);
}

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// Number of SMs of the current device (cached per device).
int sm_count();

}  // namespace fmlb

#define FMLB_REQUIRE(cond, ...)                 \
    do {                                        \
        if (!(cond)) {                          \
            ::fmlb::set_error(__VA_ARGS__);     \
            return FMLB_EINVAL;                 \
        }                                       \
    } while (0)

#define FMLB_TRY(expr)                          \
    do {                                        \
        int rc_ = (expr);                       \
        if (rc_ != FMLB_OK) return rc_;         \
    } while (0)

#define FMLB_STREAM(s) (reinterpret_cast<cudaStream_t>(s))
