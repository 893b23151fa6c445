// Library-wide entry points: error reporting, version, device queries.
#include <stdarg.h>
#include <stdio.h>

#include "common.cuh"

namespace fmlb {

static thread_local char g_last_error[1024] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof g_last_error, fmt, ap);
    va_end(ap);
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

}  // namespace fmlb

extern "C" const char *fmlb_last_error_string(void) { return fmlb::g_last_error; }

extern "C" int fmlb_version(void) { return 1; }
