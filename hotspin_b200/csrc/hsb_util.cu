// Error reporting and device queries shared by every translation unit.
#include <stdarg.h>
#include <string.h>

#include "hsb_common.cuh"

static thread_local char g_err[1024];

void hsb_set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

HSB_EXPORT const char* hsb_last_error(void) { return g_err; }

HSB_EXPORT void hsb_clear_error(void) { g_err[0] = 0; }

int hsb_sm_count() {
    static int cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

HSB_EXPORT int hsb_version(void) { return 1; }
