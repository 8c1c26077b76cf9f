// Error reporting and device queries shared by every translation unit.
#include <stdarg.h>
#include <string.h>

#include <array>

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

// CRC-64 with the ISO polynomial in Go's hash/crc64 convention (reflected, register and result
// complemented), as hotspin's dump writer seals each frame (dump/writer.go:46-76).
HSB_EXPORT uint64_t hsb_crc64_iso(const void* data, int64_t n) {
    static const std::array<uint64_t, 256> table = [] {   // thread-safe one-time set-up
        std::array<uint64_t, 256> t{};
        for (int i = 0; i < 256; i++) {
            uint64_t c = (uint64_t)i;
            for (int b = 0; b < 8; b++) c = (c & 1) ? (c >> 1) ^ 0xD800000000000000ULL : c >> 1;
            t[i] = c;
        }
        return t;
    }();
    if (!data || n <= 0) return 0;
    const unsigned char* p = (const unsigned char*)data;
    uint64_t crc = ~0ULL;
    for (int64_t i = 0; i < n; i++) crc = table[(crc ^ p[i]) & 0xFF] ^ (crc >> 8);
    return ~crc;
}
