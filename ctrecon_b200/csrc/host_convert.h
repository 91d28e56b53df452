// host_convert.h -- the host threads' FP64 <-> FP32 conversions of the host calls (api.cpp):
// plain loops over a range, the results written with streaming stores where SSE2 is there.
// Header-only so that the CPU tests can build and check them without a GPU.
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__SSE2__)
#include <emmintrin.h>
#endif

namespace ctr {

// dst[i] = (float)src[i], the FP32 results written around the caches (they only go on to
// the device): no read for ownership of the slot lines, a quarter less memory traffic. The
// SSE2 conversion rounds to nearest even, as the cast does.
inline void convert_stream(const double* src, float* dst, size_t n) {
#if defined(__SSE2__)
    size_t i = 0;
    for (; i < n && ((uintptr_t)(dst + i) & 15u) != 0; ++i) dst[i] = (float)src[i];
    for (; i + 4 <= n; i += 4) {
        const __m128 lo = _mm_cvtpd_ps(_mm_loadu_pd(src + i));
        const __m128 hi = _mm_cvtpd_ps(_mm_loadu_pd(src + i + 2));
        _mm_stream_ps(dst + i, _mm_movelh_ps(lo, hi));
    }
    for (; i < n; ++i) dst[i] = (float)src[i];
    _mm_sfence();  // the streamed stores are visible before the slot is handed to the copy
#else
    for (size_t i = 0; i < n; ++i) dst[i] = (float)src[i];
#endif
}

// dst[i] = (double)src[i] (exact), the FP64 results written around the caches.
inline void widen_stream(const float* src, double* dst, size_t n) {
#if defined(__SSE2__)
    size_t i = 0;
    if (((uintptr_t)dst & 7u) == 0) {
        for (; i < n && ((uintptr_t)(dst + i) & 15u) != 0; ++i) dst[i] = (double)src[i];
        for (; i + 2 <= n; i += 2) {
            const __m128 f = _mm_castpd_ps(_mm_load_sd(reinterpret_cast<const double*>(src + i)));
            _mm_stream_pd(dst + i, _mm_cvtps_pd(f));
        }
    }
    for (; i < n; ++i) dst[i] = (double)src[i];
    _mm_sfence();
#else
    for (size_t i = 0; i < n; ++i) dst[i] = (double)src[i];
#endif
}

}  // namespace ctr
