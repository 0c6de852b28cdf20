/*
 * ref_common.h -- TEST INFRASTRUCTURE ONLY (oracle). Helpers shared by the three
 * reference-kernel replay units (ref_fht.cpp, ref_bic.cpp, ref_3d.cpp).
 */
#pragma once
#include <charconv>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "clshim.h"

namespace refcommon {

/* The Java host writes a float placeholder as `"" + f` (Float.toString, the shortest decimal
 * that round-trips) and the OpenCL compiler reads that text back as an unsuffixed decimal
 * literal (a double).  std::to_chars gives the same shortest round-trip text. */
inline double java_float_literal(float f) {
    char buf[64];
    auto res = std::to_chars(buf, buf + sizeof(buf) - 1, f);
    *res.ptr = 0;
    return std::strtod(buf, nullptr);
}

/* Replays a 1-D NDRange `[0, n)` of a kernel functor, in parallel over work-items. */
template <class F>
inline void range1d(long n, F&& kernel) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        clshim::gid[0] = (size_t)i;
        clshim::gid[1] = 0;
        clshim::gid[2] = 0;
        kernel();
    }
}

/* Replays a 3-D NDRange `(nx, ny, nz)`. */
template <class F>
inline void range3d(long nx, long ny, long nz, F&& kernel) {
    long total = nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < total; ++i) {
        long z = i / (nx * ny);
        long r = i - z * nx * ny;
        long y = r / nx;
        long x = r - y * nx;
        clshim::gid[0] = (size_t)x;
        clshim::gid[1] = (size_t)y;
        clshim::gid[2] = (size_t)z;
        kernel();
    }
}

/* readSRRFbuffer's host-side NaN->0 clean-up (LiveSRRF_CL.java:789). */
inline void nan_to_zero(float* p, long n) {
    for (long i = 0; i < n; ++i)
        if (std::isnan(p[i])) p[i] = 0.0f;
}

}  // namespace refcommon
