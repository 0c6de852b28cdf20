/*
 * clshim.h -- TEST INFRASTRUCTURE ONLY (oracle). Never linked into the product.
 *
 * Lets the reference's OpenCL C kernel sources (resources/liveSRRF_noInterpolation.cl,
 * resources/liveSRRF.cl, resources/live3DSRRF.cl) compile unchanged as C++ on the host,
 * so that the reference's own kernel arithmetic can serve as the FP32 parity target.
 *
 * The reference specialises its kernels by replacing `$PLACEHOLDER$` tokens with Java
 * `"" + value` strings (nanoj/liveSRRF/LiveSRRF_CL.java:311-342, 496-509).  GCC accepts `$`
 * inside identifiers, so each placeholder is declared here as a namespace-scope variable of
 * the same spelling; the harness (ref_harness.cpp) assigns it the value the Java host would
 * have substituted.  Integer placeholders are `int`; placeholders the Java host formats from
 * a `float` become `double` because the substituted text is an unsuffixed decimal literal,
 * which is a double constant in C and in OpenCL C on fp64-capable devices.
 *
 * get_global_id() reads a per-thread index triple that the harness sets before each call,
 * which replays an NDRange as a plain loop.
 */
#pragma once
#include <cmath>
#include <cstddef>

#define __kernel
#define __global

namespace clshim {
extern thread_local size_t gid[3];
}
static inline size_t get_global_id(int d) { return clshim::gid[d]; }

/* OpenCL integer min/max and the float builtins used by the kernels. */
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }
using std::cos;
using std::exp;
using std::fabs;
using std::floor;
using std::fmax;
using std::fmin;
using std::isnan;
using std::pow;
using std::sin;
using std::sqrt;
