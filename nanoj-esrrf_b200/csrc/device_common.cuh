// device_common.cuh -- device helpers shared by the RGC kernels of the three paths.
#pragma once
#include <cuda_runtime.h>

namespace esrrf {
namespace dev {

// CGLH >= 0 ? pow(CGLH, S) : 0, NaN -> 0 (liveSRRF_noInterpolation.cl:349-353,
// liveSRRF.cl:357-359, live3DSRRF.cl:429-431); small integer S by repeated products.
__device__ __forceinline__ float cglh_power(float c, float s) {
    if (!(c >= 0.f)) return 0.f;
    if (s == 1.f) return c;
    if (s == 2.f) return c * c;
    if (s == 3.f) return c * c * c;
    if (s == 4.f) {
        const float c2 = c * c;
        return c2 * c2;
    }
    return powf(c, s);
}

// Catmull-Rom kernel, a = 0.5 (liveSRRF.cl:26-35).
__device__ __forceinline__ float cubic(float x) {
    const float a = 0.5f;
    if (x < 0.0f) x = -x;
    float z = 0.0f;
    if (x < 1.0f)
        z = x * x * (x * (-a + 2.0f) + (a - 3.0f)) + 1.0f;
    else if (x < 2.0f)
        z = -a * x * x * x + 5.0f * a * x * x - 8.0f * a * x + 4.0f * a;
    return z;
}

// Bicubic sample when the 4x4 support is interior, else bilinear with extrapolation
// (getInterpolatedValue, liveSRRF.cl:39-133).
__device__ __forceinline__ float sample2d(const float* __restrict__ a, int w, int h, float x, float y) {
    const int u0 = (int)floorf(x);
    const int v0 = (int)floorf(y);
    if (u0 > 0 && u0 < w - 2 && v0 > 0 && v0 < h - 2) {
        float q = 0.0f;
#pragma unroll
        for (int j = 0; j <= 3; j++) {
            const int v = min(max(v0 - 1 + j, 0), h - 1);
            float p = 0.0f;
#pragma unroll
            for (int i = 0; i <= 3; i++) {
                const int u = min(max(u0 - 1 + i, 0), w - 1);
                p = p + __ldg(a + (long)v * w + u) * cubic(x - (float)u);
            }
            q = q + p * cubic(y - (float)v);
        }
        return q;
    }
    const int xb = (int)fminf((float)w - 2, fmaxf(x, 0.0f));
    const int yb = (int)fminf((float)h - 2, fmaxf(y, 0.0f));
    const float xf = x - (float)xb, yf = y - (float)yb;
    const float ll = __ldg(a + (long)yb * w + xb), lr = __ldg(a + (long)yb * w + xb + 1);
    const float ur = __ldg(a + (long)(yb + 1) * w + xb + 1), ul = __ldg(a + (long)(yb + 1) * w + xb);
    const float upper = ul + xf * (ur - ul);
    const float lower = ll + xf * (lr - ll);
    return lower + yf * (upper - lower);
}

// sample2d split into the part that depends only on the position (support, interior test,
// Catmull-Rom weights) and the part that reads the image, for a position sampled in many frames;
// same arithmetic and accumulation order as sample2d.
struct Sample2dAt {
    bool interior;
    int o;               // interior: offset of (u0 - 1, v0 - 1); else of (xb, yb)
    float cx[4], cy[4];  // interior: weights of columns u0 - 1 .. u0 + 2 and rows; else cx[0] = xf, cy[0] = yf
};

__device__ __forceinline__ Sample2dAt sample2d_at(int w, int h, float x, float y) {
    Sample2dAt s;
    const int u0 = (int)floorf(x);
    const int v0 = (int)floorf(y);
    s.interior = u0 > 0 && u0 < w - 2 && v0 > 0 && v0 < h - 2;
    if (s.interior) {
        // the clamps of sample2d are no-ops inside the interior support
        s.o = (v0 - 1) * w + (u0 - 1);
#pragma unroll
        for (int i = 0; i <= 3; i++) {
            s.cx[i] = cubic(x - (float)(u0 - 1 + i));
            s.cy[i] = cubic(y - (float)(v0 - 1 + i));
        }
    } else {
        const int xb = (int)fminf((float)w - 2, fmaxf(x, 0.0f));
        const int yb = (int)fminf((float)h - 2, fmaxf(y, 0.0f));
        s.o = yb * w + xb;
        s.cx[0] = x - (float)xb;
        s.cy[0] = y - (float)yb;
#pragma unroll
        for (int i = 1; i <= 3; i++) s.cx[i] = s.cy[i] = 0.0f;
    }
    return s;
}

__device__ __forceinline__ float sample2d_apply(const float* __restrict__ a, int w, const Sample2dAt& s) {
    const float* r = a + s.o;
    if (s.interior) {
        float q = 0.0f;
#pragma unroll
        for (int j = 0; j <= 3; j++) {
            float p = 0.0f;
#pragma unroll
            for (int i = 0; i <= 3; i++) p = p + __ldg(r + (long)j * w + i) * s.cx[i];
            q = q + p * s.cy[j];
        }
        return q;
    }
    const float xf = s.cx[0], yf = s.cy[0];
    const float ll = __ldg(r), lr = __ldg(r + 1);
    const float ur = __ldg(r + w + 1), ul = __ldg(r + w);
    const float upper = ul + xf * (ur - ul);
    const float lower = ll + xf * (lr - ll);
    return lower + yf * (upper - lower);
}

// sample2d at one position (x, y) of four planes a + plane[k] * pl: the support, the branch and the
// 4 x 4 cubic weights are shared, each plane keeps sample2d's own accumulation order.
__device__ __forceinline__ void sample2d_x4(const float* __restrict__ a, long pl, const int (&plane)[4],
                                            int w, int h, float x, float y, float (&out)[4]) {
    const int u0 = (int)floorf(x);
    const int v0 = (int)floorf(y);
    if (u0 > 0 && u0 < w - 2 && v0 > 0 && v0 < h - 2) {
        int us[4];
        float cx[4];
#pragma unroll
        for (int i = 0; i <= 3; i++) {
            us[i] = min(max(u0 - 1 + i, 0), w - 1);
            cx[i] = cubic(x - (float)us[i]);
        }
        float q[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int j = 0; j <= 3; j++) {
            const int v = min(max(v0 - 1 + j, 0), h - 1);
            const float cy = cubic(y - (float)v);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float* r = a + plane[k] * pl + (long)v * w;
                float p = 0.0f;
#pragma unroll
                for (int i = 0; i <= 3; i++) p = p + __ldg(r + us[i]) * cx[i];
                q[k] = q[k] + p * cy;
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) out[k] = q[k];
        return;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = sample2d(a + plane[k] * pl, w, h, x, y);
}

__device__ __forceinline__ float load_px(const void* raw, int is_u16, long idx) {
    return is_u16 ? (float)__ldg((const unsigned short*)raw + idx) : __ldg((const float*)raw + idx);
}

}  // namespace dev
}  // namespace esrrf
