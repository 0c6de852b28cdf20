// rgc_bic.cu -- the 2-D bicubic ("BIC") path: what LiveSRRF_CL runs with doFHTinterpolation off
// (prepareBuffersBICinterpolation loads liveSRRF.cl, LiveSRRF_CL.java:266-459), and the
// macro-pixel (MP) map correction shared with the 3-D path.
//
// Per frame: 2-point gradient on the raw frame (liveSRRF.cl:187-214), Catmull-Rom 2x resampling
// of the gradient (:217-233), RGC on the 2x gradient grid with bicubic intensity (:238-401).
// Each output pixel is one thread that walks the frames of a launch with its cumulants in
// registers; the reference instead relaunches per frame and read-modify-writes global memory.
#include <math.h>

#include "device_common.cuh"
#include "esrrf_internal.h"

namespace esrrf {

namespace {

using dev::cglh_power;
using dev::load_px;
using dev::sample2d;

__global__ void bic_grad_kernel(const void* raw, int is_u16, int w, int h, float* __restrict__ fraw,
                                float* __restrict__ gx, float* __restrict__ gy) {
    const int x1 = blockIdx.x * blockDim.x + threadIdx.x;
    const int y1 = blockIdx.y;
    const long f = blockIdx.z;
    if (x1 >= w) return;
    const long base = f * (long)w * h;
    const int x0 = max(x1 - 1, 0), y0 = max(y1 - 1, 0);
    const float p = load_px(raw, is_u16, base + (long)y1 * w + x1);
    fraw[base + (long)y1 * w + x1] = p;
    gx[base + (long)y1 * w + x1] = p - load_px(raw, is_u16, base + (long)y1 * w + x0);
    gy[base + (long)y1 * w + x1] = p - load_px(raw, is_u16, base + (long)y0 * w + x1);
}

// Generic 2x lateral resampling of `planes` consecutive [h][w] planes into [2h][2w].
__global__ void grad2x_kernel(const float* __restrict__ g, int w, int h, float* __restrict__ gi) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const long pl = blockIdx.z;
    if (x >= 2 * w) return;
    gi[pl * 4L * w * h + (long)y * 2 * w + x] =
        sample2d(g + pl * (long)w * h, w, h, (float)x / 2.0f, (float)y / 2.0f);
}

__global__ void __launch_bounds__(256) bic_rgc_kernel(BicRgcArgs a) {
    const long pix = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int WM = a.w * a.M, HM = a.h * a.M;
    const long whM = (long)WM * HM;
    if (pix >= whM) return;
    const int yM = (int)(pix / WM), xM = (int)(pix - (long)yM * WM);
    const int w2 = 2 * a.w, h2 = 2 * a.h;
    const int r0 = -(int)(2.0f * a.radius), r1 = (int)(2.0f * a.radius + 1);
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    float prev = a.st.prev[pix];
    for (int f = 0; f < a.F; ++f) {
        const float* gxi = a.gxi + (long)f * w2 * h2;
        const float* gyi = a.gyi + (long)f * w2 * h2;
        const float* fr = a.fraw + (long)f * a.w * a.h;
        // drift is stored x M by the host and used as raw-pixel units (liveSRRF.cl:263-264)
        const float sx = a.shift[f], sy = a.shift[a.F + f];
        const float xc = (float)(((double)xM + 0.5) / a.M + (double)sx);
        const float yc = (float)(((double)yM + 0.5) / a.M + (double)sy);
        const int kx = (int)(2.0f * xc), ky = (int)(2.0f * yc);
        float cglh = 0.f, wsum = 0.f;
        for (int j = r0; j <= r1; ++j) {
            const float vy = ((float)ky + (float)j) / 2.0f;
            if (!(vy > 0 && vy < (float)a.h)) continue;
            for (int i = r0; i <= r1; ++i) {
                const float vx = ((float)kx + (float)i) / 2.0f;
                if (!(vx > 0 && vx < (float)a.w)) continue;
                const float dx = vx - xc, dy = vy - yc;
                const float d = sqrtf(dx * dx + dy * dy);
                if (!(d != 0.f && d <= a.tSO)) continue;
                const int ax = min(max((int)(2 * ((double)vx - 0.5)), 0), w2 - 1);
                const int ay = min(max((int)(2 * ((double)vy - 0.5)), 0), h2 - 1);
                const int ax1 = min(max((int)(2 * ((double)vx - 0.5) + 1), 0), w2 - 1);
                const int ay1 = min(max((int)(2 * ((double)vy - 0.5) + 1), 0), h2 - 1);
                const float Gx = __ldg(gxi + (long)ay * w2 + ax1);
                const float Gy = __ldg(gyi + (long)ay1 * w2 + ax);
                float wt = d * expf(-(d * d) / a.tSS);
                wt = wt * wt * wt * wt;
                wsum += wt;
                if (Gx * dx + Gy * dy < 0) {
                    const float gm = sqrtf(Gx * Gx + Gy * Gy);
                    float dk = fabsf(Gy * dx - Gx * dy) / gm;
                    if (isnan(dk)) dk = d;
                    dk = 1 - dk / d;
                    cglh += dk * wt;
                }
            }
        }
        const float cg = cglh_power(cglh / wsum, a.sens);
        const float v = sample2d(fr, a.w, a.h, (float)xM / (float)a.M + sx - 0.5f,
                                 (float)yM / (float)a.M + sy - 0.5f);
        const float x = a.int_weighting ? v * cg : cg;
        s0 += x;
        s1 += (double)x * x;
        if (a.t0 + f > 0) s2 += (double)x * prev;
        s3 += v;
        prev = x;
    }
    a.st.acc[pix] += s0;
    a.st.acc[whM + pix] += s1;
    a.st.acc[2 * whM + pix] += s2;
    a.st.acc[3 * whM + pix] += s3;
    a.st.prev[pix] = prev;
}

// Mean of each sub-pixel phase of AVG, VAR and TAC2 over all macro-pixels
// (kernelCalculateMPmap, liveSRRF.cl:464-487, live3DSRRF.cl:561-588).  One CTA per phase.
__global__ void mp_map_kernel(const float* __restrict__ out, int w, int h, int P, int M, int is3d,
                              float* __restrict__ map) {
    const int phases = is3d ? M * M * M : M * M;
    const int idx = blockIdx.x;  // c * phases + phase
    const int c = idx / phases, ph = idx - c * phases;
    const int pz = is3d ? ph / (M * M) : 0;
    const int py = (ph - pz * M * M) / M;
    const int px = ph - pz * M * M - py * M;
    const long WM = (long)w * M, HM = (long)h * M, PM = is3d ? (long)P * M : 1;
    const long plane4 = WM * HM * PM;
    const long cells = (long)w * h * (is3d ? P : 1);
    double s = 0.0;
    for (long i = threadIdx.x; i < cells; i += blockDim.x) {
        const long z = i / ((long)w * h);
        const long r = i - z * w * h;
        const long y = r / w, x = r - (r / w) * w;
        const long zz = is3d ? pz + z * M : 0;
        s += out[c * plane4 + zz * WM * HM + (py + y * M) * WM + px + x * M];
    }
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) map[idx] = (float)(red[0] / (double)cells);
}

// Divide AVG, VAR, TAC2 by their phase means, then the readback's NaN->0
// (kernelCorrectMPmap, liveSRRF.cl:490-505, live3DSRRF.cl:591-611).
__global__ void mp_correct_kernel(float* __restrict__ out, int w, int h, int P, int M, int is3d,
                                  const float* __restrict__ map) {
    const long WM = (long)w * M, HM = (long)h * M, PM = is3d ? (long)P * M : 1;
    const long plane4 = WM * HM * PM;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 3 * plane4) return;
    const int c = (int)(idx / plane4);
    const long r = idx - c * plane4;
    const long zM = r / (WM * HM);
    const long yM = (r - zM * WM * HM) / WM;
    const long xM = r - zM * WM * HM - yM * WM;
    const int phases = is3d ? M * M * M : M * M;
    const int ph = (int)((is3d ? (zM % M) * M * M : 0) + (yM % M) * M + (xM % M));
    const float v = out[idx] / map[c * phases + ph];
    out[idx] = isnan(v) ? 0.f : v;
}

}  // namespace

cudaError_t bic_prepare(const void* raw, int is_u16, int w, int h, int F, float* fraw, float* gx,
                        float* gy, float* gxi, float* gyi, cudaStream_t stream) {
    bic_grad_kernel<<<dim3((w + 127) / 128, h, F), 128, 0, stream>>>(raw, is_u16, w, h, fraw, gx, gy);
    grad2x_kernel<<<dim3((2 * w + 127) / 128, 2 * h, F), 128, 0, stream>>>(gx, w, h, gxi);
    grad2x_kernel<<<dim3((2 * w + 127) / 128, 2 * h, F), 128, 0, stream>>>(gy, w, h, gyi);
    return cudaGetLastError();
}

cudaError_t grad2x(const float* g, int w, int h, int planes, float* gi, cudaStream_t stream) {
    grad2x_kernel<<<dim3((2 * w + 127) / 128, 2 * h, planes), 128, 0, stream>>>(g, w, h, gi);
    return cudaGetLastError();
}

cudaError_t bic_rgc(const BicRgcArgs& a, cudaStream_t stream) {
    const long whM = (long)a.w * a.M * a.h * a.M;
    bic_rgc_kernel<<<(unsigned)((whM + 255) / 256), 256, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t mp_correct(float* out, int w, int h, int P, int M, int is3d, float* map,
                       cudaStream_t stream) {
    const int phases = is3d ? M * M * M : M * M;
    mp_map_kernel<<<3 * phases, 256, 0, stream>>>(out, w, h, P, M, is3d, map);
    const long plane4 = (long)w * M * h * M * (is3d ? (long)P * M : 1);
    mp_correct_kernel<<<(unsigned)((3 * plane4 + 255) / 256), 256, 0, stream>>>(out, w, h, P, M, is3d, map);
    return cudaGetLastError();
}

}  // namespace esrrf
