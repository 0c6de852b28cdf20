// rgc_fht.cu -- radial gradient convergence on Fourier-interpolated frames (the default 2-D
// path: LiveSRRF_CL.prepareBuffersFHTinterpolation loads liveSRRF_noInterpolation.cl,
// LiveSRRF_CL.java:462-579).
//
// Two kernels compute the same map:
//  * fht_rgc_plain_kernel: one thread per output pixel, the reference's per-tap arithmetic
//    (liveSRRF_noInterpolation.cl:245-393) on a separately computed Roberts-cross gradient
//    (:138-159); handles frames with drift.  Cumulants are kept in registers across the frames
//    of one launch instead of the reference's per-frame global read-modify-write.
//  * fht_rgc_fused_kernel: 32x64-pixel output tiles; per frame it stages the interpolated tile
//    plus the RGC halo in shared memory, forms the unit gradient field there, and runs the tap
//    loop with each thread owning 8 vertically adjacent outputs so that one shared-memory load
//    feeds up to 8 taps.  With zero drift the tap offsets are integers (dx = i, dy = j), so the
//    distance weights are a per-launch table and the contribution of an inward tap reduces to
//    w - (w/d) |g_y i - g_x j| on the unit gradient g.
#include <math.h>

#include <algorithm>

#include "device_common.cuh"
#include "esrrf_internal.h"
#include "fht_fused.cuh"

namespace esrrf {

FhtGeometry fht_geometry(int M, float fwhm, int sensitivity) {
    // Java float arithmetic of prepareBuffersFHTinterpolation (LiveSRRF_CL.java:490-500).
    FhtGeometry g;
    const float Mf = (float)M;
    g.sigma = fwhm / 2.354f;
    float t = 2.0f * g.sigma;
    t = t * Mf;
    t = t * g.sigma;
    t = t * Mf;
    g.tSS = t;
    g.tSO = (2.0f * g.sigma + 1.0f) * Mf;
    g.radius = Mf * ((float)((int)(2.0f * g.sigma)) + 1.0f);
    g.r0 = -(int)g.radius;
    g.r1 = (int)(g.radius + 1.0f);
    g.S = g.r1 - g.r0 + 1;
    g.sensitivity = (float)sensitivity;
    const int S = g.S;
    g.w.assign((size_t)S * S, 0.f);
    g.wd.assign((size_t)S * S, 0.f);
    g.jlo.assign(S, S);
    g.jhi.assign(S, -1);
    float wsum = 0.f;
    for (int jj = 0; jj < S; ++jj) {
        for (int ii = 0; ii < S; ++ii) {
            const int i = g.r0 + ii, j = g.r0 + jj;
            const float d = sqrtf((float)(i * i + j * j));
            if (!(d != 0.f && d <= g.tSO)) continue;
            const float dd = d * d;
            float w = d * expf(-dd / g.tSS);
            w = w * w * w * w;
            g.w[(size_t)jj * S + ii] = w;
            g.wd[(size_t)jj * S + ii] = w / d;
            wsum += w;
            g.jlo[ii] = std::min(g.jlo[ii], jj);
            g.jhi[ii] = std::max(g.jhi[ii], jj);
        }
    }
    g.wsum_interior = wsum;
    return g;
}

namespace {

using dev::cglh_power;
using dev::sample2d;

__global__ void robx_kernel(const float* __restrict__ p, int W, int H, long plane,
                            float* __restrict__ gx, float* __restrict__ gy) {
    const int x1 = blockIdx.x * blockDim.x + threadIdx.x;
    const int y1 = blockIdx.y;
    const long f = blockIdx.z;
    if (x1 >= W) return;
    const int x0 = max(x1 - 1, 0), y0 = max(y1 - 1, 0);
    const float* q = p + f * plane;
    const float a = q[(long)y0 * W + x1], b = q[(long)y1 * W + x0];
    const float c = q[(long)y1 * W + x1], d = q[(long)y0 * W + x0];
    gx[f * plane + (long)y1 * W + x1] = a - b + c - d;
    gy[f * plane + (long)y1 * W + x1] = -a + b + c - d;
}

struct PlainParams {
    float tSS, tSO, radius, sens;
};

__global__ void __launch_bounds__(256) fht_rgc_plain_kernel(FhtRgcArgs a, PlainParams pp) {
    const long pix = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long wh = (long)a.W * a.H;
    if (pix >= wh) return;
    const int yM = (int)(pix / a.W), xM = (int)(pix - (long)yM * a.W);
    const int r0 = -(int)pp.radius, r1 = (int)(pp.radius + 1);
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    float prev = a.st.prev[pix];
    for (int f = 0; f < a.F; ++f) {
        const float* fr = a.interp + (long)f * wh;
        const float* gxf = a.gx + (long)f * wh;
        const float* gyf = a.gy + (long)f * wh;
        const float sx = a.shift[f], sy = a.shift[a.F + f];
        const float xc = (float)((double)xM + 0.5 + (double)sx);
        const float yc = (float)((double)yM + 0.5 + (double)sy);
        const int bx = (int)((double)xc - 0.5), by = (int)((double)yc - 0.5);
        float cglh = 0.f, wsum = 0.f;
        for (int j = r0; j <= r1; ++j) {
            const float vy = (float)((double)((float)by + (float)j) + 0.5);
            if (!(vy > 0 && vy < (float)a.H)) continue;
            for (int i = r0; i <= r1; ++i) {
                const float vx = (float)((double)((float)bx + (float)i) + 0.5);
                if (!(vx > 0 && vx < (float)a.W)) continue;
                const float dx = vx - xc, dy = vy - yc;
                const float d = sqrtf(dx * dx + dy * dy);
                if (!(d != 0.f && d <= pp.tSO)) continue;
                const int gxx = min(max((int)((double)vx - 0.5 + 1), 0), a.W - 1);
                const int gxy = min(max((int)((double)vy - 0.5), 0), a.H - 1);
                const int gyx = min(max((int)((double)vx - 0.5), 0), a.W - 1);
                const int gyy = min(max((int)((double)vy - 0.5 + 1), 0), a.H - 1);
                const float Gx = __ldg(gxf + (long)gxy * a.W + gxx);
                const float Gy = __ldg(gyf + (long)gyy * a.W + gyx);
                float w = d * expf(-(d * d) / pp.tSS);
                w = w * w * w * w;
                wsum += w;
                if (Gx * dx + Gy * dy < 0) {
                    const float gm = sqrtf(Gx * Gx + Gy * Gy);
                    float dk = fabsf(Gy * dx - Gx * dy) / gm;
                    if (isnan(dk)) dk = d;
                    dk = 1 - dk / d;
                    cglh += dk * w;
                }
            }
        }
        const float cg = cglh_power(cglh / wsum, pp.sens);
        float v;
        if (sx == 0.f && sy == 0.f)
            v = __ldg(fr + pix);
        else
            v = sample2d(fr, a.W, a.H, (float)xM + sx, (float)yM + sy);
        const float x = a.int_weighting ? v * cg : cg;
        s0 += x;
        s1 += (double)x * x;
        if (a.t0 + f > 0) s2 += (double)x * prev;
        s3 += v;
        prev = x;
    }
    a.st.acc[pix] += s0;
    a.st.acc[wh + pix] += s1;
    a.st.acc[2 * wh + pix] += s2;
    a.st.acc[3 * wh + pix] += s3;
    a.st.prev[pix] = prev;
}

// Per-pixel sum of tap weights over in-image taps, in the reference's (j outer, i inner)
// float order, so interior and border pixels normalise exactly as liveSRRF_noInterpolation.cl.
__global__ void wsum_kernel(const float* __restrict__ wtab, int r0, int S, int W, int H,
                            float* __restrict__ wsum) {
    const long pix = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= (long)W * H) return;
    const int yM = (int)(pix / W), xM = (int)(pix - (long)yM * W);
    float s = 0.f;
    for (int jj = 0; jj < S; ++jj) {
        const int Y = yM + r0 + jj;
        if (Y < 0 || Y >= H) continue;
        for (int ii = 0; ii < S; ++ii) {
            const int X = xM + r0 + ii;
            if (X < 0 || X >= W) continue;
            const float w = wtab[jj * S + ii];
            if (w != 0.f) s += w;
        }
    }
    wsum[pix] = s;
}

}  // namespace

// Multiprocessor count of a device, queried once per device.
int sm_count(int dev) {
    static int cache[64] = {0};
    if (dev < 0 || dev >= 64) return 148;
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
            cudaGetLastError();
            n = 148;
        }
        cache[dev] = n;
    }
    return cache[dev];
}

namespace {

__global__ void finalize_kernel(BlockState st, int n, int tac_div2, float* __restrict__ out) {
    const long pix = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long P = st.pixels;
    if (pix >= P) return;
    const double avg = st.acc[pix] / n;
    const double av2 = avg * avg;
    double tac = 0.0;
    if (n > 1) {
        tac = st.acc[2 * P + pix] / (n - 1);
        if (tac_div2) tac /= (n - 1);
    }
    float o[4] = {(float)avg, (float)(st.acc[P + pix] / n - av2), (float)(tac - av2),
                  (float)(st.acc[3 * P + pix] / n)};
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k * P + pix] = isnan(o[k]) ? 0.f : o[k];
}

}  // namespace

cudaError_t fht_robx(const float* interp, int W, int H, int F, float* gx, float* gy,
                     cudaStream_t stream) {
    dim3 grid((W + 127) / 128, H, F);
    robx_kernel<<<grid, 128, 0, stream>>>(interp, W, H, (long)W * H, gx, gy);
    return cudaGetLastError();
}

cudaError_t fht_rgc_plain(const FhtGeometry& g, const FhtRgcArgs& a, cudaStream_t stream) {
    PlainParams pp{g.tSS, g.tSO, g.radius, g.sensitivity};
    const long wh = (long)a.W * a.H;
    fht_rgc_plain_kernel<<<(unsigned)((wh + 255) / 256), 256, 0, stream>>>(a, pp);
    return cudaGetLastError();
}

cudaError_t fht_fused_tables(const FhtGeometry& g, int W, int H, FhtFusedTables& t,
                             cudaStream_t stream) {
    cudaError_t e;
    const int S = g.S;
    std::vector<int> jr(2 * S);
    for (int ii = 0; ii < S; ++ii) {
        jr[2 * ii] = g.jlo[ii];
        jr[2 * ii + 1] = g.jhi[ii];
    }
    if ((e = cudaMalloc(&t.wtab, sizeof(float) * S * S)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&t.wdtab, sizeof(float) * S * S)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&t.jrange, sizeof(int) * 2 * S)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&t.wsum, sizeof(float) * (size_t)W * H)) != cudaSuccess) return e;
    cudaMemcpyAsync(t.wtab, g.w.data(), sizeof(float) * S * S, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(t.wdtab, g.wd.data(), sizeof(float) * S * S, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(t.jrange, jr.data(), sizeof(int) * 2 * S, cudaMemcpyHostToDevice, stream);
    const long wh = (long)W * H;
    wsum_kernel<<<(unsigned)((wh + 255) / 256), 256, 0, stream>>>(t.wtab, g.r0, S, W, H, t.wsum);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(stream);  // host tables above are stack temporaries
}

void fht_fused_tables_free(FhtFusedTables& t) {
    cudaFree(t.wtab);
    cudaFree(t.wdtab);
    cudaFree(t.jrange);
    cudaFree(t.wsum);
    t = FhtFusedTables();
}

cudaError_t fht_rgc_fused(const FhtGeometry& g, const FhtFusedTables& t, const FhtRgcArgs& a,
                          cudaStream_t stream) {
    const fused::FusedParams fp{g.r0, g.sensitivity, t.wtab, t.wdtab, t.jrange, t.wsum};
    return fused::launch_fused_in<false, 4, 32>(g.S, g.r0, g.sensitivity, fp, fused::DriftParams{}, a, stream);
}

// Sum of a tap table over the in-image taps of every pixel (the wsum_kernel above, exported).
cudaError_t tap_table_sum(const float* tab, int r0, int S, int W, int H, float* out,
                          cudaStream_t stream) {
    const long wh = (long)W * H;
    wsum_kernel<<<(unsigned)((wh + 255) / 256), 256, 0, stream>>>(tab, r0, S, W, H, out);
    return cudaGetLastError();
}

bool fht_fused_supported(const FhtGeometry& g) {
    return g.S >= 4 && g.S <= 32 && g.S % 2 == 0 && g.r0 == -(g.S - 2) / 2;
}

cudaError_t finalize_block(const BlockState& st, int n, int tac_div2, float* out,
                           cudaStream_t stream) {
    finalize_kernel<<<(unsigned)((st.pixels + 255) / 256), 256, 0, stream>>>(st, n, tac_div2, out);
    return cudaGetLastError();
}

cudaError_t zero_block(BlockState& st, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(st.acc, 0, sizeof(double) * 4 * st.pixels, stream);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(st.prev, 0, sizeof(float) * st.pixels, stream);
}

}  // namespace esrrf

namespace esrrf {

// Same tables as fht_fused_tables, laid out in caller-provided device memory from `base` (each
// piece 256-byte aligned).  With base == nullptr only the byte count is computed.
cudaError_t fht_fused_tables_place(const FhtGeometry& g, int W, int H, FhtFusedTables& t,
                                   unsigned char* base, size_t* bytes, cudaStream_t stream) {
    const int S = g.S;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    size_t off = 0;
    const size_t o_w = off;  off += al(sizeof(float) * S * S);
    const size_t o_wd = off; off += al(sizeof(float) * S * S);
    const size_t o_jr = off; off += al(sizeof(int) * 2 * S);
    const size_t o_ws = off; off += al(sizeof(float) * (size_t)W * H);
    *bytes = off;
    if (!base) return cudaSuccess;
    t.wtab = (float*)(base + o_w);
    t.wdtab = (float*)(base + o_wd);
    t.jrange = (int*)(base + o_jr);
    t.wsum = (float*)(base + o_ws);
    std::vector<int> jr(2 * S);
    for (int ii = 0; ii < S; ++ii) {
        jr[2 * ii] = g.jlo[ii];
        jr[2 * ii + 1] = g.jhi[ii];
    }
    cudaError_t e;
    if ((e = cudaMemcpyAsync(t.wtab, g.w.data(), sizeof(float) * S * S, cudaMemcpyHostToDevice, stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(t.wdtab, g.wd.data(), sizeof(float) * S * S, cudaMemcpyHostToDevice, stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(t.jrange, jr.data(), sizeof(int) * 2 * S, cudaMemcpyHostToDevice, stream)) != cudaSuccess) return e;
    const long wh = (long)W * H;
    wsum_kernel<<<(unsigned)((wh + 255) / 256), 256, 0, stream>>>(t.wtab, g.r0, S, W, H, t.wsum);
    return cudaGetLastError();
}

}  // namespace esrrf
