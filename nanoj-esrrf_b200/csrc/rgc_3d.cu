// rgc_3d.cu -- the 3-D path for multi-focus (MFM) data: LiveSRRF_CL with a calibration table
// (LiveSRRF_CL.java:159-264; FHT interpolation is forced off in 3-D, :166-168) runs
// live3DSRRF.cl.
//
// Per frame: split the camera frame into its planes and normalise them (reshapeImageStack3D,
// LiveSRRF_CL.java:963-994, done on the host by the reference), rotate and shift each plane
// (kernelAlignPixels, live3DSRRF.cl:204-224), 3-D 2-point gradient (:229-279), lateral 2x
// resampling of the three components (:282-320), then 3-D RGC with xy taps on the 2x grid and z
// taps on whole planes, cubic-in-z intensity of four bicubic samples (:325-498).
#include <math.h>

#include "device_common.cuh"
#include "esrrf_internal.h"

namespace esrrf {

BicGeometry bic_geometry(float fwhm, int sensitivity) {
    // Java float arithmetic of prepareBuffersBICinterpolation (LiveSRRF_CL.java:301-321).
    BicGeometry g;
    const int gradientMag = 2;
    g.sigma = fwhm / 2.354f;
    g.radius = ((float)((int)(gradientMag * 2 * g.sigma))) / gradientMag + 1;
    g.tSS = 2 * g.sigma * g.sigma;
    g.tSO = 2 * g.sigma + 1;
    g.sensitivity = (float)sensitivity;
    return g;
}

namespace {

using dev::cglh_power;
using dev::load_px;
using dev::sample2d;

__global__ void mfm_split_kernel(const void* raw, int is_u16, int W, int H, int P, int ws, int hs,
                                 const int* __restrict__ tx0, const int* __restrict__ ty0,
                                 const float* __restrict__ coeff, float background,
                                 float* __restrict__ planes) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z % P;
    const long f = blockIdx.z / P;
    if (x >= ws) return;
    const float p = load_px(raw, is_u16, f * (long)W * H + (long)(ty0[z] + y) * W + tx0[z] + x);
    planes[((f * P + z) * hs + y) * (long)ws + x] = (p - background) / coeff[z];
}

__global__ void align_kernel(const float* __restrict__ planes, int ws, int hs, int P,
                             const float* __restrict__ ct, const float* __restrict__ st,
                             const float* __restrict__ shx, const float* __restrict__ shy,
                             float* __restrict__ apx) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z % P;
    const long fz = blockIdx.z;
    if (x >= ws) return;
    const float cx = (float)(ws - 1) / 2.0f, cy = (float)(hs - 1) / 2.0f;
    const float xa = ((float)x - cx) * ct[z] - ((float)y - cy) * st[z] + cx - shx[z];
    const float ya = ((float)x - cx) * st[z] + ((float)y - cy) * ct[z] + cy - shy[z];
    apx[fz * (long)ws * hs + (long)y * ws + x] = sample2d(planes + fz * (long)ws * hs, ws, hs, xa, ya);
}

__global__ void grad3d_kernel(const float* __restrict__ apx, int ws, int hs, int P,
                              float* __restrict__ gx, float* __restrict__ gy, float* __restrict__ gz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z % P;
    const long f = blockIdx.z / P;
    if (x >= ws) return;
    const long plane = (long)ws * hs;
    const long base = f * P * plane;
    const int x0 = max(x - 1, 0), y0 = max(y - 1, 0), z0 = max(z - 1, 0);
    const long o = base + z * plane + (long)y * ws + x;
    const float p = apx[o];
    gx[o] = p - apx[base + z * plane + (long)y * ws + x0];
    gy[o] = p - apx[base + z * plane + (long)y0 * ws + x];
    gz[o] = p - apx[base + z0 * plane + (long)y * ws + x];
}

__global__ void __launch_bounds__(256) rgc_3d_kernel(Rgc3dArgs a) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int WM = a.w * a.M, HM = a.h * a.M, PM = a.P * a.M;
    const long whM = (long)WM * HM;
    const long total = whM * PM;
    if (idx >= total) return;
    const int zM = (int)(idx / whM);
    const int yM = (int)((idx - (long)zM * whM) / WM);
    const int xM = (int)(idx - (long)zM * whM - (long)yM * WM);
    const int w2 = 2 * a.w, h2 = 2 * a.h;
    const long pl2 = (long)w2 * h2, pl = (long)a.w * a.h;
    const int r0 = -(int)(2.0f * a.radius), r1 = (int)(2.0f * a.radius + 1);
    const int k0 = -(int)a.radius, k1 = (int)a.radius + 1;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    float prev = a.st.prev[idx];
    for (int f = 0; f < a.F; ++f) {
        const float* gxi = a.gxi + (long)f * a.P * pl2;
        const float* gyi = a.gyi + (long)f * a.P * pl2;
        const float* gzi = a.gzi + (long)f * a.P * pl2;
        const float* ap = a.apx + (long)f * a.P * pl;
        const float sx = a.shift[f], sy = a.shift[a.F + f];
        const float xc = (float)(((double)xM + 0.5) / a.M + (double)sx);
        const float yc = (float)(((double)yM + 0.5) / a.M + (double)sy);
        const float zc = (float)(((double)zM + 0.5) / a.M);
        const int kx = (int)(2.0f * xc), ky = (int)(2.0f * yc);
        float cglh = 0.f, wsum = 0.f;
        for (int j = r0; j <= r1; ++j) {
            const float vy = ((float)ky + (float)j) / 2.0f;
            if (!(vy > 0 && vy < (float)a.h)) continue;
            for (int i = r0; i <= r1; ++i) {
                const float vx = ((float)kx + (float)i) / 2.0f;
                if (!(vx > 0 && vx < (float)a.w)) continue;
                const int ax = min(max((int)(2 * ((double)vx - 0.5)), 0), w2 - 1);
                const int ay = min(max((int)(2 * ((double)vy - 0.5)), 0), h2 - 1);
                const int ax1 = min(max((int)(2 * ((double)vx - 0.5) + 1), 0), w2 - 1);
                const int ay1 = min(max((int)(2 * ((double)vy - 0.5) + 1), 0), h2 - 1);
                for (int k = k0; k <= k1; ++k) {
                    const float vz = (float)((int)zc) + (float)k;
                    if (!(vz > 0 && vz < (float)a.P)) continue;
                    const float dx = vx - xc, dy = vy - yc, dz = vz - zc;
                    const float d = sqrtf(dx * dx + dy * dy + dz * dz);
                    if (!(d != 0.f && d <= a.tSO)) continue;
                    const long az = (long)min(max((int)vz, 0), a.P - 1) * pl2;
                    const float Gx = __ldg(gxi + az + (long)ay * w2 + ax1);
                    const float Gy = __ldg(gyi + az + (long)ay1 * w2 + ax);
                    const float Gz = __ldg(gzi + az + (long)ay * w2 + ax);
                    float wt = d * expf(-(d * d) / a.tSS);
                    wt = wt * wt * wt * wt;
                    wsum += wt;
                    if (Gx * dx + Gy * dy + Gz * dz < 0) {
                        const float gm = sqrtf(Gx * Gx + Gy * Gy + Gz * Gz);
                        const float c1 = dy * Gz - dz * Gy, c2 = dz * Gx - dx * Gz, c3 = dx * Gy - dy * Gx;
                        float dk = sqrtf(c1 * c1 + c2 * c2 + c3 * c3) / gm;
                        if (isnan(dk)) dk = d;
                        dk = 1 - dk / d;
                        cglh += dk * wt;
                    }
                }
            }
        }
        const float cg = cglh_power(cglh / wsum, a.sens);
        // cubic z interpolation of four bicubic samples; the fourth plane repeats z0+1
        // (live3DSRRF.cl:434-456)
        int z0;
        const float zcof = zc - 0.5f;
        if (zcof < 0)
            z0 = 0;
        else if (zcof >= (float)(a.P - 1))
            z0 = a.P - 2;
        else
            z0 = (int)floorf(zcof);
        const float px = (float)xM / (float)a.M + sx - 0.5f;
        const float py = (float)yM / (float)a.M + sy - 0.5f;
        const float v_1 = sample2d(ap + (long)max(z0 - 1, 0) * pl, a.w, a.h, px, py);
        const float v0 = sample2d(ap + (long)z0 * pl, a.w, a.h, px, py);
        const float v1 = sample2d(ap + (long)(z0 + 1) * pl, a.w, a.h, px, py);
        const float v2 = sample2d(ap + (long)min(z0 + 1, a.P - 1) * pl, a.w, a.h, px, py);
        const float z01 = zc - (float)(z0 + 0.5f);
        const float ca = -0.5f * v_1 + 1.5f * v0 - 1.5f * v1 + 0.5f * v2;
        const float cb = v_1 - 2.5f * v0 + 2.0f * v1 - 0.5f * v2;
        const float cc = -0.5f * v_1 + 0.5f * v1;
        const float v = ca * z01 * z01 * z01 + cb * z01 * z01 + cc * z01 + v0;
        const float x = a.int_weighting ? v * cg : cg;
        s0 += x;
        s1 += (double)x * x;
        if (a.t0 + f > 0) s2 += (double)x * prev;
        s3 += v;
        prev = x;
    }
    a.st.acc[idx] += s0;
    a.st.acc[total + idx] += s1;
    a.st.acc[2 * total + idx] += s2;
    a.st.acc[3 * total + idx] += s3;
    a.st.prev[idx] = prev;
}

}  // namespace

cudaError_t mfm_prepare(const void* raw, int is_u16, int W, int H, int P, int ws, int hs, int F,
                        const Mfm3dTables& t, float background, float* planes, float* apx,
                        float* gx, float* gy, float* gz, float* gxi, float* gyi, float* gzi,
                        cudaStream_t stream) {
    const dim3 grid((ws + 127) / 128, hs, F * P);
    mfm_split_kernel<<<grid, 128, 0, stream>>>(raw, is_u16, W, H, P, ws, hs, t.tile_x0, t.tile_y0,
                                               t.coeff, background, planes);
    align_kernel<<<grid, 128, 0, stream>>>(planes, ws, hs, P, t.cos_t, t.sin_t, t.shx, t.shy, apx);
    grad3d_kernel<<<grid, 128, 0, stream>>>(apx, ws, hs, P, gx, gy, gz);
    cudaError_t e;
    if ((e = grad2x(gx, ws, hs, F * P, gxi, stream)) != cudaSuccess) return e;
    if ((e = grad2x(gy, ws, hs, F * P, gyi, stream)) != cudaSuccess) return e;
    if ((e = grad2x(gz, ws, hs, F * P, gzi, stream)) != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t rgc_3d(const Rgc3dArgs& a, cudaStream_t stream) {
    const long total = (long)a.w * a.M * a.h * a.M * a.P * a.M;
    rgc_3d_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace esrrf
