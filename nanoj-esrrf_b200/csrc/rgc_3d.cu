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

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>

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

// The z-phase ranges [a, b] of z-blocked entries (M z-phases; an entry is a tap of a contiguous
// range of z-phases, dz being monotonic in the z-phase): class 0 is the full range [0, M - 1],
// then the others in (a, b) order.  upper: b, else a.
__host__ __device__ constexpr int z3d_class_range(int M, int c, bool upper) {
    if (c == 0) return upper ? M - 1 : 0;
    int k = 1;
    for (int a = 0; a < M; ++a)
        for (int b = a; b < M; ++b) {
            if (a == 0 && b == M - 1) continue;
            if (k == c) return upper ? b : a;
            ++k;
        }
    return -1;
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

// Unit gradient of each 2x-grid source point: the reference reads Gx at (x+1, y), Gy at (x, y+1)
// and Gz at (x, y) of the 2x-resampled components (live3DSRRF.cl RGC; for an in-bounds tap the
// clamps never bind), so the tap test and |d x G| / |G| = |d x g| only need g = G / |G|.
// The field is written into the interior of a zero halo, columns split by parity so that a warp's
// 32 consecutive voxels read 32 consecutive entries.  Every point no tap may read (outside the
// volume, the last 2x-grid column and row, plane 0, which the reference never takes a tap from
// since it requires vz > 0) holds a zero gradient: never inward, so out-of-range taps add
// nothing, as the reference skips them.
__global__ void unit_grad3d_kernel(const float* __restrict__ gxi, const float* __restrict__ gyi,
                                   const float* __restrict__ gzi, int w, int h, int P, int padx,
                                   int pady, int padz_lo, int W2p, int H2p, int Pp,
                                   float4* __restrict__ U) {
    const int ax = blockIdx.x * blockDim.x + threadIdx.x;
    const int ay = blockIdx.y;
    const int f = blockIdx.z / P, az = blockIdx.z % P;
    const int w2 = 2 * w, h2 = 2 * h;
    if (ax >= w2) return;
    float4 u = make_float4(0.f, 0.f, 0.f, 0.f);
    if (az > 0 && ax < w2 - 1 && ay < h2 - 1) {
        const long pl = (long)blockIdx.z * w2 * h2;
        const float Gx = __ldg(gxi + pl + (long)ay * w2 + ax + 1);
        const float Gy = __ldg(gyi + pl + (long)(ay + 1) * w2 + ax);
        const float Gz = __ldg(gzi + pl + (long)ay * w2 + ax);
        const float n2 = Gx * Gx + Gy * Gy + Gz * Gz;
        if (n2 > 0.f) {
            const float inv = rsqrtf(n2);
            u = make_float4(Gx * inv, Gy * inv, Gz * inv, 0.f);
        }
    }
    const int xp = ax + padx;  // padx is even: same parity as ax
    U[((long)(f * Pp + az + padz_lo) * H2p + ay + pady) * W2p + (xp & 1) * (W2p / 2) + (xp >> 1)] = u;
}

__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Dk w = w - (w / d) |d x g| for an inward tap, |d x g| from the cross product itself
// (d^2 - (d.g)^2 would cancel for taps along the gradient, which carry the largest terms).
__device__ __forceinline__ float tap_term(const float4& A, const float4& B, const float4& u) {
    const float cx = fmaf(A.z, u.z, -A.w * u.y);  // dy gz - dz gy
    const float cy = fmaf(A.w, u.x, -A.y * u.z);  // dz gx - dx gz
    const float cz = fmaf(A.y, u.y, -A.z * u.x);  // dx gy - dy gx
    return fmaf(-B.z, sqrt_approx(fmaf(cx, cx, fmaf(cy, cy, cz * cz))), B.y);
}

__device__ __forceinline__ void unpack_offsets(float bits, int& sx, int& sy, int& sz) {
    const int pk = __float_as_int(bits);
    sx = (int)((unsigned)pk << 22) >> 22;
    sy = (int)((unsigned)pk << 12) >> 22;
    sz = pk >> 20;
}

// Sum of weights over each output voxel's in-range taps (the reference's Σw, in its tap order),
// once per handle: it depends on the voxel's phase and on how close it is to the volume's faces.
__global__ void wsum3d_kernel(Rgc3dTables t, int w, int h, int P, int M, float* __restrict__ out) {
    const int WM = w * M, HM = h * M;
    const long total = (long)WM * HM * P * M;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int zM = (int)(idx / ((long)WM * HM));
    const int yM = (int)((idx / WM) % HM), xM = (int)(idx % WM);
    const int qx = xM / M, qy = yM / M, qz = zM / M;
    const int phase = ((zM % M) * M + yM % M) * M + xM % M;
    float ws = 0.f;
    for (int k = t.start[phase]; k < t.start[phase + 1]; ++k) {
        const float4 B = t.tabb[k];
        int sx, sy, sz;
        unpack_offsets(B.w, sx, sy, sz);
        const int ax = 2 * qx + sx, ay = 2 * qy + sy, az = qz + sz;
        if (ax < 0 || ax > 2 * w - 2 || ay < 0 || ay > 2 * h - 2 || az < 1 || az > P - 1) continue;
        ws += B.y;
    }
    out[idx] = ws;
}

// One thread per output voxel; a CTA is 32 x 8 input cells of one (x, y) phase and one output
// plane, so the whole CTA walks the same tap list (broadcast from shared memory) and a warp's
// gradient reads are contiguous.  The zero halo makes every tap readable, so there are no bounds
// tests; Σw comes from the per-voxel table.
__global__ void __launch_bounds__(256) rgc3d_tab_kernel(Rgc3dTabArgs a) {
    extern __shared__ float4 stab[];  // [2 n]: A entries, then B entries
    const int M = a.M, M2 = M * M;
    const int zM = blockIdx.z / M2, pxy = blockIdx.z % M2;
    const int px = pxy % M, py = pxy / M;
    const int qz = zM / M, pz = zM % M;
    const int phase = (pz * M + py) * M + px;
    const int t0 = a.tab.start[phase], n = a.tab.start[phase + 1] - t0;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int i = tid; i < n; i += 256) {
        stab[i] = a.tab.taba[t0 + i];
        stab[n + i] = a.tab.tabb[t0 + i];
    }
    __syncthreads();
    const int qx_raw = blockIdx.x * 32 + threadIdx.x, qy_raw = blockIdx.y * 8 + threadIdx.y;
    const bool valid = qx_raw < a.w && qy_raw < a.h;
    const int qx = min(qx_raw, a.w - 1), qy = min(qy_raw, a.h - 1);
    const int xM = qx * M + px, yM = qy * M + py;
    const int WM = a.w * M, HM = a.h * M;
    const long whM = (long)WM * HM, total = whM * a.P * M;
    const long idx = (long)zM * whM + (long)yM * WM + xM;
    const long pl = (long)a.w * a.h;
    const float wsum = a.tab.wsum[idx];
    const long fstride = (long)a.tab.Pp * a.tab.H2p * a.tab.W2p;
    const float4* U0 = a.U + ((long)(qz + a.tab.padz_lo) * a.tab.H2p + 2 * qy + a.tab.pady) * a.tab.W2p +
                       a.tab.padx / 2 + qx;
    // intensity: cubic in z of four bicubic samples, the fourth plane repeating z0 + 1
    // (live3DSRRF.cl:434-456), no shift
    const float zc = (float)(((double)zM + 0.5) / M);
    int z0;
    const float zcof = zc - 0.5f;
    if (zcof < 0)
        z0 = 0;
    else if (zcof >= (float)(a.P - 1))
        z0 = a.P - 2;
    else
        z0 = (int)floorf(zcof);
    const float pxf = (float)xM / (float)M - 0.5f;
    const float pyf = (float)yM / (float)M - 0.5f;
    const float z01 = zc - (float)(z0 + 0.5f);

    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    float prev = valid ? a.st.prev[idx] : 0.f;
    for (int f = 0; f < a.F; ++f) {
        const float4* U = U0 + f * fstride;
        float cglh = 0.f;
#pragma unroll 2
        for (int t = 0; t < n; ++t) {
            const float4 A = stab[t];
            const float4 u = __ldg(U + __float_as_int(A.x));
            const float dot = fmaf(u.x, A.y, fmaf(u.y, A.z, u.z * A.w));
            if (dot < 0.f) cglh += tap_term(A, stab[n + t], u);
        }
        const float cg = cglh_power(cglh / wsum, a.sens);
        const float* ap = a.apx + (long)f * a.P * pl;
        const float v_1 = sample2d(ap + (long)max(z0 - 1, 0) * pl, a.w, a.h, pxf, pyf);
        const float v0 = sample2d(ap + (long)z0 * pl, a.w, a.h, pxf, pyf);
        const float v1 = sample2d(ap + (long)(z0 + 1) * pl, a.w, a.h, pxf, pyf);
        const float v2 = sample2d(ap + (long)min(z0 + 1, a.P - 1) * pl, a.w, a.h, pxf, pyf);
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
    if (!valid) return;
    a.st.acc[idx] += s0;
    a.st.acc[total + idx] += s1;
    a.st.acc[2 * total + idx] += s2;
    a.st.acc[3 * total + idx] += s3;
    a.st.prev[idx] = prev;
}

// The M voxels of one input cell and lateral phase that differ only in their z-phase read the
// same gradient sources (the source offsets do not depend on the z-phase), so one thread computes
// all of them: one gradient load per tap, the dz-free products shared, a (dz, w, w/d) triple per
// z-phase.  Otherwise as rgc3d_tab_kernel.
template <int MZ>
__global__ void __launch_bounds__(256, 2) rgc3d_zb_kernel(Rgc3dTabArgs a) {
    extern __shared__ float4 sz4[];  // [n][es] entries
    constexpr int M = MZ, M2 = MZ * MZ;
    const int es = a.tab.zes;
    const int qz = blockIdx.z / M2, lp = blockIdx.z % M2;
    const int px = lp % M, py = lp / M;
    const int t0 = a.tab.zstart[lp], n = a.tab.zstart[lp + 1] - t0;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int i = tid; i < n * es; i += 256) sz4[i] = a.tab.ztab[(long)t0 * es + i];
    __syncthreads();
    const float* sf = reinterpret_cast<const float*>(sz4);
    const int qx_raw = blockIdx.x * 32 + threadIdx.x, qy_raw = blockIdx.y * 8 + threadIdx.y;
    const bool valid = qx_raw < a.w && qy_raw < a.h;
    const int qx = min(qx_raw, a.w - 1), qy = min(qy_raw, a.h - 1);
    const int xM = qx * M + px, yM = qy * M + py;
    const int WM = a.w * M, HM = a.h * M;
    const long whM = (long)WM * HM, total = whM * a.P * M;
    const long pl = (long)a.w * a.h;
    const long fstride = (long)a.tab.Pp * a.tab.H2p * a.tab.W2p;
    const float4* U0 = a.U + ((long)(qz + a.tab.padz_lo) * a.tab.H2p + 2 * qy + a.tab.pady) * a.tab.W2p +
                       a.tab.padx / 2 + qx;
    const float pxf = (float)xM / (float)M - 0.5f;
    const float pyf = (float)yM / (float)M - 0.5f;
    long idx[MZ];
    float wsum[MZ], prev[MZ], z01[MZ];
    int z0[MZ];
    double s0[MZ], s1[MZ], s2[MZ], s3[MZ];
#pragma unroll
    for (int p = 0; p < MZ; ++p) {
        const int zM = qz * M + p;
        idx[p] = (long)zM * whM + (long)yM * WM + xM;
        wsum[p] = a.tab.wsum[idx[p]];
        prev[p] = valid ? a.st.prev[idx[p]] : 0.f;
        // intensity: cubic in z of four bicubic samples, the fourth plane repeating z0 + 1
        // (live3DSRRF.cl:434-456), no shift
        const float zc = (float)(((double)zM + 0.5) / M);
        const float zcof = zc - 0.5f;
        z0[p] = zcof < 0 ? 0 : (zcof >= (float)(a.P - 1) ? a.P - 2 : (int)floorf(zcof));
        z01[p] = zc - (float)(z0[p] + 0.5f);
        s0[p] = s1[p] = s2[p] = s3[p] = 0.0;
    }
    // the z-phases' base planes z0 take at most two consecutive values, so their z-cubics read
    // the four planes zlo - 1 .. zlo + 2 (clamped): phase p uses S[d], S[d + 1], S[d + 2] twice,
    // d = z0[p] - zlo
    int zlo = z0[0];
#pragma unroll
    for (int p = 1; p < MZ; ++p) zlo = min(zlo, z0[p]);
    int splane[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) splane[k] = min(max(zlo - 1 + k, 0), a.P - 1);
    for (int f = 0; f < a.F; ++f) {
        const float4* U = U0 + f * fstride;
        float cg[MZ];
#pragma unroll
        for (int p = 0; p < MZ; ++p) cg[p] = 0.f;
        for (int t = 0; t < n; ++t) {
            const float* e = sf + (long)t * es * 4;
            const float4 u = __ldg(U + __float_as_int(e[0]));
            const float dx = e[1], dy = e[2];
            const float part = fmaf(u.x, dx, u.y * dy);
            const float cz = fmaf(dx, u.y, -dy * u.x);  // dx gy - dy gx
            const float czz = cz * cz, dyuz = dy * u.z, dxuz = dx * u.z;
#pragma unroll
            for (int p = 0; p < MZ; ++p) {
                const float dz = e[3 + 3 * p], w = e[4 + 3 * p], wd = e[5 + 3 * p];
                const float dot = fmaf(u.z, dz, part);
                if (dot < 0.f) {
                    const float cx = fmaf(-dz, u.y, dyuz);  // dy gz - dz gy
                    const float cy = fmaf(dz, u.x, -dxuz);  // dz gx - dx gz
                    cg[p] += fmaf(-wd, sqrt_approx(fmaf(cx, cx, fmaf(cy, cy, czz))), w);
                }
            }
        }
        const float* ap = a.apx + (long)f * a.P * pl;
        float S[4];
        dev::sample2d_x4(ap, pl, splane, a.w, a.h, pxf, pyf, S);
#pragma unroll
        for (int p = 0; p < MZ; ++p) {
            const float c = cglh_power(cg[p] / wsum[p], a.sens);
            const bool d1 = z0[p] != zlo;
            const float v_1 = d1 ? S[1] : S[0];
            const float v0 = d1 ? S[2] : S[1];
            const float v1 = d1 ? S[3] : S[2];
            const float v2 = v1;
            const float ca = -0.5f * v_1 + 1.5f * v0 - 1.5f * v1 + 0.5f * v2;
            const float cb = v_1 - 2.5f * v0 + 2.0f * v1 - 0.5f * v2;
            const float cc = -0.5f * v_1 + 0.5f * v1;
            const float zz = z01[p];
            const float v = ca * zz * zz * zz + cb * zz * zz + cc * zz + v0;
            const float x = a.int_weighting ? v * c : c;
            s0[p] += x;
            s1[p] += (double)x * x;
            if (a.t0 + f > 0) s2[p] += (double)x * prev[p];
            s3[p] += v;
            prev[p] = x;
        }
    }
    if (!valid) return;
#pragma unroll
    for (int p = 0; p < MZ; ++p) {
        a.st.acc[idx[p]] += s0[p];
        a.st.acc[total + idx[p]] += s1[p];
        a.st.acc[2 * total + idx[p]] += s2[p];
        a.st.acc[3 * total + idx[p]] += s3[p];
        a.st.prev[idx[p]] = prev[p];
    }
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    // 16-byte asynchronous copy; valid = false writes zeros and reads nothing
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}

// rgc3d_zb_kernel with the unit-gradient field staged in shared memory one plane offset at a
// time: the entries of a lateral phase are ordered by sz, and for each (frame, sz) the CTA's slab
// of that plane (its 8 cell rows' 2x-grid rows plus the tap reach, both parity halves of its 32
// cell columns plus the reach) is copied with cp.async into one of two buffers while the taps of
// the previous slab run.  Per-thread arithmetic and tap order within a plane as rgc3d_zb_kernel.
template <int MZ>
__global__ void __launch_bounds__(256, MZ <= 3 ? 3 : 2) rgc3d_zs_kernel(Rgc3dTabArgs a) {
    extern __shared__ float4 sm4[];
    constexpr int M = MZ, M2 = MZ * MZ;
    const int es = a.tab.zes, nz = a.tab.znz;
    // phase fastest: the M^2 CTAs of a cell tile and plane, which stage the same slabs, run together
    const int lp = blockIdx.x, bx = blockIdx.y;
    const int nby = (a.h + 7) / 8;
    const int qz = blockIdx.z / nby, by = blockIdx.z - qz * nby;
    const int px = lp % M, py = lp / M;
    const int t0 = a.tab.zstart[lp], n = a.tab.zstart[lp + 1] - t0;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int row2 = 2 * a.tab.sl_nx;                       // float4s per slab row
    const int slab = a.tab.sl_rows * row2;                  // float4s per slab
    float4* stab = sm4;                                     // [n][es]
    int* sseg = reinterpret_cast<int*>(sm4 + a.tab.zmax_taps * es);  // [nz + 1]
    float4* sbuf = sm4 + a.tab.zmax_taps * es + (nz + 4) / 4;        // [2][slab]
    for (int i = tid; i < n * es; i += 256) {
        float4 v = a.tab.ztab[(long)t0 * es + i];
        if (i % es == 0) v.x = __int_as_float(a.tab.zsoff[t0 + i / es]);  // offset in the slab
        stab[i] = v;
    }
    for (int i = tid; i <= nz; i += 256) sseg[i] = a.tab.zseg[lp * (nz + 1) + i];
    const float* sf = reinterpret_cast<const float*>(stab);
    const int qx_raw = bx * 32 + threadIdx.x, qy_raw = by * 8 + threadIdx.y;
    const bool valid = qx_raw < a.w && qy_raw < a.h;
    const int qx = min(qx_raw, a.w - 1), qy = min(qy_raw, a.h - 1);
    const int xM = qx * M + px, yM = qy * M + py;
    const int WM = a.w * M, HM = a.h * M;
    const long whM = (long)WM * HM, total = whM * a.P * M;
    const long pl = (long)a.w * a.h;
    const long fstride = (long)a.tab.Pp * a.tab.H2p * a.tab.W2p;
    const int half = a.tab.W2p / 2;
    const int row0 = 2 * by * 8 + a.tab.pady + a.tab.sl_symin;
    const int cin0 = a.tab.padx / 2 + bx * 32 + a.tab.sl_fxmin;
    const int tbase = 2 * threadIdx.y * row2 + threadIdx.x;  // this thread's cell in the slab
    const float pxf = (float)xM / (float)M - 0.5f;
    const float pyf = (float)yM / (float)M - 0.5f;
    long idx[MZ];
    float wsum[MZ], prev[MZ], z01[MZ];
    int z0[MZ];
    float s0[MZ], s1[MZ], s2[MZ], s3[MZ];  // this launch's frames (at most a few) in FP32
#pragma unroll
    for (int p = 0; p < MZ; ++p) {
        const int zM = qz * M + p;
        idx[p] = (long)zM * whM + (long)yM * WM + xM;
        wsum[p] = a.tab.wsum[idx[p]];
        prev[p] = valid ? a.st.prev[idx[p]] : 0.f;
        const float zc = (float)(((double)zM + 0.5) / M);
        const float zcof = zc - 0.5f;
        z0[p] = zcof < 0 ? 0 : (zcof >= (float)(a.P - 1) ? a.P - 2 : (int)floorf(zcof));
        z01[p] = zc - (float)(z0[p] + 0.5f);
        s0[p] = s1[p] = s2[p] = s3[p] = 0.f;
    }
    int zlo = z0[0];
#pragma unroll
    for (int p = 1; p < MZ; ++p) zlo = min(zlo, z0[p]);
    int splane[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) splane[k] = min(max(zlo - 1 + k, 0), a.P - 1);

    // slab staging: warp ty copies rows ty, ty + 8, ...; lane tx the positions tx + 32 q of each
    // row, whose source column offsets (parity half + column; -1 beyond the field) are the same
    // for every row, plane and frame (row2 <= 4 x 32, checked before this form is chosen)
    int coff[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int rem = threadIdx.x + 32 * q;
        const int par = rem >= a.tab.sl_nx ? 1 : 0, cin = cin0 + rem - par * a.tab.sl_nx;
        coff[q] = rem < row2 && cin < half ? par * half + cin : -1;
    }
    // slab g = (frame g / nz, plane offset zk0 + g % nz) into buffer g & 1
    auto stage = [&](int g) {
        const int f = g / nz, sidx = g - f * nz;
        const int plane = qz + a.tab.padz_lo + a.tab.zk0 + sidx;
        const float4* Uf = a.U + f * fstride + (long)plane * a.tab.H2p * a.tab.W2p;
        float4* dst = sbuf + (g & 1) * slab;
        for (int ly = threadIdx.y; ly < a.tab.sl_rows; ly += 8) {
            const int row = row0 + ly;
            const bool rin = row < a.tab.H2p;
            const float4* src = Uf + (long)row * a.tab.W2p;
            float4* d = dst + ly * row2 + threadIdx.x;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if ((int)threadIdx.x + 32 * q >= row2) break;
                const bool in = rin && coff[q] >= 0;
                cp_async16(d + 32 * q, in ? (const void*)(src + coff[q]) : (const void*)a.U, in);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    const int G = a.F * nz;
    if (G > 0) stage(0);
    float cg[MZ];
    for (int g = 0; g < G; ++g) {
        const int f = g / nz, sidx = g - f * nz;
        if (sidx == 0) {
#pragma unroll
            for (int p = 0; p < MZ; ++p) cg[p] = 0.f;
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();  // slab g landed everywhere; buffer (g + 1) & 1 is no longer read
        if (g + 1 < G) stage(g + 1);
        const float4* sl = sbuf + (g & 1) * slab + tbase;
        const int tb = sseg[sidx], te = sseg[sidx + 1];
        for (int t = tb; t < te; ++t) {
            const float* e = sf + (long)t * es * 4;
            const float4 u = sl[__float_as_int(e[0])];
            const float dx = e[1], dy = e[2];
            const float part = fmaf(u.x, dx, u.y * dy);
            const float cz = fmaf(dx, u.y, -dy * u.x);  // dx gy - dy gx
            const float czz = cz * cz, dyuz = dy * u.z, dxuz = dx * u.z;
#pragma unroll
            for (int p = 0; p < MZ; ++p) {
                const float dz = e[3 + 3 * p], w = e[4 + 3 * p], wd = e[5 + 3 * p];
                const float dot = fmaf(u.z, dz, part);
                if (dot < 0.f) {
                    const float cx = fmaf(-dz, u.y, dyuz);  // dy gz - dz gy
                    const float cy = fmaf(dz, u.x, -dxuz);  // dz gx - dx gz
                    cg[p] += fmaf(-wd, sqrt_approx(fmaf(cx, cx, fmaf(cy, cy, czz))), w);
                }
            }
        }
        if (sidx != nz - 1) continue;
        const float* ap = a.apx + (long)f * a.P * pl;
        float S[4];
        dev::sample2d_x4(ap, pl, splane, a.w, a.h, pxf, pyf, S);
#pragma unroll
        for (int p = 0; p < MZ; ++p) {
            const float c = cglh_power(cg[p] / wsum[p], a.sens);
            const bool d1 = z0[p] != zlo;
            const float v_1 = d1 ? S[1] : S[0];
            const float v0 = d1 ? S[2] : S[1];
            const float v1 = d1 ? S[3] : S[2];
            const float v2 = v1;
            const float ca = -0.5f * v_1 + 1.5f * v0 - 1.5f * v1 + 0.5f * v2;
            const float cb = v_1 - 2.5f * v0 + 2.0f * v1 - 0.5f * v2;
            const float cc = -0.5f * v_1 + 0.5f * v1;
            const float zz = z01[p];
            const float v = ca * zz * zz * zz + cb * zz * zz + cc * zz + v0;
            const float x = a.int_weighting ? v * c : c;
            s0[p] += x;
            s1[p] = fmaf(x, x, s1[p]);
            if (a.t0 + f > 0) s2[p] = fmaf(x, prev[p], s2[p]);
            s3[p] += v;
            prev[p] = x;
        }
    }
    if (!valid) return;
#pragma unroll
    for (int p = 0; p < MZ; ++p) {
        a.st.acc[idx[p]] += (double)s0[p];
        a.st.acc[total + idx[p]] += (double)s1[p];
        a.st.acc[2 * total + idx[p]] += (double)s2[p];
        a.st.acc[3 * total + idx[p]] += (double)s3[p];
        a.st.prev[idx[p]] = prev[p];
    }
}

// Entries [tb, te) of a slab that are taps of z-phases A .. B only (the other z-phases' weights
// are 0 there, so leaving them out changes no sum), for the two cells of rgc3d_z2_kernel.
template <int MZ, int A, int B>
__device__ __forceinline__ void z2_entries(const float* __restrict__ sf, const float4* __restrict__ sl,
                                           int cell1, int tb, int te, float (&cg)[2][MZ]) {
    // two entries per iteration (their loads and dot products overlap), each entry's table row
    // read as whole float4s (ES float4s per entry, the tables' zes)
    constexpr int ES = (3 + 3 * MZ + 3) / 4;
#pragma unroll 2
    for (int t = tb; t < te; ++t) {
        float e[4 * ES];
#pragma unroll
        for (int q = 0; q < ES; ++q) {
            const float4 v = reinterpret_cast<const float4*>(sf)[(long)t * ES + q];
            e[4 * q] = v.x;
            e[4 * q + 1] = v.y;
            e[4 * q + 2] = v.z;
            e[4 * q + 3] = v.w;
        }
        const int o = __float_as_int(e[0]);
        const float dx = e[1], dy = e[2];
        float4 u[2];
        u[0] = sl[o];
        u[1] = sl[o + cell1];
        float part[2], cz2[2], dyuz[2], dxuz[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            part[c] = fmaf(u[c].x, dx, u[c].y * dy);
            const float cz = fmaf(dx, u[c].y, -dy * u[c].x);  // dx gy - dy gx
            cz2[c] = cz * cz;
            dyuz[c] = dy * u[c].z;
            dxuz[c] = dx * u[c].z;
        }
#pragma unroll
        for (int p = A; p <= B; ++p) {
            const float dz = e[3 + 3 * p], w = e[4 + 3 * p], wd = e[5 + 3 * p];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const float dot = fmaf(u[c].z, dz, part[c]);
                if (dot < 0.f) {
                    const float cx = fmaf(-dz, u[c].y, dyuz[c]);  // dy gz - dz gy
                    const float cy = fmaf(dz, u[c].x, -dxuz[c]);  // dz gx - dx gz
                    cg[c][p] += fmaf(-wd, sqrt_approx(fmaf(cx, cx, fmaf(cy, cy, cz2[c]))), w);
                }
            }
        }
    }
}

// The classes C .. of a slab's entries in turn (cs: the slab's class starts, cs[ncls] its end).
template <int MZ, int C>
__device__ __forceinline__ void z2_classes(const int* __restrict__ cs, const float* __restrict__ sf,
                                           const float4* __restrict__ sl, int cell1, float (&cg)[2][MZ]) {
    if constexpr (C < MZ * (MZ + 1) / 2) {
        z2_entries<MZ, z3d_class_range(MZ, C, false), z3d_class_range(MZ, C, true)>(sf, sl, cell1, cs[C],
                                                                                   cs[C + 1], cg);
        z2_classes<MZ, C + 1>(cs, sf, sl, cell1, cg);
    }
}

// rgc3d_zs_kernel with two cells per thread: thread (tx, ty) of a CTA computes the cells in rows
// ty and ty + 8 of a 32 x 16 cell tile (same lateral phase, so the same entry list).  Each entry's
// table values (offset, dx, dy, and per z-phase dz, w, w/d) are loaded once for both cells, and the
// two cells' dot / cross / square-root chains are independent, which doubles the work each warp
// has in flight per entry.  The per-voxel epilogue state is kept to the FP32 sums and previous
// values (index, sum of weights and z-cubic position are recomputed at the end of a timepoint), so
// that two CTAs of 256 threads run per SM without spilling.  Slab: the tile's 16 cell rows' 2x-grid
// rows plus the tap reach (16 more rows than rgc3d_zs_kernel's), same columns; the entries' slab
// offsets are the same (they depend on the row length only).
template <int MZ>
__global__ void __launch_bounds__(256, 2) rgc3d_z2_kernel(Rgc3dTabArgs a) {
    extern __shared__ float4 sm4[];
    constexpr int M = MZ;
    const int es = a.tab.zes, nz = a.tab.znz;
    const int lp = blockIdx.x, bx = blockIdx.y;
    const int nby = (a.h + 15) / 16;
    const int qz = blockIdx.z / nby, by = blockIdx.z - qz * nby;
    const int px = lp % M, py = lp / M;
    const int t0 = a.tab.zstart[lp], n = a.tab.zstart[lp + 1] - t0;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int row2 = 2 * a.tab.sl_nx;                       // float4s per slab row
    const int rows = a.tab.sl_rows + 16;                    // slab rows of 16 cell rows
    const int slab = rows * row2;                           // float4s per slab
    constexpr int NC = MZ * (MZ + 1) / 2;                   // z-phase range classes
    float4* stab = sm4;                                     // [n][es]
    int* sseg = reinterpret_cast<int*>(sm4 + a.tab.zmax_taps * es);  // [nz NC + 1] class starts
    float4* sbuf = sm4 + a.tab.zmax_taps * es + (nz * NC + 4) / 4;   // [2][slab]
    for (int i = tid; i < n * es; i += 256) {
        float4 v = a.tab.ztab[(long)t0 * es + i];
        if (i % es == 0) v.x = __int_as_float(a.tab.zsoff[t0 + i / es]);  // offset in the slab
        stab[i] = v;
    }
    for (int i = tid; i <= nz * NC; i += 256) sseg[i] = a.tab.zcseg[lp * (nz * NC + 1) + i];
    const float* sf = reinterpret_cast<const float*>(stab);
    const int qx_raw = bx * 32 + threadIdx.x;
    int qy_raw[2];
    qy_raw[0] = by * 16 + threadIdx.y;
    qy_raw[1] = qy_raw[0] + 8;
    const int WM = a.w * M, HM = a.h * M;
    const long whM = (long)WM * HM, total = whM * a.P * M;
    const long pl = (long)a.w * a.h;
    const long fstride = (long)a.tab.Pp * a.tab.H2p * a.tab.W2p;
    const int half = a.tab.W2p / 2;
    const int row0 = 2 * by * 16 + a.tab.pady + a.tab.sl_symin;
    const int cin0 = a.tab.padx / 2 + bx * 32 + a.tab.sl_fxmin;
    const int tbase = 2 * threadIdx.y * row2 + threadIdx.x;  // cell 0 in the slab; cell 1 16 rows down
    const int cell1 = 16 * row2;
    float s0[2][MZ], s1[2][MZ], s2[2][MZ], s3[2][MZ], prev[2][MZ];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const bool valid = qx_raw < a.w && qy_raw[c] < a.h;
        const int yM = min(qy_raw[c], a.h - 1) * M + py, xM = min(qx_raw, a.w - 1) * M + px;
#pragma unroll
        for (int p = 0; p < MZ; ++p) {
            const long idx = (long)(qz * M + p) * whM + (long)yM * WM + xM;
            prev[c][p] = valid ? a.st.prev[idx] : 0.f;
            s0[c][p] = s1[c][p] = s2[c][p] = s3[c][p] = 0.f;
        }
    }
    // the z-cubic's base planes: zlo is the lowest base plane of the cell's z-phases
    int zlo = a.P;
#pragma unroll
    for (int p = 0; p < MZ; ++p) {
        const float zcof = (float)(((double)(qz * M + p) + 0.5) / M) - 0.5f;
        const int z0 = zcof < 0 ? 0 : (zcof >= (float)(a.P - 1) ? a.P - 2 : (int)floorf(zcof));
        zlo = min(zlo, z0);
    }
    int splane[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) splane[k] = min(max(zlo - 1 + k, 0), a.P - 1);

    int coff[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int rem = threadIdx.x + 32 * q;
        const int par = rem >= a.tab.sl_nx ? 1 : 0, cin = cin0 + rem - par * a.tab.sl_nx;
        coff[q] = rem < row2 && cin < half ? par * half + cin : -1;
    }
    auto stage = [&](int g) {
        const int f = g / nz, sidx = g - f * nz;
        const int plane = qz + a.tab.padz_lo + a.tab.zk0 + sidx;
        const float4* Uf = a.U + f * fstride + (long)plane * a.tab.H2p * a.tab.W2p;
        float4* dst = sbuf + (g & 1) * slab;
        for (int ly = threadIdx.y; ly < rows; ly += 8) {
            const int row = row0 + ly;
            const bool rin = row < a.tab.H2p;
            const float4* src = Uf + (long)row * a.tab.W2p;
            float4* d = dst + ly * row2 + threadIdx.x;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if ((int)threadIdx.x + 32 * q >= row2) break;
                const bool in = rin && coff[q] >= 0;
                cp_async16(d + 32 * q, in ? (const void*)(src + coff[q]) : (const void*)a.U, in);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    const int G = a.F * nz;
    if (G > 0) stage(0);
    float cg[2][MZ];
    for (int g = 0; g < G; ++g) {
        const int f = g / nz, sidx = g - f * nz;
        if (sidx == 0) {
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
                for (int p = 0; p < MZ; ++p) cg[c][p] = 0.f;
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();  // slab g landed everywhere; buffer (g + 1) & 1 is no longer read
        if (g + 1 < G) stage(g + 1);
        const float4* sl = sbuf + (g & 1) * slab + tbase;
        z2_classes<MZ, 0>(sseg + sidx * NC, sf, sl, cell1, cg);
        if (sidx != nz - 1) continue;
        const float* ap = a.apx + (long)f * a.P * pl;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int yM = min(qy_raw[c], a.h - 1) * M + py, xM = min(qx_raw, a.w - 1) * M + px;
            float S[4];
            dev::sample2d_x4(ap, pl, splane, a.w, a.h, (float)xM / (float)M - 0.5f,
                             (float)yM / (float)M - 0.5f, S);
#pragma unroll
            for (int p = 0; p < MZ; ++p) {
                const int zM = qz * M + p;
                const long idx = (long)zM * whM + (long)yM * WM + xM;
                const float zc = (float)(((double)zM + 0.5) / M);
                const float zcof = zc - 0.5f;
                const int z0 = zcof < 0 ? 0 : (zcof >= (float)(a.P - 1) ? a.P - 2 : (int)floorf(zcof));
                const float zz = zc - (float)(z0 + 0.5f);
                const float cgv = cglh_power(cg[c][p] / __ldg(a.tab.wsum + idx), a.sens);
                const bool d1 = z0 != zlo;
                const float v_1 = d1 ? S[1] : S[0];
                const float v0 = d1 ? S[2] : S[1];
                const float v1 = d1 ? S[3] : S[2];
                const float v2 = v1;
                const float ca = -0.5f * v_1 + 1.5f * v0 - 1.5f * v1 + 0.5f * v2;
                const float cb = v_1 - 2.5f * v0 + 2.0f * v1 - 0.5f * v2;
                const float cc = -0.5f * v_1 + 0.5f * v1;
                const float v = ca * zz * zz * zz + cb * zz * zz + cc * zz + v0;
                const float x = a.int_weighting ? v * cgv : cgv;
                s0[c][p] += x;
                s1[c][p] = fmaf(x, x, s1[c][p]);
                if (a.t0 + f > 0) s2[c][p] = fmaf(x, prev[c][p], s2[c][p]);
                s3[c][p] += v;
                prev[c][p] = x;
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        if (qx_raw >= a.w || qy_raw[c] >= a.h) continue;
        const int yM = qy_raw[c] * M + py, xM = qx_raw * M + px;
#pragma unroll
        for (int p = 0; p < MZ; ++p) {
            const long idx = (long)(qz * M + p) * whM + (long)yM * WM + xM;
            a.st.acc[idx] += (double)s0[c][p];
            a.st.acc[total + idx] += (double)s1[c][p];
            a.st.acc[2 * total + idx] += (double)s2[c][p];
            a.st.acc[3 * total + idx] += (double)s3[c][p];
            a.st.prev[idx] = prev[c][p];
        }
    }
}

size_t z2_smem_bytes(const Rgc3dTables& t) {
    return sizeof(float4) * ((size_t)t.zmax_taps * t.zes + (t.znz * t.zncls + 4) / 4 +
                             2 * (size_t)(t.sl_rows + 16) * 2 * t.sl_nx);
}

template <int MZ>
cudaError_t launch_z2(const Rgc3dTabArgs& a, cudaStream_t stream) {
    const size_t smem = z2_smem_bytes(a.tab);
    static unsigned long long configured = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && !(configured & (1ull << dev))) {
        if ((e = cudaFuncSetAttribute(rgc3d_z2_kernel<MZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      112 * 1024)) != cudaSuccess ||
            (e = cudaFuncSetAttribute(rgc3d_z2_kernel<MZ>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      cudaSharedmemCarveoutMaxShared)) != cudaSuccess)
            return e;
        configured |= 1ull << dev;
    }
    if (smem > 112 * 1024) return cudaErrorInvalidValue;
    if ((a.w + 31) / 32 > 65535 || (long)((a.h + 15) / 16) * a.P > 65535) return cudaErrorInvalidValue;
    const dim3 grid(MZ * MZ, (a.w + 31) / 32, ((a.h + 15) / 16) * a.P);
    rgc3d_z2_kernel<MZ><<<grid, dim3(32, 8), smem, stream>>>(a);
    return cudaGetLastError();
}

size_t zs_smem_bytes(const Rgc3dTables& t) {
    return sizeof(float4) * ((size_t)t.zmax_taps * t.zes + (t.znz + 4) / 4 + 2 * (size_t)t.sl_rows * 2 * t.sl_nx);
}

template <int MZ>
cudaError_t launch_zs(const Rgc3dTabArgs& a, cudaStream_t stream) {
    const size_t smem = zs_smem_bytes(a.tab);
    static unsigned long long configured = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && !(configured & (1ull << dev))) {
        if ((e = cudaFuncSetAttribute(rgc3d_zs_kernel<MZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      112 * 1024)) != cudaSuccess ||
            (e = cudaFuncSetAttribute(rgc3d_zs_kernel<MZ>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      cudaSharedmemCarveoutMaxShared)) != cudaSuccess)
            return e;
        configured |= 1ull << dev;
    }
    if ((a.w + 31) / 32 > 65535 || (long)((a.h + 7) / 8) * a.P > 65535) return cudaErrorInvalidValue;
    const dim3 grid(MZ * MZ, (a.w + 31) / 32, ((a.h + 7) / 8) * a.P);
    rgc3d_zs_kernel<MZ><<<grid, dim3(32, 8), smem, stream>>>(a);
    return cudaGetLastError();
}

template <int MZ>
cudaError_t launch_zb(const Rgc3dTabArgs& a, cudaStream_t stream) {
    const size_t smem = sizeof(float4) * (size_t)a.tab.zmax_taps * a.tab.zes;
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static unsigned long long configured = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (smem > 48 * 1024 && dev < 64 && !(configured & (1ull << dev))) {
        if ((e = cudaFuncSetAttribute(rgc3d_zb_kernel<MZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      200 * 1024)) != cudaSuccess)
            return e;
        configured |= 1ull << dev;
    }
    const dim3 grid((a.w + 31) / 32, (a.h + 7) / 8, MZ * MZ * a.P);
    rgc3d_zb_kernel<MZ><<<grid, dim3(32, 8), smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t rgc3d_tables_build(const BicGeometry& g, int M, int w, int h, int P, Rgc3dTables& t,
                               cudaStream_t stream) {
    // Tap geometry of rgc_3d_kernel with zero shift, for the voxel of each phase in the first
    // input cell (Java float arithmetic as the reference: xc = (float)((xM + 0.5) / M)).
    const int r0 = -(int)(2.0f * g.radius), r1 = (int)(2.0f * g.radius + 1);
    const int k0 = -(int)g.radius, k1 = (int)g.radius + 1;
    const int M3 = M * M * M;
    struct Tap {
        int sx, sy, sz;
        float dx, dy, dz, d, wt;
    };
    std::vector<Tap> taps;
    std::vector<int> start(M3 + 1, 0);
    int mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
    int maxn = 0;
    for (int pz = 0; pz < M; ++pz)
        for (int py = 0; py < M; ++py)
            for (int px = 0; px < M; ++px) {
                const int phase = (pz * M + py) * M + px;
                start[phase] = (int)taps.size();
                const float xc = (float)(((double)px + 0.5) / M);
                const float yc = (float)(((double)py + 0.5) / M);
                const float zc = (float)(((double)pz + 0.5) / M);
                const int kx = (int)(2.0f * xc), ky = (int)(2.0f * yc);
                for (int j = r0; j <= r1; ++j) {
                    const float vy = ((float)ky + (float)j) / 2.0f;
                    for (int i = r0; i <= r1; ++i) {
                        const float vx = ((float)kx + (float)i) / 2.0f;
                        for (int k = k0; k <= k1; ++k) {
                            const float vz = (float)((int)zc) + (float)k;
                            const float dx = vx - xc, dy = vy - yc, dz = vz - zc;
                            const float d = sqrtf(dx * dx + dy * dy + dz * dz);
                            if (!(d != 0.f && d <= g.tSO)) continue;
                            float wt = d * expf(-(d * d) / g.tSS);
                            wt = wt * wt * wt * wt;
                            const Tap tp{kx + i - 1, ky + j - 1, k, dx, dy, dz, d, wt};
                            const int sv[3] = {tp.sx, tp.sy, tp.sz};
                            for (int c = 0; c < 3; ++c) {
                                mn[c] = std::min(mn[c], sv[c]);
                                mx[c] = std::max(mx[c], sv[c]);
                            }
                            taps.push_back(tp);
                        }
                    }
                }
                maxn = std::max(maxn, (int)taps.size() - start[phase]);
            }
    start[M3] = (int)taps.size();
    // zero halo: 2x-grid column ax = 2 qx + sx in [sx_min, 2w - 2 + sx_max], row likewise, plane
    // qz + sz in [sz_min, P - 1 + sz_max]
    t.padx = std::max(-mn[0], std::max(mx[0] - 1, 0));
    t.padx += t.padx & 1;
    t.pady = std::max(-mn[1], std::max(mx[1] - 1, 0));
    t.padz_lo = std::max(-mn[2], 0);
    t.padz_hi = std::max(mx[2], 0);
    t.W2p = 2 * w + 2 * t.padx;
    t.H2p = 2 * h + 2 * t.pady;
    t.Pp = P + t.padz_lo + t.padz_hi;
    std::vector<float4> A, B;
    A.reserve(taps.size());
    B.reserve(taps.size());
    for (const Tap& tp : taps) {
        // column 2 qx + padx + sx sits at parity (sx & 1), index qx + padx / 2 + floor(sx / 2)
        const int off = tp.sz * t.W2p * t.H2p + tp.sy * t.W2p + (tp.sx & 1) * (t.W2p / 2) + (tp.sx >> 1);
        const int pk = (int)(((unsigned)tp.sx & 0x3FFu) | (((unsigned)tp.sy & 0x3FFu) << 10) |
                             ((unsigned)tp.sz << 20));
        float offf, pkf;
        std::memcpy(&offf, &off, 4);
        std::memcpy(&pkf, &pk, 4);
        A.push_back(make_float4(offf, tp.dx, tp.dy, tp.dz));
        B.push_back(make_float4(tp.d * tp.d, tp.wt, tp.wt / tp.d, pkf));
    }
    t.max_taps = maxn;
    // z-blocked entries: per lateral phase, the (j, i, k) taps valid for at least one z-phase
    std::vector<float4> Z;
    std::vector<int> zstart(M * M + 1, 0);
    std::vector<int> zsx, zsy, zsz, zcls, zsoff, zseg, zcseg;
    if (M <= 5) {
        t.zes = (3 + 3 * M + 3) / 4;
        int zmax = 0;
        for (int py = 0; py < M; ++py)
            for (int px = 0; px < M; ++px) {
                const int lp = py * M + px;
                zstart[lp] = (int)(Z.size() / t.zes);
                const float xc = (float)(((double)px + 0.5) / M);
                const float yc = (float)(((double)py + 0.5) / M);
                const int kx = (int)(2.0f * xc), ky = (int)(2.0f * yc);
                for (int k = k0; k <= k1; ++k) {  // entries ordered by plane offset, then by class
                    struct ZEnt {
                        int cls, sx, sy, sz;
                        std::vector<float> ent;
                    };
                    std::vector<ZEnt> plane;
                    for (int j = r0; j <= r1; ++j) {
                        const float vy = ((float)ky + (float)j) / 2.0f;
                        for (int i = r0; i <= r1; ++i) {
                            const float vx = ((float)kx + (float)i) / 2.0f;
                            std::vector<float> ent(4 * t.zes, 0.f);
                            int pa = M, pb = -1, nin = 0;  // z-phases of which this is a tap
                            const float dx = vx - xc, dy = vy - yc;
                            for (int pz = 0; pz < M; ++pz) {
                                const float zc = (float)(((double)pz + 0.5) / M);
                                const float dz = ((float)((int)zc) + (float)k) - zc;
                                const float d = sqrtf(dx * dx + dy * dy + dz * dz);
                                ent[3 + 3 * pz] = dz;
                                if (!(d != 0.f && d <= g.tSO)) continue;
                                float wt = d * expf(-(d * d) / g.tSS);
                                wt = wt * wt * wt * wt;
                                ent[4 + 3 * pz] = wt;
                                ent[5 + 3 * pz] = wt / d;
                                pa = std::min(pa, pz);
                                pb = std::max(pb, pz);
                                ++nin;
                            }
                            if (nin == 0) continue;
                            // the class of [pa, pb]; a non-contiguous set (none for a sphere)
                            // would take the full range, whose other phases have weight 0
                            int cls = 0;
                            if (nin == pb - pa + 1)
                                for (int c = 0; c < M * (M + 1) / 2; ++c)
                                    if (z3d_class_range(M, c, false) == pa && z3d_class_range(M, c, true) == pb)
                                        cls = c;
                            const int sx = kx + i - 1, sy = ky + j - 1, sz = k;
                            const int off = sz * t.W2p * t.H2p + sy * t.W2p + (sx & 1) * (t.W2p / 2) + (sx >> 1);
                            std::memcpy(&ent[0], &off, 4);
                            ent[1] = dx;
                            ent[2] = dy;
                            plane.push_back(ZEnt{cls, sx, sy, sz, std::move(ent)});
                        }
                    }
                    std::stable_sort(plane.begin(), plane.end(),
                                     [](const ZEnt& x, const ZEnt& y) { return x.cls < y.cls; });
                    for (const ZEnt& z : plane) {
                        for (int q = 0; q < t.zes; ++q)
                            Z.push_back(make_float4(z.ent[4 * q], z.ent[4 * q + 1], z.ent[4 * q + 2], z.ent[4 * q + 3]));
                        zsx.push_back(z.sx);
                        zsy.push_back(z.sy);
                        zsz.push_back(z.sz);
                        zcls.push_back(z.cls);
                    }
                }
                zmax = std::max(zmax, (int)(Z.size() / t.zes) - zstart[lp]);
            }
        zstart[M * M] = (int)(Z.size() / t.zes);
        t.zmax_taps = zmax;
        // slab geometry: rows 2 qy + sy over the CTA's 8 cell rows, per parity columns
        // qx + (sx >> 1) over its 32 cell columns
        int symin = 0, symax = 0, fxmin = 0, fxmax = 0, szmin = k1, szmax = k0;
        for (size_t e = 0; e < zsx.size(); ++e) {
            symin = std::min(symin, zsy[e]);
            symax = std::max(symax, zsy[e]);
            fxmin = std::min(fxmin, zsx[e] >> 1);
            fxmax = std::max(fxmax, zsx[e] >> 1);
            szmin = std::min(szmin, zsz[e]);
            szmax = std::max(szmax, zsz[e]);
        }
        // plane offsets of actual entries only: they lie inside the field's z padding
        t.zk0 = szmin;
        t.znz = std::max(szmax - szmin + 1, 1);
        zseg.assign((size_t)M * M * (t.znz + 1), 0);
        for (int lp = 0; lp < M * M; ++lp) {
            const int e0 = zstart[lp], e1 = zstart[lp + 1];
            for (int sidx = 0; sidx <= t.znz; ++sidx) {
                int e = e0;
                while (e < e1 && zsz[e] - szmin < sidx) ++e;
                zseg[(size_t)lp * (t.znz + 1) + sidx] = e - e0;
            }
        }
        t.zncls = M * (M + 1) / 2;
        const int ncs = t.znz * t.zncls + 1;
        zcseg.assign((size_t)M * M * ncs, 0);
        for (int lp = 0; lp < M * M; ++lp) {
            const int e0 = zstart[lp], e1 = zstart[lp + 1];
            int e = e0;
            for (int sidx = 0; sidx < t.znz; ++sidx)
                for (int c = 0; c < t.zncls; ++c) {
                    zcseg[(size_t)lp * ncs + sidx * t.zncls + c] = e - e0;
                    while (e < e1 && zsz[e] - szmin == sidx && zcls[e] == c) ++e;
                }
            zcseg[(size_t)lp * ncs + t.znz * t.zncls] = e1 - e0;
            if (e != e1) return cudaErrorInvalidValue;  // entries not grouped by plane and class
        }
        t.sl_symin = symin;
        t.sl_fxmin = fxmin;
        t.sl_rows = 2 * 7 + symax - symin + 1;
        t.sl_nx = 31 + fxmax - fxmin + 1;
        zsoff.resize(zsx.size());
        for (size_t e = 0; e < zsx.size(); ++e)
            zsoff[e] = (zsy[e] - symin) * 2 * t.sl_nx + (zsx[e] & 1) * t.sl_nx + ((zsx[e] >> 1) - fxmin);
    }
    auto up = [](auto** d, const auto& v) -> cudaError_t {
        cudaError_t e = cudaMalloc((void**)d, sizeof(v[0]) * std::max<size_t>(v.size(), 1));
        if (e != cudaSuccess || v.empty()) return e;
        return cudaMemcpy(*d, v.data(), sizeof(v[0]) * v.size(), cudaMemcpyHostToDevice);
    };
    cudaError_t e;
    if ((e = up(&t.taba, A)) != cudaSuccess || (e = up(&t.tabb, B)) != cudaSuccess ||
        (e = up(&t.start, start)) != cudaSuccess)
        return e;
    if (M <= 5 && ((e = up(&t.ztab, Z)) != cudaSuccess || (e = up(&t.zstart, zstart)) != cudaSuccess ||
                   (e = up(&t.zseg, zseg)) != cudaSuccess || (e = up(&t.zsoff, zsoff)) != cudaSuccess ||
                   (e = up(&t.zcseg, zcseg)) != cudaSuccess))
        return e;
    const long total = (long)w * M * h * M * P * M;
    if ((e = cudaMalloc((void**)&t.wsum, sizeof(float) * total)) != cudaSuccess) return e;
    wsum3d_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(t, w, h, P, M, t.wsum);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return cudaStreamSynchronize(stream);
}

// ESRRF_RGC3D=voxel selects the one-voxel-per-thread form (kept for comparison and tests).
bool rgc3d_one_voxel() {
    const char* s = std::getenv("ESRRF_RGC3D");
    return s && std::strcmp(s, "voxel") == 0;
}

size_t rgc3d_field_float4s(const Rgc3dTables& t, int F) { return (size_t)F * t.Pp * t.H2p * t.W2p; }

void rgc3d_tables_free(Rgc3dTables& t) {
    cudaFree(t.taba);
    cudaFree(t.tabb);
    cudaFree(t.start);
    cudaFree(t.wsum);
    cudaFree(t.ztab);
    cudaFree(t.zstart);
    cudaFree(t.zseg);
    cudaFree(t.zcseg);
    cudaFree(t.zsoff);
    t = Rgc3dTables();
}

cudaError_t unit_grad3d(const float* gxi, const float* gyi, const float* gzi, int w, int h, int P,
                        int F, const Rgc3dTables& t, float4* U, cudaStream_t stream) {
    unit_grad3d_kernel<<<dim3((2 * w + 127) / 128, 2 * h, F * P), 128, 0, stream>>>(
        gxi, gyi, gzi, w, h, P, t.padx, t.pady, t.padz_lo, t.W2p, t.H2p, t.Pp, U);
    return cudaGetLastError();
}

cudaError_t rgc_3d_tab(const Rgc3dTabArgs& a, cudaStream_t stream) {
    if (a.tab.ztab && !rgc3d_one_voxel()) {
        // slab-staged form where two CTAs' shared memory fits an SM (ESRRF_RGC3D=zb: the form
        // that reads the field through the L1 cache)
        // and the two-cells-per-thread slab form where its taller slab fits too (ESRRF_RGC3D=zs:
        // one cell per thread)
        const char* env = std::getenv("ESRRF_RGC3D");
        int form = a.form;
        if (form == kRgc3dAuto && env)
            form = std::strcmp(env, "zb") == 0 ? kRgc3dL1 : std::strcmp(env, "zs") == 0 ? kRgc3dSlab : kRgc3dAuto;
        const bool slab = zs_smem_bytes(a.tab) <= 112 * 1024 && 2 * a.tab.sl_nx <= 128 && form != kRgc3dL1;
        const bool two = slab && z2_smem_bytes(a.tab) <= 112 * 1024 && form != kRgc3dSlab;
        switch (a.M) {
            case 2: return two ? launch_z2<2>(a, stream) : slab ? launch_zs<2>(a, stream) : launch_zb<2>(a, stream);
            case 3: return two ? launch_z2<3>(a, stream) : slab ? launch_zs<3>(a, stream) : launch_zb<3>(a, stream);
            case 4: return two ? launch_z2<4>(a, stream) : slab ? launch_zs<4>(a, stream) : launch_zb<4>(a, stream);
            case 5: return two ? launch_z2<5>(a, stream) : slab ? launch_zs<5>(a, stream) : launch_zb<5>(a, stream);
            default: break;
        }
    }
    const size_t smem = sizeof(float4) * 2 * (size_t)a.tab.max_taps;
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static unsigned long long configured = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (smem > 48 * 1024 && dev < 64 && !(configured & (1ull << dev))) {
        if ((e = cudaFuncSetAttribute(rgc3d_tab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      200 * 1024)) != cudaSuccess)
            return e;
        configured |= 1ull << dev;
    }
    const dim3 grid((a.w + 31) / 32, (a.h + 7) / 8, a.M * a.M * a.P * a.M);
    rgc3d_tab_kernel<<<grid, dim3(32, 8), smem, stream>>>(a);
    return cudaGetLastError();
}

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
