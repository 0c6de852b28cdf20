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

// ---------------------------------------------------------------------------------------------
// Fused tile kernel.
// ---------------------------------------------------------------------------------------------
constexpr int kTX = 32;          // output columns per CTA (one warp wide)
constexpr int kTYT = 8;          // thread rows per CTA
constexpr int kK = 8;            // outputs per thread (vertical)
constexpr int kTH = kTYT * kK;   // output rows per CTA

// Shared-memory layout for a tap box of side S (S = r1 - r0 + 1, always even).
template <int S>
struct FusedLayout {
    static constexpr int EW = kTX + S - 1, EH = kTH + S - 1;  // unit-gradient tile
    static constexpr int IW = EW + 2, IH = EH + 2;            // intensity tile (+1 px margin)
    static constexpr size_t I_bytes = (sizeof(float) * IW * IH + 15) & ~size_t(15);
    static constexpr size_t off_E = 0;
    static constexpr size_t off_I = off_E + ((sizeof(float2) * EW * EH + 15) & ~size_t(15));
    static constexpr size_t tail = ((sizeof(float2) * S * S + sizeof(int) * 2 * S + 15) & ~size_t(15)) +
                                   sizeof(float) * 5 * kTX * kTH;
    // A second intensity buffer (the next frame's tile prefetched during this frame's taps) is
    // used where two CTAs of 256 threads still fit in an SM's 228 KB of shared memory.
    static constexpr bool kDB = 2 * (off_I + 2 * I_bytes + tail + 1024) <= 228 * 1024;
    static constexpr int nI = kDB ? 2 : 1;
    static constexpr size_t off_wt = off_I + nI * I_bytes;
    static constexpr size_t off_jr = off_wt + sizeof(float2) * S * S;
    static constexpr size_t off_st = (off_jr + sizeof(int) * 2 * S + 15) & ~size_t(15);
    static constexpr size_t bytes = off_st + sizeof(float) * 5 * kTX * kTH;
};

struct FusedParams {
    int r0;
    float sens;
    const float* wtab;
    const float* wdtab;
    const int* jrange;
    const float* wsum;
};

// One column offset i of the tap box for a thread's 8 outputs: source rows rr = 0 .. S+6 of the
// unit-gradient tile column; row rr feeds output k with tap row jj = rr - k, j = r0 + jj, where
// r0 = -(S - 2) / 2 (the box of an integer radius R is [-R, R + 1]).  CHECK skips rows outside
// [lo, hi] (columns whose disc chord is shorter than the box).
//
// The inward test g . (i, j) < 0 with j = fr - k is, for gy > 0, k > fr + i gx / gy, and the
// reverse for gy < 0, so one threshold per source row and one compare per output replace the
// per-output dot product.  gy = +0 gives an infinite threshold of the right sign (the tile stores
// +0, never -0), a zero gradient a NaN threshold (never inward); 1 / gy is the approximate
// reciprocal, whose error only moves the threshold within rounding.  The two tests can disagree only
// where g . (i, j) is within rounding of 0, where |g x (i, j)| = d and the contribution
// w - (w / d) |g x (i, j)| vanishes quadratically.
template <int S, bool CHECK>
__device__ __forceinline__ void tap_column(const float2* __restrict__ col, float fi, int lo, int hi,
                                           const float (&w)[S], const float (&wd)[S],
                                           float (&acc)[kK]) {
    constexpr int EW = FusedLayout<S>::EW;
    constexpr float fr0 = -(float)((S - 2) / 2);
#pragma unroll
    for (int rr = 0; rr < S + kK - 1; ++rr) {
        if (CHECK && (rr < lo || rr > hi)) continue;
        const float2 e = col[rr * EW];
        const float fr = fr0 + (float)rr;       // tap row j of output k = 0
        float rgy;  // 1 / gy, +-inf for gy = +-0 (subnormals flush to a zero of their sign)
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rgy) : "f"(e.y));
        const float thr = fmaf(e.x * rgy, fi, fr);
        const bool neg = e.y < 0.f;
        const float cr0 = fmaf(-e.x, fr, e.y * fi);
#pragma unroll
        for (int k = 0; k < kK; ++k) {
            const int jj = rr - k;
            if (jj >= 0 && jj < S) {
                // cross = cr0 + k g_x (independent of k - 1)
                const float ck = k == 0 ? cr0 : fmaf((float)k, e.x, cr0);
                const float t = fmaf(-fabsf(ck), wd[jj], w[jj]);
                if (((float)k > thr) != neg) acc[k] += t;
            }
        }
    }
}

// A column whose disc chord is the compile-time tap-row range [LO, HI]: only the chord's taps
// are evaluated (rows LO .. HI + 7, and per row only the outputs whose tap row is in the chord).
template <int S, int LO, int HI>
__device__ __forceinline__ void tap_chord(const float2* __restrict__ col, float fi, const float (&w)[S],
                                          const float (&wd)[S], float (&acc)[kK]) {
    constexpr int EW = FusedLayout<S>::EW;
    constexpr float fr0 = -(float)((S - 2) / 2);
#pragma unroll
    for (int rr = LO; rr <= HI + kK - 1; ++rr) {
        const float2 e = col[rr * EW];
        const float fr = fr0 + (float)rr;
        float rgy;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rgy) : "f"(e.y));
        const float thr = fmaf(e.x * rgy, fi, fr);
        const bool neg = e.y < 0.f;
        const float cr0 = fmaf(-e.x, fr, e.y * fi);
#pragma unroll
        for (int k = 0; k < kK; ++k) {
            const int jj = rr - k;
            if (jj >= LO && jj <= HI) {
                const float ck = k == 0 ? cr0 : fmaf((float)k, e.x, cr0);
                const float t = fmaf(-fabsf(ck), wd[jj], w[jj]);
                if (((float)k > thr) != neg) acc[k] += t;
            }
        }
    }
}

// The disc is symmetric in j, so a column's chord inside the box [-R, R+1] is either the whole
// box or the rows -J .. J, i.e. tap rows [LO, S - 2 - LO]: one instantiation per LO.  Any other
// range takes the generic row-checked loop.
template <int S, int LO>
__device__ __forceinline__ void tap_dispatch(const float2* __restrict__ col, float fi, int lo, int hi,
                                             const float (&w)[S], const float (&wd)[S],
                                             float (&acc)[kK]) {
    if constexpr (LO <= (S - 2) / 2) {
        if (lo == LO && hi == S - 2 - LO) {
            tap_chord<S, LO, S - 2 - LO>(col, fi, w, wd, acc);
            return;
        }
        tap_dispatch<S, LO + 1>(col, fi, lo, hi, w, wd, acc);
    } else {
        tap_column<S, true>(col, fi, lo, hi + kK - 1, w, wd, acc);
    }
}

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}

// GROUPED: the launch may split its frames into groups (gridDim.z); the one-group instantiation
// compiles the frame loop and the fold without the group bookkeeping.
template <int S, bool GROUPED>
__global__ void __launch_bounds__(256, 2) fht_rgc_fused_kernel(FhtRgcArgs a, FusedParams fp) {
    using L = FusedLayout<S>;
    constexpr int EW = L::EW, EH = L::EH, IW = L::IW, IH = L::IH;
    extern __shared__ __align__(16) unsigned char smem[];
    float2* sE = reinterpret_cast<float2*>(smem + L::off_E);
    float* sIb = reinterpret_cast<float*>(smem + L::off_I);  // nI buffers of L::I_bytes
    float2* swt = reinterpret_cast<float2*>(smem + L::off_wt);  // [ii][jj] = (w, w/d)
    int* sjr = reinterpret_cast<int*>(smem + L::off_jr);
    float* sst = reinterpret_cast<float*>(smem + L::off_st);    // [5][kTH][kTX]

    const int tid = threadIdx.x;
    const int tx = tid & 31, ty = tid >> 5;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTH;
    const int r0 = fp.r0;
    const int W = a.W, H = a.H;
    const long wh = (long)W * H;

    for (int idx = tid; idx < S * S; idx += blockDim.x) {
        const int ii = idx / S, jj = idx - ii * S;
        swt[idx] = make_float2(fp.wtab[jj * S + ii], fp.wdtab[jj * S + ii]);
    }
    for (int i = tid; i < 2 * S; i += blockDim.x) sjr[i] = fp.jrange[i];

    const int xM = x0 + tx;
    const bool emit = a.cg_out != nullptr;
    // frame group: frames [fb, fe) of the launch (one group unless the tiles alone leave SMs
    // idle); a later group first runs frame fb - 1 only for its intensity-weighted value, the
    // previous value of TAC2's product at fb
    const int G = GROUPED ? (int)gridDim.z : 1, grp = GROUPED ? (int)blockIdx.z : 0;
    const int fb = (int)((long long)a.F * grp / G), fe = (int)((long long)a.F * (grp + 1) / G);
    const int fs = grp > 0 && !emit ? fb - 1 : fb;
    float wsum[kK];
#pragma unroll
    for (int k = 0; k < kK; ++k) {
        const int yM = y0 + ty * kK + k;
        const bool in = xM < W && yM < H;
        const long pix = (long)yM * W + xM;
        wsum[k] = in ? fp.wsum[pix] : 1.f;
        if (emit) continue;
        const int o = (ty * kK + k) * kTX + tx;
        sst[0 * kTX * kTH + o] = 0.f;
        sst[1 * kTX * kTH + o] = 0.f;
        sst[2 * kTX * kTH + o] = 0.f;
        sst[3 * kTX * kTH + o] = 0.f;
        sst[4 * kTX * kTH + o] = in ? a.st.prev[pix] : 0.f;
    }

    const int gX0 = x0 + r0 - 1, gY0 = y0 + r0 - 1;  // global origin of the intensity tile
    const float fr0 = (float)r0;
    constexpr int kIStride = (int)(L::I_bytes / sizeof(float));
    // interpolated tile of frame f with a one-pixel margin beyond the gradient halo (clamped
    // reads), copied asynchronously into dst
    auto prefetch_tile = [&](int f, float* dst) {
        const float* fr = a.interp + (long)f * wh;
        for (int ly = ty; ly < IH; ly += kTYT) {
            const long grow = (long)min(max(gY0 + ly, 0), H - 1) * W;
            for (int lx = tx; lx < IW; lx += kTX)
                cp_async4(dst + ly * IW + lx, fr + grow + min(max(gX0 + lx, 0), W - 1));
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (L::kDB && fe > fs) prefetch_tile(fs, sIb);

    for (int f = fs; f < fe; ++f) {
        float* sI = sIb + (L::kDB ? ((f - fs) & 1) * kIStride : 0);
        __syncthreads();
        // 1. this frame's intensity tile: prefetched during the previous frame, or loaded now
        if (L::kDB) {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        } else {
            const float* fr = a.interp + (long)f * wh;
            for (int ly = ty; ly < IH; ly += kTYT) {
                const long grow = (long)min(max(gY0 + ly, 0), H - 1) * W;
                for (int lx = tx; lx < IW; lx += kTX)
                    sI[ly * IW + lx] = __ldg(fr + grow + min(max(gX0 + lx, 0), W - 1));
            }
        }
        __syncthreads();
        // 2. unit gradient at each tap source: Gx read at min(X+1, W-1), Gy at min(Y+1, H-1),
        //    Roberts cross with max(.-1, 0) clamps (liveSRRF_noInterpolation.cl:144-155, 291-292)
        for (int ey = ty; ey < EH; ey += kTYT) {
            const int Y = y0 + r0 + ey;
            const bool yin = Y >= 0 && Y < H;
            const int ya0 = max(Y - 1, 0), yb = min(Y + 1, H - 1), yb0 = max(yb - 1, 0);
            for (int ex = tx; ex < EW; ex += kTX) {
                const int X = x0 + r0 + ex;
                float2 e = make_float2(0.f, 0.f);
                if (yin && X >= 0 && X < W) {
                    const int xa = min(X + 1, W - 1), xa0 = max(xa - 1, 0), xb0 = max(X - 1, 0);
                    const float ga = sI[(ya0 - gY0) * IW + (xa - gX0)];
                    const float gb = sI[(Y - gY0) * IW + (xa0 - gX0)];
                    const float gc = sI[(Y - gY0) * IW + (xa - gX0)];
                    const float gd = sI[(ya0 - gY0) * IW + (xa0 - gX0)];
                    const float Gx = ga - gb + gc - gd;
                    const float ha = sI[(yb0 - gY0) * IW + (X - gX0)];
                    const float hb = sI[(yb - gY0) * IW + (xb0 - gX0)];
                    const float hc = sI[(yb - gY0) * IW + (X - gX0)];
                    const float hd = sI[(yb0 - gY0) * IW + (xb0 - gX0)];
                    const float Gy = -ha + hb + hc - hd;
                    const float n2 = Gx * Gx + Gy * Gy;
                    if (n2 > 0.f) {
                        const float inv = rsqrtf(n2);
                        e = make_float2(Gx * inv, Gy * inv + 0.f);  // + 0: -0 becomes +0
                    }
                }
                sE[ey * EW + ex] = e;
            }
        }
        __syncthreads();
        // the next frame's tile goes into the other buffer while this frame's taps run
        if (L::kDB && f + 1 < fe) prefetch_tile(f + 1, sIb + ((f + 1 - fs) & 1) * kIStride);
        // 3. tap loop, one box column at a time with its weights in registers
        float acc[kK];
#pragma unroll
        for (int k = 0; k < kK; ++k) acc[k] = 0.f;
        for (int ii = 0; ii < S; ++ii) {
            const int lo = sjr[2 * ii], hi = sjr[2 * ii + 1];
            if (lo > hi) continue;  // no tap of the disc in this column
            const float fi = fr0 + (float)ii;
            float w[S], wd[S];
            const float4* wc = reinterpret_cast<const float4*>(swt + ii * S);
#pragma unroll
            for (int q = 0; q < S / 2; ++q) {
                const float4 v = wc[q];
                w[2 * q] = v.x;
                wd[2 * q] = v.y;
                w[2 * q + 1] = v.z;
                wd[2 * q + 1] = v.w;
            }
            const float2* col = sE + (ty * kK) * EW + tx + ii;
            if (lo == 0 && hi == S - 1)
                tap_chord<S, 0, S - 1>(col, fi, w, wd, acc);
            else
                tap_dispatch<S, 0>(col, fi, lo, hi, w, wd, acc);
        }
        // 4. normalisation, sensitivity, intensity weighting and cumulants
        if (emit) {
#pragma unroll
            for (int k = 0; k < kK; ++k) {
                const int yM = y0 + ty * kK + k;
                if (xM < W && yM < H) a.cg_out[(long)f * wh + (long)yM * W + xM] = acc[k] / wsum[k];
            }
            continue;
        }
        const int tglob = a.t0 + f;
#pragma unroll
        for (int k = 0; k < kK; ++k) {
            const int o = (ty * kK + k) * kTX + tx;
            const float cg = cglh_power(acc[k] / wsum[k], fp.sens);
            const float v = sI[(ty * kK + k + 1 - r0) * IW + (tx + 1 - r0)];
            const float x = a.int_weighting ? v * cg : cg;
            if (f < fb) {  // the frame before the group: previous value only
                sst[4 * kTX * kTH + o] = x;
                continue;
            }
            const float pv = sst[4 * kTX * kTH + o];
            sst[0 * kTX * kTH + o] += x;
            sst[1 * kTX * kTH + o] += x * x;
            if (tglob > 0) sst[2 * kTX * kTH + o] += x * pv;
            sst[3 * kTX * kTH + o] += v;
            sst[4 * kTX * kTH + o] = x;
        }
    }
    // 5. fold this launch's FP32 partial sums into the block's FP64 accumulators
    if (emit) return;
#pragma unroll
    for (int k = 0; k < kK; ++k) {
        const int yM = y0 + ty * kK + k;
        if (xM >= W || yM >= H) continue;
        const long pix = (long)yM * W + xM;
        const int o = (ty * kK + k) * kTX + tx;
        if (G == 1) {
            a.st.acc[pix] += (double)sst[0 * kTX * kTH + o];
            a.st.acc[wh + pix] += (double)sst[1 * kTX * kTH + o];
            a.st.acc[2 * wh + pix] += (double)sst[2 * kTX * kTH + o];
            a.st.acc[3 * wh + pix] += (double)sst[3 * kTX * kTH + o];
        } else {  // several groups add into the same pixels
#pragma unroll
            for (int c = 0; c < 4; ++c) atomicAdd(a.st.acc + c * wh + pix, (double)sst[c * kTX * kTH + o]);
        }
        if (grp == G - 1) (G == 1 ? a.st.prev : a.prev_out)[pix] = sst[4 * kTX * kTH + o];
    }
}

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

template <int S>
cudaError_t launch_fused(const FhtGeometry& g, const FhtFusedTables& t, const FhtRgcArgs& a,
                         cudaStream_t stream) {
    constexpr size_t bytes = FusedLayout<S>::bytes;
    // The opt-in shared-memory size is a per-device function attribute: set it once per device
    // (also keeps the call out of CUDA-graph captures after the first, uncaptured launch).
    static unsigned long long configured = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 64 || !(configured & (1ull << dev))) {
        if ((e = cudaFuncSetAttribute(fht_rgc_fused_kernel<S, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)bytes)) != cudaSuccess ||
            (e = cudaFuncSetAttribute(fht_rgc_fused_kernel<S, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)bytes)) != cudaSuccess)
            return e;
        if (dev < 64) configured |= 1ull << dev;
    }
    FusedParams fp{g.r0, g.sensitivity, t.wtab, t.wdtab, t.jrange, t.wsum};
    dim3 grid((a.W + kTX - 1) / kTX, (a.H + kTH - 1) / kTH);
    // frames split into groups across CTAs only where the tiles alone give fewer than two CTAs
    // per SM (small frames); a group keeps at least 4 frames when it pays an extra frame
    const int tiles = (int)(grid.x * grid.y), slots = 2 * sm_count(dev);
    if (tiles < slots && a.F > 1 && (a.cg_out || a.prev_out)) {
        const int gmax = a.cg_out ? a.F : std::max(1, a.F / 4);
        grid.z = (unsigned)std::max(1, std::min({(slots + tiles - 1) / tiles, gmax, 65535}));
    }
    if (grid.z > 1)
        fht_rgc_fused_kernel<S, true><<<grid, 256, bytes, stream>>>(a, fp);
    else
        fht_rgc_fused_kernel<S, false><<<grid, 256, bytes, stream>>>(a, fp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (grid.z > 1 && !a.cg_out)
        return cudaMemcpyAsync(a.st.prev, a.prev_out, sizeof(float) * (size_t)a.W * a.H,
                               cudaMemcpyDeviceToDevice, stream);
    return cudaSuccess;
}

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
    // The tap box side S = 2 * loop radius + 2 is even; one instantiation per size keeps the
    // weight offsets and the tile geometry compile-time constants.
    switch (g.S) {
        case 4: return launch_fused<4>(g, t, a, stream);
        case 6: return launch_fused<6>(g, t, a, stream);
        case 8: return launch_fused<8>(g, t, a, stream);
        case 10: return launch_fused<10>(g, t, a, stream);
        case 12: return launch_fused<12>(g, t, a, stream);
        case 14: return launch_fused<14>(g, t, a, stream);
        case 16: return launch_fused<16>(g, t, a, stream);
        case 18: return launch_fused<18>(g, t, a, stream);
        case 20: return launch_fused<20>(g, t, a, stream);
        case 22: return launch_fused<22>(g, t, a, stream);
        case 24: return launch_fused<24>(g, t, a, stream);
        case 26: return launch_fused<26>(g, t, a, stream);
        case 28: return launch_fused<28>(g, t, a, stream);
        case 30: return launch_fused<30>(g, t, a, stream);
        case 32: return launch_fused<32>(g, t, a, stream);
        default: return cudaErrorInvalidValue;  // caller uses the plain kernel
    }
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
