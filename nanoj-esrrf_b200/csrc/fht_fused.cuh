// fht_fused.cuh -- the fused tile kernel of the FHT-path RGC (liveSRRF_noInterpolation.cl:245-393),
// shared by rgc_fht.cu (frames without drift) and rgc_fht_drift.cu (launches with drift).
//
// 32x64-pixel output tiles; per frame the kernel stages the interpolated tile plus the RGC halo
// in shared memory, forms the unit gradient field there, and runs the tap loop with each thread
// owning 8 vertically adjacent outputs so that one shared-memory load feeds up to 8 taps.
//
// Tap geometry.  The reference places output pixel xM's centre at xc = xM + 0.5 + sx and takes
// taps at vx = (int)(xc - 0.5) + i + 0.5, i in [-R, R + 1], so a tap's source column is
// X = xM + floor(sx) + i and its offset from the centre dx = i - frac(sx) (up to the rounding of
// xc); the same holds in y.  A frame's shift is uniform over the frame, so the distance weights
// w and w/d of every tap (i, j) are one table per frame, the source tile moves by
// (floor(sx), floor(sy)), and the contribution of an inward tap is w - (w/d) |g x (dx, dy)| on
// the unit gradient g.  Without drift dx = i exactly and the tables are built once.
//  * DRIFT = false: one table (FusedParams), intensity = the interpolated pixel.
//  * DRIFT = true: per-frame tables (DriftParams, prefetched with the frame's tile), the source
//    tile at the frame's integer shift, per-pixel sums of weights from a per-frame 2-D prefix table
//    where the tap box leaves the image, intensity sampled from the tile at the shifted position
//    (getInterpolatedValue).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "device_common.cuh"
#include "esrrf_internal.h"

namespace esrrf {
namespace fused {

constexpr int kTX = 32;          // output columns per CTA (one warp wide)
constexpr int kTYT = 8;          // thread rows per CTA
constexpr int kK = 8;            // outputs per thread (vertical)
constexpr int kTH = kTYT * kK;   // output rows per CTA

// Shared-memory layout for a tap box of side S (S = r1 - r0 + 1, always even).  PAD = 1 (launches
// with drift) adds a column and a row to the tiles: the reference's box of a pixel whose centre
// rounds across an integer starts one source column or row further (see the kernel).
template <int S, int PAD = 0>
struct FusedLayout {
    static constexpr int EW = kTX + S - 1 + PAD, EH = kTH + S - 1 + PAD;  // unit-gradient tile
    static constexpr int IW = EW + 2, IH = EH + 2;            // intensity tile (+1 px margin)
    static constexpr size_t I_bytes = (sizeof(float) * IW * IH + 15) & ~size_t(15);
    static constexpr size_t off_E = 0;
    static constexpr size_t off_I = off_E + ((sizeof(float2) * EW * EH + 15) & ~size_t(15));
    // tap tables: weights [S][S] (w, w/d), chords [2S]; with drift also the frame's record and a
    // second set (the next frame's tables arrive with its tile)
    static constexpr size_t wt_bytes = (sizeof(float2) * S * S + 15) & ~size_t(15);
    static constexpr size_t jr_bytes = (sizeof(int) * 2 * S + 15) & ~size_t(15);
    static constexpr size_t tab_bytes = wt_bytes + jr_bytes + (PAD ? sizeof(FhtDriftFrame) : 0);
    static constexpr int nT = PAD ? 2 : 1;
    static constexpr size_t tail = nT * tab_bytes + sizeof(float) * 5 * kTX * kTH;
    // A second intensity buffer (the next frame's tile prefetched during this frame's taps) is
    // used where two CTAs of 256 threads still fit in an SM's 228 KB of shared memory.
    static constexpr bool kDB = 2 * (off_I + 2 * I_bytes + tail + 1024) <= 228 * 1024;
    static constexpr int nI = kDB ? 2 : 1;
    static constexpr size_t off_wt = off_I + nI * I_bytes;  // table set t at off_wt + t tab_bytes
    static constexpr size_t off_st = off_wt + nT * tab_bytes;
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

// Per-frame tables of a launch with drift (frame index local to the launch).
struct DriftParams {
    const FhtDriftFrame* fr;  // [F]
    const float2* wt;         // [F][S][S] (w, w/d), [ii][jj]
    const int* jr;            // [F][2S] disc chord per column
    const double* pre;        // [F][S+1][S+1] 2-D prefix sums of w
    const float* v;           // [F][H][W] intensity at the shifted position (the sweep's planes; unused here)
    float tSS, tSO;           // the per-tap arithmetic of pixels whose box is moved
};

// One column offset i of the tap box for a thread's 8 outputs: source rows rr = 0 .. S+6 of the
// unit-gradient tile column; row rr feeds output k with tap row jj = rr - k, whose offset from
// the centre is dy = fr0 + jj (fr0 = r0 without drift, r0 - frac(sy) with), and dx = fi.  CHECK
// skips rows outside [lo, hi] (columns whose disc chord is not one of the instantiated ranges).
//
// The inward test g . (dx, dy) < 0 with dy = fr - k is, for gy > 0, k > fr + dx gx / gy, and the
// reverse for gy < 0, so one threshold per source row and one compare per output replace the
// per-output dot product.  gy = +0 gives an infinite threshold of the right sign (the tile stores
// +0, never -0), a zero gradient a NaN threshold (never inward); 1 / gy is the approximate
// reciprocal, whose error only moves the threshold within rounding.  The two tests can disagree only
// where g . (dx, dy) is within rounding of 0, where |g x (dx, dy)| = d and the contribution
// w - (w / d) |g x (dx, dy)| vanishes quadratically.
template <int S, int EW, bool CHECK>
__device__ __forceinline__ void tap_column(const float2* __restrict__ col, float fi, float fr0, int lo,
                                           int hi, const float (&w)[S], const float (&wd)[S],
                                           float (&acc)[kK]) {
#pragma unroll
    for (int rr = 0; rr < S + kK - 1; ++rr) {
        if (CHECK && (rr < lo || rr > hi)) continue;
        const float2 e = col[rr * EW];
        const float fr = fr0 + (float)rr;       // tap row offset of output k = 0
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
template <int S, int EW, int LO, int HI>
__device__ __forceinline__ void tap_chord(const float2* __restrict__ col, float fi, float fr0,
                                          const float (&w)[S], const float (&wd)[S], float (&acc)[kK]) {
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

// Without drift the disc is symmetric in j, so a column's chord inside the box [-R, R+1] is
// either the whole box or the rows -J .. J, i.e. tap rows [LO, S - 2 - LO]: one instantiation per
// LO.  With drift the chords are not symmetric; a column's weights are stored from its chord's
// first row on, so the chord runs as tap rows [0, L - 1] of a column and row origin moved down by
// lo.  Tap boxes of 8 and more take tap_rot (one code path for every L); the small boxes (S 4 and
// 6) one instantiation per chord length L, found by a binary search over L.
template <int S, int EW, int A, int B>
__device__ __forceinline__ void tap_length(const float2* __restrict__ col, float fi, float fr0, int L,
                                           const float (&w)[S], const float (&wd)[S], float (&acc)[kK]) {
    if constexpr (B - A == 1) {
        tap_chord<S, EW, 0, A - 1>(col, fi, fr0, w, wd, acc);
    } else {
        constexpr int MID = (A + B) / 2;
        if (L < MID)
            tap_length<S, EW, A, MID>(col, fi, fr0, L, w, wd, acc);
        else
            tap_length<S, EW, MID, B>(col, fi, fr0, L, w, wd, acc);
    }
}

// One source row of a chord (already loaded: e, its offset fr) for the outputs KLO .. KHI, the
// weights of output k in slot (Q - k) & 7 of an 8-entry register window: the per-tap arithmetic of
// tap_chord.
template <int KLO, int KHI, int Q>
__device__ __forceinline__ void rot_row(float2 e, float fr, float fi, const float (&w8)[8], const float (&wd8)[8],
                                        float (&acc)[kK]) {
    float rgy;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rgy) : "f"(e.y));
    const float thr = fmaf(e.x * rgy, fi, fr);
    const bool neg = e.y < 0.f;
    const float cr0 = fmaf(-e.x, fr, e.y * fi);
#pragma unroll
    for (int k = KLO; k <= KHI; ++k) {
        const float ck = k == 0 ? cr0 : fmaf((float)k, e.x, cr0);
        const float t = fmaf(-fabsf(ck), wd8[(Q - k) & 7], w8[(Q - k) & 7]);
        if (((float)k > thr) != neg) acc[k] += t;
    }
}

// Head rows RR .. 6 of a chord: outputs 0 .. RR (tap rows RR .. 0, window slots RR - k).
template <int EW, int RR>
__device__ __forceinline__ void rot_head(const float2* __restrict__ col, float fr0, float fi, const float (&w8)[8],
                                         const float (&wd8)[8], float (&acc)[kK]) {
    if constexpr (RR < 7) {
        rot_row<0, RR, RR>(col[RR * EW], fr0 + (float)RR, fi, w8, wd8, acc);
        rot_head<EW, RR + 1>(col, fr0, fi, w8, wd8, acc);
    }
}

// Body rows at chunk positions Q .. 7 (Q .. NQ - 1), all outputs; the row at position q is tap
// row 8 + 8m + q, whose weight enters slot q.  frr: the row index as a float (exact), so that the
// row's offset is fr0 + (float)rr as in tap_chord.
template <int EW, int Q, int NQ>
__device__ __forceinline__ void rot_body(const float2* __restrict__ p, const float2* __restrict__ pw, float fr0,
                                         float& frr, float fi, float (&w8)[8], float (&wd8)[8], float (&acc)[kK]) {
    if constexpr (Q < NQ) {
        const float2 wv = pw[Q];
        w8[Q] = wv.x;
        wd8[Q] = wv.y;
        rot_row<0, 7, Q>(p[Q * EW], fr0 + frr, fi, w8, wd8, acc);
        frr += 1.f;
        rot_body<EW, Q + 1, NQ>(p, pw, fr0, frr, fi, w8, wd8, acc);
    }
}

// The remainder rows of the body: positions Q .. n - 1 (n < 8 at run time).
template <int EW, int Q>
__device__ __forceinline__ void rot_rest(const float2* __restrict__ p, const float2* __restrict__ pw, int n,
                                         float fr0, float& frr, float fi, float (&w8)[8], float (&wd8)[8],
                                         float (&acc)[kK]) {
    if constexpr (Q < 7) {
        if (Q < n) {
            rot_body<EW, Q, Q + 1>(p, pw, fr0, frr, fi, w8, wd8, acc);
            rot_rest<EW, Q + 1>(p, pw, n, fr0, frr, fi, w8, wd8, acc);
        }
    }
}

// Tail rows L + T .. L + 6: outputs T + 1 .. 7, tap rows L + T - k in slot T + 7 - k of the
// window reloaded with tap rows L - 7 .. L - 1.  Rows above 7 (chords shorter than 7) were head
// rows and are skipped.
template <int EW, int T>
__device__ __forceinline__ void rot_tail(const float2* __restrict__ pt, int L, float fr0, float frL, float fi,
                                         const float (&w8)[8], const float (&wd8)[8], float (&acc)[kK]) {
    if constexpr (T < 7) {
        if (L + T >= 7) rot_row<T + 1, 7, T + 7>(pt[T * EW], fr0 + (frL + (float)T), fi, w8, wd8, acc);
        rot_tail<EW, T + 1>(pt, L, fr0, frL, fi, w8, wd8, acc);
    }
}

// A chord of runtime length L (tap rows 0 .. L - 1 of the column from col, weights from wc, both
// from the chord's first row; wc is zero beyond L up to S - 1, S >= 8) in one code path for every
// length, so that the code a frame runs stays small: the weights live in an 8-slot register window
// (tap row jj in slot jj & 7) that advances with the rows.  Head rows 0 .. 6 (outputs 0 .. rr; for
// L < 7 the rows past the chord add taps of weight 0), row 7 and the body rows 8 .. L - 1 (all
// outputs; 8-row chunks, then up to 7 remainder rows), and tail rows L .. L + 6 (outputs
// rr - L + 1 .. 7) with the chord's last 7 weights reloaded in a fixed order.  Each output's taps
// are added in increasing tap row, as in tap_chord, so the sums are the same.
template <int S, int EW>
__device__ __forceinline__ void tap_rot(const float2* __restrict__ col, const float2* __restrict__ wc, float fi,
                                        float fr0, int L, float (&acc)[kK]) {
    static_assert(S >= 8, "the head window reads 8 weights of the column");
    float w8[8], wd8[8];
    const float4* w4 = reinterpret_cast<const float4*>(wc);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 v = w4[q];
        w8[2 * q] = v.x;
        wd8[2 * q] = v.y;
        w8[2 * q + 1] = v.z;
        wd8[2 * q + 1] = v.w;
    }
    rot_head<EW, 0>(col, fr0, fi, w8, wd8, acc);
    if (L >= 8) {
        rot_row<0, 7, 7>(col[7 * EW], fr0 + 7.f, fi, w8, wd8, acc);
        int rr = 8;
        float frr = 8.f;
        const float2* p = col + 8 * EW;
        const float2* pw = wc + 8;
#pragma unroll 1
        for (; rr + 8 <= L; rr += 8, p += 8 * EW, pw += 8) rot_body<EW, 0, 8>(p, pw, fr0, frr, fi, w8, wd8, acc);
        rot_rest<EW, 0>(p, pw, L - rr, fr0, frr, fi, w8, wd8, acc);
    }
#pragma unroll
    for (int j = 0; j < 7; ++j) {
        const float2 wv = wc[max(L - 7 + j, 0)];
        w8[j] = wv.x;
        wd8[j] = wv.y;
    }
    rot_tail<EW, 0>(col + L * EW, L, fr0, (float)L, fi, w8, wd8, acc);
}

template <int S, int EW, int LO>
__device__ __forceinline__ void tap_dispatch_sym(const float2* __restrict__ col, float fi, float fr0, int lo,
                                                 int hi, const float (&w)[S], const float (&wd)[S],
                                                 float (&acc)[kK]) {
    if constexpr (LO <= (S - 2) / 2) {
        if (lo == LO && hi == S - 2 - LO) {
            tap_chord<S, EW, LO, S - 2 - LO>(col, fi, fr0, w, wd, acc);
            return;
        }
        tap_dispatch_sym<S, EW, LO + 1>(col, fi, fr0, lo, hi, w, wd, acc);
    } else {
        tap_column<S, EW, true>(col, fi, fr0, lo, hi + kK - 1, w, wd, acc);
    }
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}

// Sum of the tap weights of output (xM, yM) over its in-image taps for a frame with drift where
// the tap box leaves the image: the in-image rectangle of the box from the frame's 2-D prefix
// table (where the box is inside after all, the whole table's sum in the reference's (j, i)
// order).  Called for the pixels of threads near the border only, so not inlined.
template <int S>
static __device__ __noinline__ float drift_wsum_border(const FhtDriftFrame& d, const double* __restrict__ pre,
                                                       int xM, int yM, int r0, int W, int H) {
    const int bx = xM + d.ix + r0, by = yM + d.iy + r0;  // source of tap (ii, jj) = (0, 0)
    const int i0 = max(0, -bx), i1 = min(S - 1, W - 1 - bx);
    const int j0 = max(0, -by), j1 = min(S - 1, H - 1 - by);
    if (i0 == 0 && i1 == S - 1 && j0 == 0 && j1 == S - 1) return d.wsum_int;
    if (i0 > i1 || j0 > j1) return 0.f;
    constexpr int P = S + 1;
    return (float)(pre[(j1 + 1) * P + i1 + 1] - pre[j0 * P + i1 + 1] - pre[(j1 + 1) * P + i0] +
                   pre[j0 * P + i0]);
}

// (int)((double)xc - 0.5), the reference's tap-box start for a float centre xc, in FP32: the
// subtraction rounded towards zero keeps the integer part of the exact difference (the integer
// below |xc - 0.5| is representable and lies between the two), so the truncation agrees.
__device__ __forceinline__ int box_start(float xc) { return __float2int_rz(__fsub_rz(xc, 0.5f)); }

// Intensity of output (xM, yM) of a frame with drift, as the reference reads it
// (liveSRRF_noInterpolation.cl:355-357): the pixel itself for a frame without shift, else
// getInterpolatedValue(xM + sx, yM + sy) -- bicubic from the staged tile where its 4 x 4 support is
// interior (the support lies inside the tile: the tile starts at the frame's floor(sx) plus the
// tap box's first column, less one), bilinear with extrapolation from global memory at the border.
// Not inlined: the tap loop of the kernel that calls it keeps its registers.
static __device__ __noinline__ float drift_intensity(const FhtDriftFrame* d, const float* __restrict__ sI,
                                              const float* __restrict__ frame, int W, int H, int xM, int yM,
                                              int gX0, int gY0, int IW) {
    if (xM >= W || yM >= H) return 0.f;
    if (d->zero) return sI[(yM - gY0) * IW + (xM - gX0)];
    const float x = (float)xM + d->sx, y = (float)yM + d->sy;
    const int u0 = (int)floorf(x), v0 = (int)floorf(y);
    if (!(u0 > 0 && u0 < W - 2 && v0 > 0 && v0 < H - 2)) return dev::sample2d(frame, W, H, x, y);
    const float* r = sI + (v0 - 1 - gY0) * IW + (u0 - 1 - gX0);
    float cx[4];
#pragma unroll
    for (int i = 0; i <= 3; ++i) cx[i] = dev::cubic(x - (float)(u0 - 1 + i));
    float q = 0.f;
#pragma unroll
    for (int j = 0; j <= 3; ++j) {
        float p = 0.f;
#pragma unroll
        for (int i = 0; i <= 3; ++i) p = p + r[j * IW + i] * cx[i];
        q = q + p * dev::cubic(y - (float)(v0 - 1 + j));
    }
    return q;
}

// The reference's box of pixel (xM, yM) of a frame with drift starts at (int)(xc - 0.5) with
// xc = (float)(xM + 0.5 + sx) (liveSRRF_noInterpolation.cl:264-281): one column (row) further than
// the table's floor(sx) where the float rounding of xc reaches the next integer or the truncation
// of a negative xc - 0.5 goes towards zero (mx, my = 1).  The offsets of the taps the two boxes
// share agree (to the rounding of xc), so such a pixel's sums (cg, ws) are corrected by its box's
// moved edges only: the taps of the table's first column (row) leave, those of column (row) S
// come in (the tiles carry that column and row).  sEk: the unit-gradient tile at the pixel's
// table tap (0, 0).  Rare (a fraction within rounding of 1, or pixels left of or above the
// shifted image), so not inlined: the common path keeps its registers and its code compact.
template <int S, int EW>
static __device__ __noinline__ float2 drift_edge(const FhtDriftFrame& df, const float2* __restrict__ sEk, int xM,
                                                 int yM, int mx, int my, int W, int H, float tSO, float tSS,
                                                 float cg, float ws) {
    constexpr int r0c = -(S - 2) / 2;
    const int bx = xM + df.ix + r0c, by = yM + df.iy + r0c;  // source of table tap (0, 0)
    // tap (ii, jj) of the table's geometry, added (sign +1) or removed (-1)
    auto edge = [&](int ii, int jj, float sign) {
        const int X = bx + ii, Y = by + jj;
        if (X < 0 || X >= W || Y < 0 || Y >= H) return;
        // the table's arithmetic (drift_tables_kernel): the removed taps cancel exactly
        const float dx = (float)((double)(r0c + ii) - (double)df.fx);
        const float dy = (float)((double)(r0c + jj) - (double)df.fy);
        const float d = sqrtf(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
        if (!(d != 0.f && d <= tSO)) return;
        float w = __fmul_rn(d, expf(-__fmul_rn(d, d) / tSS));
        w = __fmul_rn(__fmul_rn(__fmul_rn(w, w), w), w);
        ws += sign * w;
        const float2 g = sEk[jj * EW + ii];
        if (g.x * dx + g.y * dy < 0.f) cg += sign * (w - (w / d) * fabsf(g.y * dx - g.x * dy));
    };
    if (mx == 1) {
        for (int jj = 0; jj < S; ++jj) edge(0, jj, -1.f);        // first column leaves
        for (int jj = my; jj < S + my; ++jj) edge(S, jj, 1.f);   // column S comes in
    }
    if (my == 1) {
        for (int ii = mx; ii < S; ++ii) edge(ii, 0, -1.f);       // first row leaves
        for (int ii = mx; ii < S; ++ii) edge(ii, S, 1.f);        // row S comes in
    }
    return make_float2(cg, ws);
}

// GROUPED: the launch may split its frames into groups (gridDim.z); the one-group instantiation
// compiles the frame loop and the fold without the group bookkeeping.
template <int S, bool GROUPED, bool DRIFT>
__global__ void __launch_bounds__(256, 2) fht_rgc_fused_kernel(FhtRgcArgs a, FusedParams fp, DriftParams dp) {
    using L = FusedLayout<S, DRIFT ? 1 : 0>;
    constexpr int EW = L::EW, EH = L::EH, IW = L::IW, IH = L::IH;
    constexpr int r0c = -(S - 2) / 2;
    extern __shared__ __align__(16) unsigned char smem[];
    float2* sE = reinterpret_cast<float2*>(smem + L::off_E);
    float* sIb = reinterpret_cast<float*>(smem + L::off_I);  // nI buffers of L::I_bytes
    float2* swt = reinterpret_cast<float2*>(smem + L::off_wt);  // [ii][jj] = (w, w/d)
    int* sjr = reinterpret_cast<int*>(smem + L::off_wt + L::wt_bytes);
    float* sst = reinterpret_cast<float*>(smem + L::off_st);    // [5][kTH][kTX]

    const int tid = threadIdx.x;
    const int tx = tid & 31, ty = tid >> 5;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTH;
    const int W = a.W, H = a.H;
    const long wh = (long)W * H;

    if constexpr (!DRIFT) {
        for (int idx = tid; idx < S * S; idx += blockDim.x) {
            const int ii = idx / S, jj = idx - ii * S;
            swt[idx] = make_float2(fp.wtab[jj * S + ii], fp.wdtab[jj * S + ii]);
        }
        for (int i = tid; i < 2 * S; i += blockDim.x) sjr[i] = fp.jrange[i];
    }

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
        wsum[k] = DRIFT ? 1.f : (in ? fp.wsum[pix] : 1.f);
        if (emit) continue;
        const int o = (ty * kK + k) * kTX + tx;
        sst[0 * kTX * kTH + o] = 0.f;
        sst[1 * kTX * kTH + o] = 0.f;
        sst[2 * kTX * kTH + o] = 0.f;
        sst[3 * kTX * kTH + o] = 0.f;
        sst[4 * kTX * kTH + o] = in ? a.st.prev[pix] : 0.f;
    }

    constexpr int kIStride = (int)(L::I_bytes / sizeof(float));
    // global origin of frame f's intensity tile: the tap box's first source column and row (at
    // the frame's integer shift) minus the one-pixel margin
    auto origin = [&](int f, int& gx0, int& gy0) {
        int ox = 0, oy = 0;
        if constexpr (DRIFT) {
            ox = dp.fr[f].ix;
            oy = dp.fr[f].iy;
        }
        gx0 = x0 + ox + r0c - 1;
        gy0 = y0 + oy + r0c - 1;
    };
    // interpolated tile of frame f with a one-pixel margin beyond the gradient halo (clamped
    // reads), copied asynchronously into dst; with drift also the frame's tap tables and record
    // into table set tb
    auto prefetch_tile = [&](int f, float* dst, int tb) {
        int gX0, gY0;
        origin(f, gX0, gY0);
        const float* fr = a.interp + (long)f * wh;
        for (int ly = ty; ly < IH; ly += kTYT) {
            const long grow = (long)min(max(gY0 + ly, 0), H - 1) * W;
            for (int lx = tx; lx < IW; lx += kTX)
                cp_async4(dst + ly * IW + lx, fr + grow + min(max(gX0 + lx, 0), W - 1));
        }
        if constexpr (DRIFT) {
            unsigned char* tab = smem + L::off_wt + tb * L::tab_bytes;
            const unsigned char* gw = reinterpret_cast<const unsigned char*>(dp.wt + (long)f * S * S);
            const unsigned char* gj = reinterpret_cast<const unsigned char*>(dp.jr + (long)f * 2 * S);
            constexpr int nw = (int)(sizeof(float2) * S * S / 16), nj = (int)(sizeof(int) * 2 * S / 16);
            constexpr int nr = (int)(sizeof(FhtDriftFrame) / 16);
            for (int q = tid; q < nw + nj + nr; q += blockDim.x) {
                if (q < nw)
                    cp_async16(tab + 16 * q, gw + 16 * q);
                else if (q < nw + nj)
                    cp_async16(tab + L::wt_bytes + 16 * (q - nw), gj + 16 * (q - nw));
                else
                    cp_async16(tab + L::wt_bytes + L::jr_bytes + 16 * (q - nw - nj),
                               reinterpret_cast<const unsigned char*>(dp.fr + f) + 16 * (q - nw - nj));
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (L::kDB && fe > fs) prefetch_tile(fs, sIb, 0);

    for (int f = fs; f < fe; ++f) {
        float* sI = sIb + (L::kDB ? ((f - fs) & 1) * kIStride : 0);
        __syncthreads();
        // 0. this frame's tap tables (drift): prefetched with the tile, or loaded now
        FhtDriftFrame df{};
        float fi0 = (float)r0c, fj0 = (float)r0c;
        const int tb = DRIFT && L::kDB ? ((f - fs) & 1) : 0;
        if constexpr (DRIFT) {
            swt = reinterpret_cast<float2*>(smem + L::off_wt + tb * L::tab_bytes);
            sjr = reinterpret_cast<int*>(smem + L::off_wt + tb * L::tab_bytes + L::wt_bytes);
            if (!L::kDB) {
                const float2* wt = dp.wt + (long)f * S * S;
                for (int idx = tid; idx < S * S; idx += blockDim.x) swt[idx] = wt[idx];
                for (int i = tid; i < 2 * S; i += blockDim.x) sjr[i] = dp.jr[(long)f * 2 * S + i];
            }
        }
        int gX0, gY0;
        origin(f, gX0, gY0);
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
        // the frame's record: in shared memory with its prefetched tables, else in global memory;
        // only the tap origins are read before the tap loop (the rest after it, to keep the loop's
        // registers free)
        const FhtDriftFrame* rec =
            L::kDB ? reinterpret_cast<const FhtDriftFrame*>(smem + L::off_wt + tb * L::tab_bytes + L::wt_bytes +
                                                            L::jr_bytes)
                   : dp.fr + f;
        if constexpr (DRIFT) {
            fi0 = rec->fi0;
            fj0 = rec->fj0;
        }
        // 2. unit gradient at each tap source: Gx read at min(X+1, W-1), Gy at min(Y+1, H-1),
        //    Roberts cross with max(.-1, 0) clamps (liveSRRF_noInterpolation.cl:144-155, 291-292)
        for (int ey = ty; ey < EH; ey += kTYT) {
            const int Y = gY0 + 1 + ey;
            const bool yin = Y >= 0 && Y < H;
            const int ya0 = max(Y - 1, 0), yb = min(Y + 1, H - 1), yb0 = max(yb - 1, 0);
            for (int ex = tx; ex < EW; ex += kTX) {
                const int X = gX0 + 1 + ex;
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
        if (L::kDB && f + 1 < fe) prefetch_tile(f + 1, sIb + ((f + 1 - fs) & 1) * kIStride, (f + 1 - fs) & 1);
        // 3. tap loop, one box column at a time with its weights in registers
        float acc[kK];
#pragma unroll
        for (int k = 0; k < kK; ++k) acc[k] = 0.f;
        for (int ii = 0; ii < S; ++ii) {
            const int lo = sjr[2 * ii], hi = sjr[2 * ii + 1];
            if (lo > hi) continue;  // no tap of the disc in this column
            const float fi = fi0 + (float)ii;
            if constexpr (DRIFT && S >= 8) {
                // weights stored from the chord's first row: rows lo .. hi as 0 .. L - 1
                tap_rot<S, EW>(sE + (ty * kK + lo) * EW + tx + ii, swt + ii * S, fi, fj0 + (float)lo,
                               min(hi - lo + 1, S), acc);
                continue;
            }
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
            if constexpr (DRIFT) {
                // weights stored from the chord's first row: rows lo .. hi as 0 .. L - 1
                tap_length<S, EW, 1, S + 1>(col + lo * EW, fi, fj0 + (float)lo, min(hi - lo + 1, S), w, wd, acc);
            } else if (lo == 0 && hi == S - 1) {
                tap_chord<S, EW, 0, S - 1>(col, fi, fj0, w, wd, acc);
            } else {
                tap_dispatch_sym<S, EW, 0>(col, fi, fj0, lo, hi, w, wd, acc);
            }
        }
        if constexpr (DRIFT) {
            df = *rec;
            gX0 = x0 + df.ix + r0c - 1;
            gY0 = y0 + df.iy + r0c - 1;
            // sums of weights: the table's where the thread's 8 tap boxes lie inside the image
            {
                const int bx = xM + df.ix + r0c, by = y0 + ty * kK + df.iy + r0c;
                const bool inside = bx >= 0 && bx + S - 1 < W && by >= 0 && by + kK - 1 + S - 1 < H;
                const double* pre = dp.pre + (long)f * (S + 1) * (S + 1);
#pragma unroll
                for (int k = 0; k < kK; ++k)
                    wsum[k] = inside ? df.wsum_int : drift_wsum_border<S>(df, pre, xM, y0 + ty * kK + k, r0c, W, H);
            }
            // pixels whose reference box starts one column or row further (drift_edge).  The
            // centre xc = (float)(xM + 0.5 + sx) (liveSRRF_noInterpolation.cl:264-265): xM + 0.5
            // is exact in FP32, so one rounded addition gives it.  mx once per thread; my per row
            // only where it can be non-zero, i.e. where the rounding of yc (at most half an ulp of
            // |yc| <= H + |sy| + 1, below 2^-24 of it) can reach the next integer, or for rows at
            // or above the shifted image's top
            const float xc = __fadd_rn((float)xM + 0.5f, df.sx);
            const int mx = box_start(xc) - (xM + df.ix);
            const bool ychk = (1.f - df.fy) * 4194304.f <= (float)H + fabsf(df.sy) + 2.f || y0 + ty * kK + df.iy < 1;
            if (mx != 0 || ychk) {
#pragma unroll
                for (int k = 0; k < kK; ++k) {
                    const int yM = y0 + ty * kK + k;
                    const float yc = __fadd_rn((float)yM + 0.5f, df.sy);
                    const int my = box_start(yc) - (yM + df.iy);
                    if ((mx == 0 && my == 0) || mx < 0 || mx > 1 || my < 0 || my > 1 || xM >= W || yM >= H)
                        continue;
                    const float2 r = drift_edge<S, EW>(df, sE + (ty * kK + k) * EW + tx, xM, yM, mx, my, W, H,
                                                       dp.tSO, dp.tSS, acc[k], wsum[k]);
                    acc[k] = r.x;
                    wsum[k] = r.y;
                }
            }
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
        // Intensities of a frame with drift, separably: the thread's 8 outputs share their column,
        // so the x weights of getInterpolatedValue's bicubic; where the 8 shifted rows
        // (float)(yM + sy) also share their fraction (all of them in binades where the rounding of
        // yM + sy gives the same fraction, which the first and last row decide) they share the y
        // weights, and the horizontal sum of a tile row (the bicubic's inner loop) is the same for
        // each of the 4 outputs whose support holds the row: 11 row sums serve the 8 outputs, each
        // output's sums in the reference's order.  Otherwise (borders, binade changes, zero shift)
        // each output is sampled alone (drift_intensity).
        bool sep = false;
        float cxw[4], cyw[4], hp0 = 0.f, hp1 = 0.f, hp2 = 0.f;
        const float* hr = sI;
        if constexpr (DRIFT) {
            const int yA = y0 + ty * kK, yB = yA + kK - 1;
            if (!rec->zero && xM < W && yB < H) {
                const float x = (float)xM + rec->sx;
                const int u0 = (int)floorf(x);
                const float ya = (float)yA + rec->sy, yb = (float)yB + rec->sy;
                const int va = (int)floorf(ya), vb = (int)floorf(yb);
                sep = u0 > 0 && u0 < W - 2 && va > 0 && vb < H - 2 && vb - va == kK - 1 &&
                      ya - (float)va == yb - (float)vb;
                if (sep) {
#pragma unroll
                    for (int i = 0; i <= 3; ++i) {
                        cxw[i] = dev::cubic(x - (float)(u0 - 1 + i));
                        cyw[i] = dev::cubic(ya - (float)(va - 1 + i));
                    }
                    hr = sI + (va - 1 - gY0) * IW + (u0 - 1 - gX0);
                    auto hrow = [&](int m) {
                        float p = 0.f;
#pragma unroll
                        for (int i = 0; i <= 3; ++i) p = p + hr[m * IW + i] * cxw[i];
                        return p;
                    };
                    hp0 = hrow(0);
                    hp1 = hrow(1);
                    hp2 = hrow(2);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kK; ++k) {
            const int o = (ty * kK + k) * kTX + tx;
            const float cg = dev::cglh_power(acc[k] / wsum[k], fp.sens);
            float v;
            if constexpr (DRIFT) {
                if (sep) {
                    float hp3 = 0.f;
#pragma unroll
                    for (int i = 0; i <= 3; ++i) hp3 = hp3 + hr[(k + 3) * IW + i] * cxw[i];
                    float q = 0.f;
                    q = q + hp0 * cyw[0];
                    q = q + hp1 * cyw[1];
                    q = q + hp2 * cyw[2];
                    q = q + hp3 * cyw[3];
                    v = q;
                    hp0 = hp1;
                    hp1 = hp2;
                    hp2 = hp3;
                } else {
                    v = drift_intensity(rec, sI, a.interp + (long)f * wh, W, H, xM, y0 + ty * kK + k, gX0, gY0,
                                        IW);
                }
            } else {
                v = sI[(ty * kK + k + 1 - r0c) * IW + (tx + 1 - r0c)];
            }
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

// Frames of a launch split into g groups across CTAs (blockIdx.z): the g that minimises the
// launch's modelled time, waves(g) x (frames of the largest group + extra), with waves(g) =
// ceil(tiles g / slots) for `slots` resident CTAs.  In the cumulant mode a later group also runs
// the frame before its range (TAC2's previous value), one extra frame, and keeps at least 4
// frames; in the per-frame mode (emit) the frames are independent.  A quarter frame per CTA
// stands for its fixed work (tables, the first tile); g = 1 unless another count is 2 % faster.
// (64 x 64 frames at M5, 50 tiles on 296 slots, 50 frames: 5 groups fit one wave where the
// fewest groups that cover every slot, 6, spill 4 CTAs into a second one.)
inline int frame_groups(int tiles, int F, int slots, bool emit) {
    if (F <= 1 || tiles <= 0 || slots <= 0) return 1;
    const int gmax = std::min(emit ? std::min(F, 64) : std::max(1, F / 4), 65535);
    auto cost = [&](int g) {
        const long waves = ((long)tiles * g + slots - 1) / slots;
        return (double)waves * ((F + g - 1) / g + (g > 1 && !emit ? 1.0 : 0.0) + 0.25);
    };
    int best = 1;
    double tbest = cost(1);
    for (int g = 2; g <= gmax; ++g) {
        const double t = cost(g);
        if (t < 0.98 * tbest) {
            best = g;
            tbest = t;
        }
    }
    return best;
}

// Launch of one tap-box size: the grid, the frame groups and the copy of the last group's
// previous values.
template <int S, bool DRIFT>
cudaError_t launch_fused(int r0, float sens, const FusedParams& fp_in, const DriftParams& dp,
                         const FhtRgcArgs& a, cudaStream_t stream) {
    constexpr size_t bytes = FusedLayout<S, DRIFT ? 1 : 0>::bytes;
    // The opt-in shared-memory size is a per-device function attribute: set it once per device
    // (also keeps the call out of CUDA-graph captures after the first, uncaptured launch).
    static unsigned long long configured = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 64 || !(configured & (1ull << dev))) {
        if ((e = cudaFuncSetAttribute(fht_rgc_fused_kernel<S, false, DRIFT>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes)) != cudaSuccess ||
            (e = cudaFuncSetAttribute(fht_rgc_fused_kernel<S, true, DRIFT>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes)) != cudaSuccess)
            return e;
        if (dev < 64) configured |= 1ull << dev;
    }
    FusedParams fp = fp_in;
    fp.r0 = r0;
    fp.sens = sens;
    dim3 grid((a.W + kTX - 1) / kTX, (a.H + kTH - 1) / kTH);
    const int tiles = (int)(grid.x * grid.y), slots = 2 * sm_count(dev);
    if (a.F > 1 && (a.cg_out || a.prev_out))
        grid.z = (unsigned)frame_groups(tiles, a.F, slots, a.cg_out != nullptr);
    if (grid.z > 1)
        fht_rgc_fused_kernel<S, true, DRIFT><<<grid, 256, bytes, stream>>>(a, fp, dp);
    else
        fht_rgc_fused_kernel<S, false, DRIFT><<<grid, 256, bytes, stream>>>(a, fp, dp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (grid.z > 1 && !a.cg_out)
        return cudaMemcpyAsync(a.st.prev, a.prev_out, sizeof(float) * (size_t)a.W * a.H,
                               cudaMemcpyDeviceToDevice, stream);
    return cudaSuccess;
}

// The tap box side S = 2 * loop radius + 2 is even; one instantiation per size keeps the weight
// offsets and the tile geometry compile-time constants.  Sizes SLO .. SHI (even) are dispatched
// here; others return cudaErrorInvalidValue (the caller uses the plain kernel).
template <bool DRIFT, int SLO, int SHI>
cudaError_t launch_fused_in(int S, int r0, float sens, const FusedParams& fp, const DriftParams& dp,
                            const FhtRgcArgs& a, cudaStream_t stream) {
    if (S == SLO) return launch_fused<SLO, DRIFT>(r0, sens, fp, dp, a, stream);
    if constexpr (SLO + 2 <= SHI) return launch_fused_in<DRIFT, SLO + 2, SHI>(S, r0, sens, fp, dp, a, stream);
    return cudaErrorInvalidValue;
}

}  // namespace fused
}  // namespace esrrf
