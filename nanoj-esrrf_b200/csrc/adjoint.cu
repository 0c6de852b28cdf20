// adjoint.cu -- differentiable eSRRF: a fidelity loss of the 2-D FHT-path AVG reconstruction
// and its hand-written adjoint, with respect to the radius (fwhm), a real-valued sensitivity S,
// the re-blur sigma and every input pixel.
//
// Loss (a SQUIRREL-style error, cf. ErrorMapLiveSRRF.java:81-233; the reference has no
// differentiable form):  R = (1/T) sum_t I_t C_t^S  (I_t interpolated frames, C_t = CGLH / sum of
// weights), B = Gaussian(sigma) * R, D = M x M box average of B, F = frame average of the input,
// alpha, beta = least-squares fit F ~ alpha D + beta, loss = mean((alpha D + beta - F)^2).
// alpha and beta are refitted for every evaluation, so their own derivatives drop out.
//
// The forward pass of a gradient evaluation runs kernel A's tap loop in its emit form: per frame
// and output pixel C_t and the d^2-weighted sum of the inward taps' terms (what dC/dtSS needs),
// kept for the backward pass with the interpolated frames (a loss-only evaluation runs the fused
// forward kernel instead).  Backward pass, per chunk of frames:
//   kernel A's terms (adj_tail_kernel, per pixel): b = dL/dN (N = C * sum of weights), the
//             intensity-weighting term of dL/dI_t, and the sums dL/dS and dL/dtSS;
//   kernel B: at every tap source, gather dL/dg over the taps whose outputs it feeds
//             (dphi/dg = [g.t < 0] (w/d) sgn(c) (t_y, -t_x), c = g_y t_x - g_x t_y), project onto
//             the unit-vector tangent, and scatter through the Roberts cross (atomics) into
//             dL/dI_t;
//   then the transposed Fourier interpolation (interp.cu) gives dL/draw_t.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/esrrf.h"
#include "device_common.cuh"
#include "esrrf_internal.h"

using namespace esrrf;

namespace {

constexpr int kTX = 32, kTYT = 8, kK = 8, kTH = 64;
constexpr int kMaxGauss = 129;  // taps of the 1-D re-blur kernel (radius <= 64)

template <int S>
struct AdjLayout {
    static constexpr int EW = kTX + S - 1, EH = kTH + S - 1;
    static constexpr int IW = EW + 2, IH = EH + 2;
    static constexpr size_t I_bytes = (sizeof(float) * IW * IH + 15) & ~size_t(15);
    static constexpr size_t off_E = 0;
    static constexpr size_t off_I = (off_E + sizeof(float2) * EW * EH + 15) & ~size_t(15);  // 2 buffers
    static constexpr size_t off_wt = off_I + 2 * I_bytes;
    static constexpr size_t bytes = off_wt + sizeof(float4) * S * S;
};

// 4-byte asynchronous copy into shared memory; valid = false writes a zero and reads nothing
__device__ __forceinline__ void cp_async4z(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(valid ? 4 : 0)
                 : "memory");
}

struct AdjAArgs {
    const float* I;      // [F][H][W] interpolated frames of the chunk
    const float* a;      // [H][W] dL/dR / T
    const float4* tab;   // [ii][jj] (w, w/d, kappa = 4 d^2 / tSS^2, 0); the taps use w and w/d
    const float* wsum;   // [H][W]
    const float* dwsum;  // [H][W] d(sum of weights)/dtSS
    const int* jr;       // [S][2] disc chord (first, last tap row) of each tap column
    int W, H, F, r0;
    float kscale;        // 4 / tSS^2: dw/dtSS = w 4 d^2 / tSS^2
    float sens;
    float* b;            // [F][H][W] dL/dN
    float* gI;           // [F][H][W] initialised with the intensity-weighting term
    double* acc;         // [2]: dL/dS, dL/dtSS
    // forward of a gradient evaluation: if set, write C = CGLH / sum of weights and the
    // d^2-weighted inward tap sum per frame and pixel instead of the backward terms (b, gI, acc)
    float* c_out = nullptr;  // [F][H][W]
    float* q_out = nullptr;  // [F][H][W]
};

// One tap column of kernel A restricted to its disc chord [LO, HI] (compile-time, as in the fused
// forward kernel), with the forward kernel's per-row inward threshold.
template <int S, int LO, int HI>
__device__ __forceinline__ void chord_a(const float2* __restrict__ col, float fi, const float (&w)[S],
                                        const float (&wd)[S], float (&acc)[kK], float (&acc2)[kK]) {
    constexpr int EW = AdjLayout<S>::EW;
    constexpr float fr0 = -(float)((S - 2) / 2);
#pragma unroll
    for (int rr = LO; rr <= HI + kK - 1; ++rr) {
        const float2 e = col[rr * EW];
        const float fr = fr0 + (float)rr;
        // inward test g . (i, fr - k) < 0 as one threshold per source row (as the forward fused
        // kernel): k > thr for gy > 0, k < thr for gy < 0, thr = fr + i gx / gy
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
                if (((float)k > thr) != neg) {
                    acc[k] += t;
                    const float j = fr0 + (float)jj;
                    acc2[k] = fmaf(j * j, t, acc2[k]);  // j^2 t; i^2 t is added per column
                }
            }
        }
    }
}

// The whole box, rows checked by weight (any chord shape; the disc gives the two forms below).
template <int S>
__device__ __forceinline__ void box_a(const float2* __restrict__ col, float fi, const float (&w)[S],
                                      const float (&wd)[S], float (&acc)[kK], float (&acc2)[kK]) {
    constexpr int EW = AdjLayout<S>::EW;
    constexpr float fr0 = -(float)((S - 2) / 2);
#pragma unroll
    for (int rr = 0; rr < S + kK - 1; ++rr) {
        const float2 e = col[rr * EW];
        const float frr = fr0 + (float)rr;
        const float dot0 = fmaf(e.y, frr, e.x * fi);
        const float cr0 = fmaf(-e.x, frr, e.y * fi);
#pragma unroll
        for (int k = 0; k < kK; ++k) {
            const int jj = rr - k;
            if (jj >= 0 && jj < S) {
                const float dk = k == 0 ? dot0 : fmaf(-(float)k, e.y, dot0);
                const float ck = k == 0 ? cr0 : fmaf((float)k, e.x, cr0);
                const float t = fmaf(-fabsf(ck), wd[jj], w[jj]);
                if (dk < 0.f) {
                    acc[k] += t;
                    const float j = fr0 + (float)jj;
                    acc2[k] = fmaf(j * j, t, acc2[k]);  // j^2 t; i^2 t is added per column
                }
            }
        }
    }
}

// A column's chord in the box [-R, R+1] is the whole box or tap rows [LO, S - 2 - LO].
template <int S, int LO>
__device__ __forceinline__ void dispatch_a(const float2* __restrict__ col, float fi, int lo, int hi,
                                           const float (&w)[S], const float (&wd)[S], float (&acc)[kK],
                                           float (&acc2)[kK]) {
    if constexpr (LO <= (S - 2) / 2) {
        if (lo == LO && hi == S - 2 - LO) {
            chord_a<S, LO, S - 2 - LO>(col, fi, w, wd, acc, acc2);
            return;
        }
        dispatch_a<S, LO + 1>(col, fi, lo, hi, w, wd, acc, acc2);
    } else {
        box_a<S>(col, fi, w, wd, acc, acc2);
    }
}

// Kernel A: forward tap loop with a second accumulator for dN/dtSS.
template <int S>
__global__ void __launch_bounds__(256, 2) adj_a_kernel(AdjAArgs g) {
    using L = AdjLayout<S>;
    constexpr int EW = L::EW, EH = L::EH, IW = L::IW, IH = L::IH;
    extern __shared__ __align__(16) unsigned char smem[];
    float2* sE = reinterpret_cast<float2*>(smem + L::off_E);
    float* sIb = reinterpret_cast<float*>(smem + L::off_I);
    float4* stab = reinterpret_cast<float4*>(smem + L::off_wt);
    constexpr int kIS = (int)(L::I_bytes / sizeof(float));
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTH, r0 = g.r0;
    const int W = g.W, H = g.H;
    const long wh = (long)W * H;
    for (int i = tid; i < S * S; i += blockDim.x) stab[i] = g.tab[i];
    const int xM = x0 + tx;
    const int gX0 = x0 + r0 - 1, gY0 = y0 + r0 - 1;
    const float fr0 = (float)r0;
    double dS = 0.0, dT = 0.0;
    // intensity tile of frame f (clamped reads) copied asynchronously into dst: the next frame's
    // tile lands in the other buffer while this frame's taps run
    auto prefetch = [&](int f, float* dst) {
        const float* fr = g.I + (long)f * wh;
        for (int ly = ty; ly < IH; ly += kTYT) {
            const long grow = (long)min(max(gY0 + ly, 0), H - 1) * W;
            for (int lx = tx; lx < IW; lx += kTX) cp_async4z(dst + ly * IW + lx, fr + grow + min(max(gX0 + lx, 0), W - 1), true);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // frames [fb, fe) of the launch (several groups across CTAs where the tiles alone would leave
    // the last wave of CTAs short; every frame is independent here)
    const int fb = (int)((long long)g.F * blockIdx.z / gridDim.z);
    const int fe = (int)((long long)g.F * (blockIdx.z + 1) / gridDim.z);
    if (fe > fb) prefetch(fb, sIb + (fb & 1) * kIS);
    for (int f = fb; f < fe; ++f) {
        float* sI = sIb + (f & 1) * kIS;
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();  // frame f's tile landed; every thread is done with frame f - 1's buffer
        if (f + 1 < fe) prefetch(f + 1, sIb + ((f + 1) & 1) * kIS);
        for (int ey = ty; ey < EH; ey += kTYT) {
            const int Y = y0 + r0 + ey;
            const bool yin = Y >= 0 && Y < H;
            const int ya0 = max(Y - 1, 0), yb = min(Y + 1, H - 1), yb0 = max(yb - 1, 0);
            for (int ex = tx; ex < EW; ex += kTX) {
                const int X = x0 + r0 + ex;
                float2 e = make_float2(0.f, 0.f);
                if (yin && X >= 0 && X < W) {
                    const int xa = min(X + 1, W - 1), xa0 = max(xa - 1, 0), xb0 = max(X - 1, 0);
                    const float Gx = sI[(ya0 - gY0) * IW + (xa - gX0)] - sI[(Y - gY0) * IW + (xa0 - gX0)] +
                                     sI[(Y - gY0) * IW + (xa - gX0)] - sI[(ya0 - gY0) * IW + (xa0 - gX0)];
                    const float Gy = -sI[(yb0 - gY0) * IW + (X - gX0)] + sI[(yb - gY0) * IW + (xb0 - gX0)] +
                                     sI[(yb - gY0) * IW + (X - gX0)] - sI[(yb0 - gY0) * IW + (xb0 - gX0)];
                    const float n2 = Gx * Gx + Gy * Gy;
                    if (n2 > 0.f) {
                        const float inv = rsqrtf(n2);
                        e = make_float2(Gx * inv, Gy * inv);
                    }
                }
                sE[ey * EW + ex] = e;
            }
        }
        __syncthreads();
        float acc[kK], acc2[kK];
#pragma unroll
        for (int k = 0; k < kK; ++k) acc[k] = acc2[k] = 0.f;
        for (int ii = 0; ii < S; ++ii) {
            const int lo = __ldg(g.jr + 2 * ii), hi = __ldg(g.jr + 2 * ii + 1);
            if (lo > hi) continue;  // no tap of the disc in this column
            const float fi = fr0 + (float)ii;
            float w[S], wd[S], before[kK];
#pragma unroll
            for (int jj = 0; jj < S; ++jj) {
                const float4 t = stab[ii * S + jj];
                w[jj] = t.x;
                wd[jj] = t.y;
            }
#pragma unroll
            for (int k = 0; k < kK; ++k) before[k] = acc[k];
            const float2* col = sE + (ty * kK) * EW + tx + ii;
            if (lo == 0 && hi == S - 1)
                chord_a<S, 0, S - 1>(col, fi, w, wd, acc, acc2);
            else
                dispatch_a<S, 0>(col, fi, lo, hi, w, wd, acc, acc2);
            // d^2 = i^2 + j^2: the column's i^2 times its inward sum
#pragma unroll
            for (int k = 0; k < kK; ++k) acc2[k] = fmaf(fi * fi, acc[k] - before[k], acc2[k]);
        }
        if (g.c_out) {
#pragma unroll
            for (int k = 0; k < kK; ++k) {
                const int yM = y0 + ty * kK + k;
                if (xM >= W || yM >= H) continue;
                const long pix = (long)yM * W + xM;
                g.c_out[(long)f * wh + pix] = acc[k] / __ldg(g.wsum + pix);
                g.q_out[(long)f * wh + pix] = acc2[k];
            }
            continue;
        }
#pragma unroll
        for (int k = 0; k < kK; ++k) {
            const int yM = y0 + ty * kK + k;
            if (xM >= W || yM >= H) continue;
            const long pix = (long)yM * W + xM;
            const float v = sI[(ty * kK + k + 1 - r0) * IW + (tx + 1 - r0)];
            const float ws = __ldg(g.wsum + pix), av = __ldg(g.a + pix);
            const float C = acc[k] / ws;
            float Cs = 0.f, dC = 0.f, b = 0.f;
            if (C > 0.f && C < INFINITY) {
                const float lc = logf(C);
                Cs = expf(g.sens * lc);
                dC = av * v * g.sens * Cs / C;
                b = dC / ws;
                dS += (double)av * v * Cs * lc;
                dT += (double)b * (acc2[k] * g.kscale - C * __ldg(g.dwsum + pix));
            }
            g.gI[(long)f * wh + pix] = av * Cs;
            g.b[(long)f * wh + pix] = b;
        }
    }
    // block reduction of the two parameter partials
    __shared__ double red[2][8];
    for (int o = 16; o > 0; o >>= 1) {
        dS += __shfl_xor_sync(0xffffffffu, dS, o);
        dT += __shfl_xor_sync(0xffffffffu, dT, o);
    }
    if (tx == 0) {
        red[0][ty] = dS;
        red[1][ty] = dT;
    }
    __syncthreads();
    if (tid == 0 && g.acc) {  // (none in the emit form)
        double s0 = 0, s1 = 0;
        for (int i = 0; i < kTYT; ++i) {
            s0 += red[0][i];
            s1 += red[1][i];
        }
        atomicAdd(g.acc, s0);
        atomicAdd(g.acc + 1, s1);
    }
}

template <int S>
struct AdjBLayout {
    static constexpr int BW = kTX + S - 1, BH = kTH + S - 1;  // dL/dN tile, origin (x0-r1, y0-r1)
    static constexpr int IW = kTX + 2, IH = kTH + 2;          // intensity around the sources
    static constexpr size_t B_bytes = (sizeof(float) * BW * BH + 15) & ~size_t(15);
    static constexpr size_t I_bytes = (sizeof(float) * IW * IH + 15) & ~size_t(15);
    static constexpr size_t off_B = 0;                  // 2 buffers
    static constexpr size_t off_I = off_B + 2 * B_bytes;  // 2 buffers
    static constexpr size_t off_wd = off_I + 2 * I_bytes;
    static constexpr size_t bytes = off_wd + sizeof(float) * S * S;
};

struct AdjBArgs {
    const float* I;     // [F][H][W]
    const float* b;     // [F][H][W]
    const float* wdB;   // [ii'][jj'] = w/d of tap (r1 - ii', r1 - jj')
    const int* jr;      // [S][2] disc chord of each tap column, kernel A's (forward) order
    int W, H, F, r1;
    float* gI;          // [F][H][W], accumulated atomically
};

// One column ii' of kernel B's gather over its chord of tap rows [LO, HI] (jj' = r1 - t_y).
template <int S, int LO, int HI>
__device__ __forceinline__ void chord_b(const float* __restrict__ col, float tx_f, const float (&wd)[S],
                                        const float (&gx)[kK], const float (&gy)[kK], const float (&Ak)[kK],
                                        const float (&Bk)[kK], float (&Sx)[kK], float (&Tx)[kK],
                                        float (&Sy)[kK]) {
    constexpr int BW = AdjBLayout<S>::BW;
#pragma unroll
    for (int rr = LO; rr <= HI + kK - 1; ++rr) {
        const float bv = col[rr * BW];
#pragma unroll
        for (int k = 0; k < kK; ++k) {
            const int jj = rr - k;  // t_y = r1 - jj = r1 + k - rr
            if (jj >= LO && jj <= HI) {
                const float dot = fmaf(-gy[k], (float)rr, Ak[k]);
                const float c = fmaf(gx[k], (float)rr, Bk[k]);
                if (dot < 0.f) {
                    // (w/d) b sgn(c): flip the sign bit of (w/d) b by that of c
                    const float sv = __int_as_float(__float_as_int(wd[jj] * bv) ^
                                                    (__float_as_int(c) & 0x80000000));
                    Sx[k] += sv;
                    Tx[k] = fmaf(sv, (float)rr, Tx[k]);  // Sy gets t_x times the column's sum of sv
                }
            }
        }
    }
}

// Kernel B's column ii' is the forward column S - 1 - ii' read from the other end, so its
// chords are the whole box or tap rows [LO + 1, S - 1 - LO]; any other shape takes the box.
template <int S, int LO>
__device__ __forceinline__ void dispatch_b(const float* __restrict__ col, float tx_f, int lo, int hi,
                                           const float (&wd)[S], const float (&gx)[kK], const float (&gy)[kK],
                                           const float (&Ak)[kK], const float (&Bk)[kK], float (&Sx)[kK],
                                           float (&Tx)[kK], float (&Sy)[kK]) {
    if constexpr (LO <= (S - 2) / 2) {
        if (lo == LO + 1 && hi == S - 1 - LO) {
            chord_b<S, LO + 1, S - 1 - LO>(col, tx_f, wd, gx, gy, Ak, Bk, Sx, Tx, Sy);
            return;
        }
        dispatch_b<S, LO + 1>(col, tx_f, lo, hi, wd, gx, gy, Ak, Bk, Sx, Tx, Sy);
    } else {
        chord_b<S, 0, S - 1>(col, tx_f, wd, gx, gy, Ak, Bk, Sx, Tx, Sy);  // zero w/d off the disc
    }
}

// Kernel B: per tap source, gather over the taps of the outputs it feeds.
template <int S>
__global__ void __launch_bounds__(256, 2) adj_b_kernel(AdjBArgs g) {
    using L = AdjBLayout<S>;
    constexpr int BW = L::BW, BH = L::BH, IW = L::IW, IH = L::IH;
    extern __shared__ __align__(16) unsigned char smem[];
    float* sBb = reinterpret_cast<float*>(smem + L::off_B);
    float* sIb = reinterpret_cast<float*>(smem + L::off_I);
    float* swd = reinterpret_cast<float*>(smem + L::off_wd);
    constexpr int kBS = (int)(L::B_bytes / sizeof(float)), kIS = (int)(L::I_bytes / sizeof(float));
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTH, r1 = g.r1;
    const int W = g.W, H = g.H;
    const long wh = (long)W * H;
    for (int i = tid; i < S * S; i += blockDim.x) swd[i] = g.wdB[i];
    const int X = x0 + tx;
    const float fr1 = (float)r1;
    // dL/dN tile (zero outside the image) and intensity tile (clamped reads) of frame f copied
    // asynchronously into buffer f & 1 while the previous frame's taps run
    auto prefetch = [&](int f) {
        const float* fr = g.I + (long)f * wh;
        const float* bf = g.b + (long)f * wh;
        float* dB = sBb + (f & 1) * kBS;
        float* dI = sIb + (f & 1) * kIS;
        for (int ly = ty; ly < BH; ly += kTYT) {
            const int q_y = y0 - r1 + ly;
            for (int lx = tx; lx < BW; lx += kTX) {
                const int q_x = x0 - r1 + lx;
                const bool in = q_x >= 0 && q_x < W && q_y >= 0 && q_y < H;
                cp_async4z(dB + ly * BW + lx, in ? bf + (long)q_y * W + q_x : bf, in);
            }
        }
        for (int ly = ty; ly < IH; ly += kTYT) {
            const long grow = (long)min(max(y0 - 1 + ly, 0), H - 1) * W;
            for (int lx = tx; lx < IW; lx += kTX) cp_async4z(dI + ly * IW + lx, fr + grow + min(max(x0 - 1 + lx, 0), W - 1), true);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // frames [fb, fe) of the launch, as in kernel A
    const int fb = (int)((long long)g.F * blockIdx.z / gridDim.z);
    const int fe = (int)((long long)g.F * (blockIdx.z + 1) / gridDim.z);
    if (fe > fb) prefetch(fb);
    for (int f = fb; f < fe; ++f) {
        const float* sB = sBb + (f & 1) * kBS;
        const float* sI = sIb + (f & 1) * kIS;
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();  // frame f's tiles landed; every thread is done with frame f - 1's buffers
        if (f + 1 < fe) prefetch(f + 1);
        // unit gradient at this thread's 8 sources
        float gx[kK], gy[kK], inv[kK];
#pragma unroll
        for (int k = 0; k < kK; ++k) {
            const int Y = y0 + ty * kK + k;
            gx[k] = gy[k] = inv[k] = 0.f;
            if (X < W && Y < H) {
                const int xa = min(X + 1, W - 1), xa0 = max(xa - 1, 0), ya0 = max(Y - 1, 0);
                const int yb = min(Y + 1, H - 1), yb0 = max(yb - 1, 0), xb0 = max(X - 1, 0);
                const int ox = x0 - 1, oy = y0 - 1;
                const float Gx = sI[(ya0 - oy) * IW + (xa - ox)] - sI[(Y - oy) * IW + (xa0 - ox)] +
                                 sI[(Y - oy) * IW + (xa - ox)] - sI[(ya0 - oy) * IW + (xa0 - ox)];
                const float Gy = -sI[(yb0 - oy) * IW + (X - ox)] + sI[(yb - oy) * IW + (xb0 - ox)] +
                                 sI[(yb - oy) * IW + (X - ox)] - sI[(yb0 - oy) * IW + (xb0 - ox)];
                const float n2 = Gx * Gx + Gy * Gy;
                if (n2 > 0.f) {
                    inv[k] = rsqrtf(n2);
                    gx[k] = Gx * inv[k];
                    gy[k] = Gy * inv[k];
                }
            }
        }
        float Sx[kK], Tx[kK], Sy[kK];
#pragma unroll
        for (int k = 0; k < kK; ++k) Sx[k] = Tx[k] = Sy[k] = 0.f;
        for (int ii = 0; ii < S; ++ii) {   // ii' : t_x = r1 - ii'
            // forward column S - 1 - ii', rows reflected
            const int lof = __ldg(g.jr + 2 * (S - 1 - ii)), hif = __ldg(g.jr + 2 * (S - 1 - ii) + 1);
            if (lof > hif) continue;  // no tap of the disc in this column
            const int lo = S - 1 - hif, hi = S - 1 - lof;
            const float tx_f = fr1 - (float)ii;
            float wd[S];
#pragma unroll
            for (int jj = 0; jj < S; ++jj) wd[jj] = swd[ii * S + jj];
            float Ak[kK], Bk[kK];
#pragma unroll
            for (int k = 0; k < kK; ++k) {
                Ak[k] = fmaf(gx[k], tx_f, gy[k] * (fr1 + (float)k));
                Bk[k] = fmaf(gy[k], tx_f, -gx[k] * (fr1 + (float)k));
            }
            const float* col = sB + (ty * kK) * BW + tx + ii;
            float before[kK];
#pragma unroll
            for (int k = 0; k < kK; ++k) before[k] = Sx[k];
            if (lo == 0 && hi == S - 1)
                chord_b<S, 0, S - 1>(col, tx_f, wd, gx, gy, Ak, Bk, Sx, Tx, Sy);
            else
                dispatch_b<S, 0>(col, tx_f, lo, hi, wd, gx, gy, Ak, Bk, Sx, Tx, Sy);
            // t_x is the column's constant: Sy = sum sv t_x gains t_x (column sum of sv)
#pragma unroll
            for (int k = 0; k < kK; ++k) Sy[k] = fmaf(tx_f, Sx[k] - before[k], Sy[k]);
        }
        // project onto the tangent of the unit vector and scatter through the Roberts cross
#pragma unroll
        for (int k = 0; k < kK; ++k) {
            const int Y = y0 + ty * kK + k;
            if (X >= W || Y >= H || inv[k] == 0.f) continue;
            const float dgx = (fr1 + (float)k) * Sx[k] - Tx[k];
            const float dgy = -Sy[k];
            const float pd = gx[k] * dgx + gy[k] * dgy;
            const float dEx = (dgx - gx[k] * pd) * inv[k];
            const float dEy = (dgy - gy[k] * pd) * inv[k];
            float* gf = g.gI + (long)f * wh;
            const int xa = min(X + 1, W - 1), xa0 = max(xa - 1, 0), ya0 = max(Y - 1, 0);
            atomicAdd(gf + (long)ya0 * W + xa, dEx);
            atomicAdd(gf + (long)Y * W + xa0, -dEx);
            atomicAdd(gf + (long)Y * W + xa, dEx);
            atomicAdd(gf + (long)ya0 * W + xa0, -dEx);
            const int yb = min(Y + 1, H - 1), yb0 = max(yb - 1, 0), xb0 = max(X - 1, 0);
            atomicAdd(gf + (long)yb0 * W + X, -dEy);
            atomicAdd(gf + (long)yb * W + xb0, dEy);
            atomicAdd(gf + (long)yb * W + X, dEy);
            atomicAdd(gf + (long)yb0 * W + xb0, -dEy);
        }
    }
}

// Kernel A's per-pixel terms from the forward's planes (kernel A in its emit form wrote C and the
// d^2-weighted tap sum Q of every frame, so the backward pass needs no second tap loop): the same
// arithmetic as kernel A's epilogue, over the F frames of a chunk, grid-stride over (frame, pixel).
struct AdjTailArgs {
    const float* I;      // [F][P] interpolated frames of the chunk
    const float* C;      // [F][P] CGLH / sum of weights
    const float* Q;      // [F][P] sum over the inward taps of d^2 (w - (w/d) |c|)
    const float* a;      // [P] dL/dR / T
    const float* wsum;   // [P]
    const float* dwsum;  // [P] d(sum of weights)/dtSS
    long P;
    int F;
    float kscale, sens;
    float* b;            // [F][P] dL/dN
    float* gI;           // [F][P] the intensity-weighting term of dL/dI
    double* acc;         // [2]: dL/dS, dL/dtSS
};

__global__ void __launch_bounds__(256) adj_tail_kernel(AdjTailArgs g) {
    double dS = 0.0, dT = 0.0;
    const long n = g.P * g.F;
    for (long o = (long)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (long)gridDim.x * blockDim.x) {
        const long pix = o % g.P;
        const float v = g.I[o], C = g.C[o];
        const float ws = __ldg(g.wsum + pix), av = __ldg(g.a + pix);
        float Cs = 0.f, b = 0.f;
        if (C > 0.f && C < INFINITY) {
            const float lc = logf(C);
            Cs = expf(g.sens * lc);
            const float dC = av * v * g.sens * Cs / C;
            b = dC / ws;
            dS += (double)av * v * Cs * lc;
            dT += (double)b * (g.Q[o] * g.kscale - C * __ldg(g.dwsum + pix));
        }
        g.gI[o] = av * Cs;
        g.b[o] = b;
    }
    __shared__ double red[2][8];
    for (int s = 16; s > 0; s >>= 1) {
        dS += __shfl_xor_sync(0xffffffffu, dS, s);
        dT += __shfl_xor_sync(0xffffffffu, dT, s);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        red[0][warp] = dS;
        red[1][warp] = dT;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0;
        for (int i = 0; i < 8; ++i) {
            s0 += red[0][i];
            s1 += red[1][i];
        }
        atomicAdd(g.acc, s0);
        atomicAdd(g.acc + 1, s1);
    }
}

// ---- loss side ---------------------------------------------------------------------------------
struct Gauss {
    int r;
    float k[kMaxGauss];
};

__global__ void frame_mean_kernel(const float* __restrict__ raw, int T, long P, float* __restrict__ Fm) {
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    double s = 0;
    for (int t = 0; t < T; ++t) s += raw[(long)t * P + p];
    Fm[p] = (float)(s / T);
}

// R = (1/T) sum_t I_t pow(C_t, S), C <= 0 or NaN contributes 0.
__global__ void recon_kernel(const float* __restrict__ I, const float* __restrict__ C, int T, long P,
                             float sens, float* __restrict__ R) {
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    double s = 0;
    for (int t = 0; t < T; ++t) {
        const float c = C[(long)t * P + p];
        if (c > 0.f && c < INFINITY) s += (double)I[(long)t * P + p] * expf(sens * logf(c));
    }
    R[p] = (float)(s / T);
}

// separable zero-padded convolution along x (dir 0) or y (dir 1)
__global__ void blur1d_kernel(const float* __restrict__ in, int W, int H, int dir, Gauss g,
                              float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    float s = 0.f;
    for (int u = -g.r; u <= g.r; ++u) {
        const int xx = dir == 0 ? x + u : x, yy = dir == 0 ? y : y + u;
        if (xx >= 0 && xx < W && yy >= 0 && yy < H) s = fmaf(g.k[u + g.r], in[(long)yy * W + xx], s);
    }
    out[(long)y * W + x] = s;
}

__global__ void downsample_stats_kernel(const float* __restrict__ B, int w, int h, int M,
                                        const float* __restrict__ Fm, float* __restrict__ D,
                                        double* __restrict__ stats) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    double d = 0, f = 0;
    if (x < w) {
        const int WM = w * M;
        for (int a = 0; a < M; ++a)
            for (int c = 0; c < M; ++c) d += B[(long)(y * M + a) * WM + x * M + c];
        d /= (double)(M * M);
        f = Fm[(long)y * w + x];
        D[(long)y * w + x] = (float)d;
    }
    double v[5] = {d, f, d * d, d * f, f * f};
    for (int i = 0; i < 5; ++i) {
        double t = v[i];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(stats + i, t);
    }
}

// residual r = alpha D + beta - F: gD (upsampled, / M^2) into gB, dL/dF into dF
__global__ void residual_kernel(const float* __restrict__ D, const float* __restrict__ Fm, int w,
                                int h, int M, double alpha, double beta, float* __restrict__ gB,
                                float* __restrict__ dF) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y;
    const int WM = w * M;
    if (X >= WM) return;
    const int x = X / M, y = Y / M;
    const double r = alpha * D[(long)y * w + x] + beta - Fm[(long)y * w + x];
    const double n = (double)w * h;
    gB[(long)Y * WM + X] = (float)(2.0 * alpha * r / n / (M * M));
    if (X % M == 0 && Y % M == 0) dF[(long)y * w + x] = (float)(-2.0 * r / n);
}

__global__ void dot_kernel(const float* __restrict__ a, const float* __restrict__ b1,
                           const float* __restrict__ b2, long P, double* __restrict__ out) {
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double t = p < P ? (double)a[p] * ((double)b1[p] + (double)b2[p]) : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, t);
}

__global__ void scale_kernel(float* __restrict__ x, long P, float s) {
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < P) x[p] *= s;
}

// graw[f] = dF / T (the frame-average term), before the interpolation adjoint adds L^T gI.
__global__ void init_graw_kernel(const float* __restrict__ dF, long P, int F, float invT,
                                 float* __restrict__ graw) {
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P * F) return;
    graw[p] = dF[p % P] * invT;
}

__global__ void transpose_kernel(const float* __restrict__ in, int rows, int cols, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
    if (c < cols) out[(long)c * rows + r] = in[(long)r * cols + c];
}

// Frame groups (gridDim.z) for a launch of `tiles` CTAs over F independent frames: the smallest
// count, up to 8 and at most F / 2 (two frames per group keep the tile prefetch useful), whose CTAs
// fill the waves of `slots` resident CTAs within 2 % of the best count (1024 x 1024 outputs: 512
// tiles on 296 slots are 1.73 waves, 87 % filled; four groups make 6.92 waves, 99 %).
int frame_groups(int tiles, int F, int slots) {
    const int gmax = std::max(1, std::min(8, F / 2));
    auto fill = [&](int g) {
        const double waves = (double)tiles * g / std::max(1, slots);
        return waves / std::ceil(waves);
    };
    double best = 0;
    for (int g = 1; g <= gmax; ++g) best = std::max(best, fill(g));
    for (int g = 1; g <= gmax; ++g)
        if (fill(g) >= best - 0.02) return g;
    return 1;
}

template <int S>
cudaError_t launch_adj(const AdjAArgs& a, AdjBArgs b, bool backward_b, cudaStream_t st) {
    static unsigned long long done_a = 0, done_b = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    const int tiles = backward_b ? ((b.W + kTX - 1) / kTX) * ((b.H + kTH - 1) / kTH)
                                 : ((a.W + kTX - 1) / kTX) * ((a.H + kTH - 1) / kTH);
    const unsigned groups = (unsigned)frame_groups(tiles, backward_b ? b.F : a.F, 2 * sm_count(dev));
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0;
    cudaError_t e;
    if (!backward_b) {
        if (!(done_a & bit)) {
            if ((e = cudaFuncSetAttribute(adj_a_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)AdjLayout<S>::bytes)) != cudaSuccess)
                return e;
            done_a |= bit;
        }
        adj_a_kernel<S><<<dim3((a.W + kTX - 1) / kTX, (a.H + kTH - 1) / kTH, groups), 256, AdjLayout<S>::bytes, st>>>(a);
    } else {
        if (!(done_b & bit)) {
            if ((e = cudaFuncSetAttribute(adj_b_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)AdjBLayout<S>::bytes)) != cudaSuccess)
                return e;
            done_b |= bit;
        }
        adj_b_kernel<S><<<dim3((b.W + kTX - 1) / kTX, (b.H + kTH - 1) / kTH, groups), 256, AdjBLayout<S>::bytes, st>>>(b);
    }
    return cudaGetLastError();
}

cudaError_t launch_adj_any(int S, const AdjAArgs& a, const AdjBArgs& b, bool backward_b, cudaStream_t st) {
    switch (S) {
        case 6: return launch_adj<6>(a, b, backward_b, st);
        case 8: return launch_adj<8>(a, b, backward_b, st);
        case 10: return launch_adj<10>(a, b, backward_b, st);
        case 12: return launch_adj<12>(a, b, backward_b, st);
        case 14: return launch_adj<14>(a, b, backward_b, st);
        case 16: return launch_adj<16>(a, b, backward_b, st);
        case 18: return launch_adj<18>(a, b, backward_b, st);
        case 20: return launch_adj<20>(a, b, backward_b, st);
        case 22: return launch_adj<22>(a, b, backward_b, st);
        case 24: return launch_adj<24>(a, b, backward_b, st);
        case 26: return launch_adj<26>(a, b, backward_b, st);
        default: return cudaErrorInvalidValue;
    }
}

Gauss make_gauss(double sigma, bool derivative) {
    // normalised sampled Gaussian, radius ceil(4 sigma); derivative: d/dsigma of the normalised
    // kernel, k (u^2 - sum_u k u^2) / sigma^3
    Gauss g{};
    g.r = (int)std::ceil(4.0 * sigma);
    std::vector<double> k(2 * g.r + 1);
    double z = 0, m2 = 0;
    for (int u = -g.r; u <= g.r; ++u) z += (k[u + g.r] = std::exp(-(double)u * u / (2 * sigma * sigma)));
    for (int u = -g.r; u <= g.r; ++u) m2 += (k[u + g.r] /= z) * u * u;
    for (int u = -g.r; u <= g.r; ++u)
        g.k[u + g.r] = (float)(derivative ? k[u + g.r] * ((double)u * u - m2) / (sigma * sigma * sigma)
                                          : k[u + g.r]);
    return g;
}

}  // namespace

struct esrrf_adjoint {
    int w = 0, h = 0, T = 0, M = 0, device = -1, Fc = 8;
    int WM = 0, HM = 0;
    cudaStream_t stream = nullptr;
    InterpPlan plan;
    InterpScratch scratch;
    float* dx = nullptr;               // Dx row-major [WM][N]
    float cur_fwhm = -1.f;
    FhtGeometry geo;
    FhtFusedTables tables;
    float4* tabA = nullptr;            // [S][S]
    float* wdB = nullptr;              // [S][S]
    float* kwtab = nullptr;            // [S][S] kappa * w (for d sum w / dtSS)
    float* dwsum = nullptr;            // [HM][WM]
    float *I = nullptr, *C = nullptr;  // [T][HM][WM]
    float* Q = nullptr;                // [T][HM][WM] d^2-weighted inward tap sums (gradient forward)
    bool q_valid = false;              // C and Q come from a gradient forward at the current radius
    float *R = nullptr, *tmp = nullptr, *Bb = nullptr, *gB = nullptr, *gR = nullptr, *t1 = nullptr, *t2 = nullptr;
    float *Fm = nullptr, *D = nullptr, *dF = nullptr;  // [h][w]
    float *bbuf = nullptr, *gI = nullptr;              // [Fc][HM][WM]
    float *T1 = nullptr, *gX = nullptr, *proj = nullptr, *dvec = nullptr;
    float* graw_tmp = nullptr;         // [T][h][w] when the caller passes no gradient buffer
    double* dstat = nullptr;           // [8]: stats(5), dS, dtSS, dsigma
    double alpha = 0, beta = 0;
    std::string err;

    esrrf_status fail(esrrf_status s, const std::string& m) {
        err = m;
        return s;
    }
    esrrf_status fail_cuda(cudaError_t e, const char* what) {
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? ESRRF_ERR_NOMEM : ESRRF_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorName(e));
    }
    esrrf_status set_radius(float fwhm);
    esrrf_status forward(const float* frames, float fwhm, float sens, float sigma_b, double* loss,
                         bool for_grad = false);
    esrrf_status backward(const float* frames, float fwhm, float sens, float sigma_b, double* grads,
                          float* graw);
    void release();
};

#define AK(call, what)                                         \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return fail_cuda(_e, what);     \
    } while (0)

esrrf_status esrrf_adjoint::set_radius(float fwhm) {
    if (fwhm == cur_fwhm) return ESRRF_OK;
    fht_fused_tables_free(tables);
    cudaFree(tabA);
    cudaFree(wdB);
    cudaFree(kwtab);
    tabA = nullptr;
    wdB = kwtab = nullptr;
    geo = fht_geometry(M, fwhm, 1);
    if (!fht_fused_supported(geo) || geo.S < 6 || geo.S > 26)
        return fail(ESRRF_ERR_INVALID, "radius gives a tap box outside 6..26 pixels for the adjoint");
    AK(fht_fused_tables(geo, WM, HM, tables, stream), "RGC tables");
    const int S = geo.S;
    std::vector<float4> ta(S * S);
    std::vector<float> wb(S * S), kw(S * S);
    const double tSS = geo.tSS;
    for (int jj = 0; jj < S; ++jj)
        for (int ii = 0; ii < S; ++ii) {
            const int i = geo.r0 + ii, j = geo.r0 + jj;
            const float w = geo.w[jj * S + ii], wd = geo.wd[jj * S + ii];
            const double d2 = (double)i * i + (double)j * j;
            const float kap = (float)(4.0 * d2 / (tSS * tSS));
            ta[ii * S + jj] = make_float4(w, wd, kap, 0.f);
            kw[jj * S + ii] = kap * w;
            // kernel B's order: tap (r1 - ii', r1 - jj') at [ii'][jj']
            const int iip = geo.r1 - i, jjp = geo.r1 - j;
            wb[iip * S + jjp] = wd;
        }
    AK(cudaMalloc(&tabA, sizeof(float4) * S * S), "tables");
    AK(cudaMalloc(&wdB, sizeof(float) * S * S), "tables");
    AK(cudaMalloc(&kwtab, sizeof(float) * S * S), "tables");
    AK(cudaMemcpy(tabA, ta.data(), sizeof(float4) * S * S, cudaMemcpyHostToDevice), "tables");
    AK(cudaMemcpy(wdB, wb.data(), sizeof(float) * S * S, cudaMemcpyHostToDevice), "tables");
    AK(cudaMemcpy(kwtab, kw.data(), sizeof(float) * S * S, cudaMemcpyHostToDevice), "tables");
    AK(tap_table_sum(kwtab, geo.r0, S, WM, HM, dwsum, stream), "dwsum");
    AK(cudaStreamSynchronize(stream), "tables");
    cur_fwhm = fwhm;
    return ESRRF_OK;
}

esrrf_status esrrf_adjoint::forward(const float* frames, float fwhm, float sens, float sigma_b, double* loss,
                                    bool for_grad) {
    esrrf_status r = set_radius(fwhm);
    if (r != ESRRF_OK) return r;
    if (!(sigma_b > 0.f) || 4.0 * sigma_b > (kMaxGauss - 1) / 2) return fail(ESRRF_ERR_INVALID, "sigma out of range");
    if (!(sens >= 0.f) || sens > 64.f) return fail(ESRRF_ERR_INVALID, "sensitivity must be in [0, 64]");
    const long P = (long)WM * HM, p = (long)w * h;
    frame_mean_kernel<<<(unsigned)((p + 255) / 256), 256, 0, stream>>>(frames, T, p, Fm);
    for (int t = 0; t < T; t += Fc) {
        const int n = std::min(Fc, T - t);
        AK(interp_run(plan, scratch, frames + (size_t)t * w * h, false, n, I + (size_t)t * P, stream, nullptr),
           "interpolation");
    }
    q_valid = false;
    if (for_grad) {
        // the backward pass needs, besides C, each pixel's d^2-weighted tap sum: kernel A's tap
        // loop produces both in one pass, so the backward pass has no second tap loop
        AdjAArgs A{};
        A.I = I;
        A.tab = tabA;
        A.wsum = tables.wsum;
        A.jr = tables.jrange;
        A.W = WM;
        A.H = HM;
        A.F = T;
        A.r0 = geo.r0;
        A.c_out = C;
        A.q_out = Q;
        AdjBArgs B{};
        AK(launch_adj_any(geo.S, A, B, false, stream), "RGC with tap sums");
        q_valid = true;
    } else {
        FhtRgcArgs a{};
        a.interp = I;
        a.W = WM;
        a.H = HM;
        a.F = T;
        a.int_weighting = 1;
        a.cg_out = C;
        AK(fht_rgc_fused(geo, tables, a, stream), "RGC");
    }
    recon_kernel<<<(unsigned)((P + 255) / 256), 256, 0, stream>>>(I, C, T, P, sens, R);
    const Gauss g = make_gauss(sigma_b, false);
    blur1d_kernel<<<dim3((WM + 127) / 128, HM), 128, 0, stream>>>(R, WM, HM, 0, g, tmp);
    blur1d_kernel<<<dim3((WM + 127) / 128, HM), 128, 0, stream>>>(tmp, WM, HM, 1, g, Bb);
    AK(cudaMemsetAsync(dstat, 0, sizeof(double) * 8, stream), "memset");
    downsample_stats_kernel<<<dim3((w + 127) / 128, h), 128, 0, stream>>>(Bb, w, h, M, Fm, D, dstat);
    double st[5];
    AK(cudaMemcpyAsync(st, dstat, sizeof(double) * 5, cudaMemcpyDeviceToHost, stream), "stats");
    AK(cudaStreamSynchronize(stream), "forward");
    bool tc_failed = false;
    AK(interp_tc_check(plan, stream, &tc_failed), "interpolation status");
    if (tc_failed) return fail(ESRRF_ERR_TIMEOUT, "interpolation tensor-core pass: a bounded wait gave up");
    const double n = (double)p;
    const double md = st[0] / n, mf = st[1] / n;
    const double vdd = st[2] / n - md * md, vdf = st[3] / n - md * mf;
    alpha = vdd > 0 ? vdf / vdd : 0.0;
    beta = mf - alpha * md;
    // mean((alpha d + beta - f)^2) expanded in the sums
    const double L = (alpha * alpha * st[2] + beta * beta * n + st[4] + 2 * alpha * beta * st[0] -
                      2 * alpha * st[3] - 2 * beta * st[1]) / n;
    if (loss) *loss = L;
    return ESRRF_OK;
}

esrrf_status esrrf_adjoint::backward(const float* frames, float fwhm, float sens, float sigma_b,
                                     double* grads, float* graw) {
    const long P = (long)WM * HM, p = (long)w * h;
    residual_kernel<<<dim3((WM + 127) / 128, HM), 128, 0, stream>>>(D, Fm, w, h, M, alpha, beta, gB, dF);
    const Gauss g = make_gauss(sigma_b, false), dg = make_gauss(sigma_b, true);
    // dL/dR = G^T gB (symmetric kernel, zero padding)
    blur1d_kernel<<<dim3((WM + 127) / 128, HM), 128, 0, stream>>>(gB, WM, HM, 0, g, t1);
    blur1d_kernel<<<dim3((WM + 127) / 128, HM), 128, 0, stream>>>(t1, WM, HM, 1, g, gR);
    // dL/dsigma = <gB, (dG/dsigma) * R>
    blur1d_kernel<<<dim3((WM + 127) / 128, HM), 128, 0, stream>>>(R, WM, HM, 0, dg, t1);
    blur1d_kernel<<<dim3((WM + 127) / 128, HM), 128, 0, stream>>>(t1, WM, HM, 1, g, t2);
    blur1d_kernel<<<dim3((WM + 127) / 128, HM), 128, 0, stream>>>(tmp, WM, HM, 1, dg, t1);
    dot_kernel<<<(unsigned)((P + 255) / 256), 256, 0, stream>>>(gB, t1, t2, P, dstat + 7);
    scale_kernel<<<(unsigned)((P + 255) / 256), 256, 0, stream>>>(gR, P, 1.0f / T);
    float* out = graw ? graw : graw_tmp;
    for (int t = 0; t < T; t += Fc) {
        const int n = std::min(Fc, T - t);
        AdjAArgs A{};
        A.I = I + (size_t)t * P;
        A.a = gR;
        A.tab = tabA;
        A.wsum = tables.wsum;
        A.dwsum = dwsum;
        A.jr = tables.jrange;
        A.kscale = (float)(4.0 / ((double)geo.tSS * (double)geo.tSS));
        A.W = WM;
        A.H = HM;
        A.F = n;
        A.r0 = geo.r0;
        A.sens = sens;
        A.b = bbuf;
        A.gI = gI;
        A.acc = dstat + 5;
        AdjBArgs B{};
        B.I = A.I;
        B.b = bbuf;
        B.wdB = wdB;
        B.jr = tables.jrange;
        B.W = WM;
        B.H = HM;
        B.F = n;
        B.r1 = geo.r1;
        B.gI = gI;
        if (!q_valid) return fail(ESRRF_ERR_STATE, "the backward pass needs the gradient forward's tap sums");
        AdjTailArgs Tl{};
        Tl.I = A.I;
        Tl.C = C + (size_t)t * P;
        Tl.Q = Q + (size_t)t * P;
        Tl.a = gR;
        Tl.wsum = tables.wsum;
        Tl.dwsum = dwsum;
        Tl.P = P;
        Tl.F = n;
        Tl.kscale = A.kscale;
        Tl.sens = sens;
        Tl.b = bbuf;
        Tl.gI = gI;
        Tl.acc = dstat + 5;
        {
            int dev = 0, nsm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            const long blocks = std::min<long>((P * n + 255) / 256, 8L * std::max(nsm, 1));
            adj_tail_kernel<<<(unsigned)blocks, 256, 0, stream>>>(Tl);
        }
        AK(cudaGetLastError(), "adjoint A terms");
        AK(launch_adj_any(geo.S, A, B, true, stream), "adjoint B");
        float* gr = out + (size_t)t * p;
        init_graw_kernel<<<(unsigned)((p * n + 255) / 256), 256, 0, stream>>>(dF, p, n, 1.0f / T, gr);
        AK(interp_adjoint_run(plan, dx, gI, n, T1, gX, proj, dvec, gr, stream), "interpolation adjoint");
    }
    double st[3];
    AK(cudaMemcpyAsync(st, dstat + 5, sizeof(double) * 3, cudaMemcpyDeviceToHost, stream), "grads");
    AK(cudaStreamSynchronize(stream), "backward");
    const double sigma = (double)(fwhm / 2.354f);
    const double dtss_dfwhm = 4.0 * sigma * (double)M * M / 2.354;
    if (grads) {
        grads[0] = st[1] * dtss_dfwhm;  // radius (fwhm)
        grads[1] = st[0];               // sensitivity
        grads[2] = st[2];               // re-blur sigma
    }
    return ESRRF_OK;
}

void esrrf_adjoint::release() {
    if (device >= 0) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    interp_plan_destroy(plan);
    fht_fused_tables_free(tables);
    for (void* q : {(void*)scratch.rowT, (void*)scratch.xs, (void*)scratch.alt, (void*)scratch.vec, (void*)dx, (void*)tabA,
                    (void*)wdB, (void*)kwtab, (void*)dwsum, (void*)I, (void*)C, (void*)Q, (void*)R, (void*)tmp,
                    (void*)Bb, (void*)gB, (void*)gR, (void*)t1, (void*)t2, (void*)Fm, (void*)D, (void*)dF,
                    (void*)bbuf, (void*)gI, (void*)T1, (void*)gX, (void*)proj, (void*)dvec,
                    (void*)graw_tmp, (void*)dstat})
        cudaFree(q);
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
}

namespace {
std::mutex g_adj_mu;
std::string g_adj_error;
}  // namespace

extern "C" {

esrrf_status esrrf_adjoint_create(int width, int height, int n_frames, int magnification, int device,
                                  esrrf_adjoint** out) {
    if (!out) return ESRRF_ERR_INVALID;
    *out = nullptr;
    auto reject = [](const char* m) {
        std::lock_guard<std::mutex> lk(g_adj_mu);
        g_adj_error = m;
        return ESRRF_ERR_INVALID;
    };
    if (width < 4 || height < 4 || n_frames < 1) return reject("bad stack size");
    if (magnification < 1 || magnification > 16) return reject("magnification out of range");
    esrrf_adjoint* a = new esrrf_adjoint();
    a->w = width;
    a->h = height;
    a->T = n_frames;
    // frames per chunk of the passes: equal chunks of at most 32 (the transposed interpolation's
    // GEMMs have only 16 and 4 CTAs per frame at 256 x 256, M4, so fewer frames leave SMs idle)
    {
        const int chunks = (n_frames + 31) / 32;
        a->Fc = (n_frames + chunks - 1) / chunks;
    }
    a->M = magnification;
    a->device = device >= 0 ? device : 0;
    a->WM = width * magnification;
    a->HM = height * magnification;
    auto bail = [&](esrrf_status s) {
        {
            std::lock_guard<std::mutex> lk(g_adj_mu);
            g_adj_error = a->err;
        }
        a->release();
        delete a;
        return s;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(a->device)) != cudaSuccess) return bail(a->fail_cuda(e, "cudaSetDevice"));
    if ((e = cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(a->fail_cuda(e, "stream"));
    if ((e = interp_plan_create(a->plan, width, height, magnification, 0)) != cudaSuccess)
        return bail(a->fail_cuda(e, "interpolation plan"));
    const int N = a->plan.N, Fc = a->Fc;
    const long P = (long)a->WM * a->HM, p = (long)width * height;
    auto al = [&](auto** ptr, size_t bytes) { return cudaMalloc((void**)ptr, bytes); };
    if (a->plan.tc && (e = al(&a->scratch.xs, sizeof(float) * Fc * interp_xs_floats(a->plan))) != cudaSuccess)
        return bail(a->fail_cuda(e, "buffers"));
    if ((e = al(&a->scratch.rowT, sizeof(float) * Fc * interp_rowT_floats(a->plan))) != cudaSuccess ||
        (e = al(&a->scratch.alt, sizeof(float) * Fc * interp_alt_floats(N))) != cudaSuccess ||
        (e = al(&a->scratch.vec, sizeof(float) * Fc * interp_vec_floats(a->HM, a->WM))) != cudaSuccess ||
        (e = al(&a->dx, sizeof(float) * (size_t)a->WM * N)) != cudaSuccess ||
        (e = al(&a->dwsum, sizeof(float) * P)) != cudaSuccess ||
        (e = al(&a->I, sizeof(float) * P * n_frames)) != cudaSuccess ||
        (e = al(&a->C, sizeof(float) * P * n_frames)) != cudaSuccess ||
        (e = al(&a->Q, sizeof(float) * P * n_frames)) != cudaSuccess ||
        (e = al(&a->R, sizeof(float) * P)) != cudaSuccess || (e = al(&a->tmp, sizeof(float) * P)) != cudaSuccess ||
        (e = al(&a->Bb, sizeof(float) * P)) != cudaSuccess || (e = al(&a->gB, sizeof(float) * P)) != cudaSuccess ||
        (e = al(&a->gR, sizeof(float) * P)) != cudaSuccess || (e = al(&a->t1, sizeof(float) * P)) != cudaSuccess ||
        (e = al(&a->t2, sizeof(float) * P)) != cudaSuccess || (e = al(&a->Fm, sizeof(float) * p)) != cudaSuccess ||
        (e = al(&a->D, sizeof(float) * p)) != cudaSuccess || (e = al(&a->dF, sizeof(float) * p)) != cudaSuccess ||
        (e = al(&a->bbuf, sizeof(float) * P * Fc)) != cudaSuccess ||
        (e = al(&a->gI, sizeof(float) * P * Fc)) != cudaSuccess ||
        (e = al(&a->T1, sizeof(float) * Fc * (size_t)N * a->WM)) != cudaSuccess ||
        (e = al(&a->gX, sizeof(float) * Fc * (size_t)N * N)) != cudaSuccess ||
        (e = al(&a->proj, sizeof(float) * Fc * (size_t)(2 * a->HM + 2 * a->WM))) != cudaSuccess ||
        (e = al(&a->dvec, sizeof(float) * Fc * (size_t)(2 * N + 1))) != cudaSuccess ||
        (e = al(&a->graw_tmp, sizeof(float) * p * n_frames)) != cudaSuccess ||
        (e = al(&a->dstat, sizeof(double) * 8)) != cudaSuccess)
        return bail(a->fail_cuda(e, "adjoint buffers"));
    a->scratch.capacity = Fc;
    transpose_kernel<<<dim3((a->WM + 127) / 128, N), 128, 0, a->stream>>>(a->plan.dxT, N, a->WM, a->dx);
    if ((e = cudaStreamSynchronize(a->stream)) != cudaSuccess) return bail(a->fail_cuda(e, "set-up"));
    *out = a;
    return ESRRF_OK;
}

esrrf_status esrrf_adjoint_forward(esrrf_adjoint* a, const float* d_frames, float fwhm, float sensitivity,
                                   float sigma_b, double* loss) {
    if (!a || !d_frames) return ESRRF_ERR_INVALID;
    if (cudaSetDevice(a->device) != cudaSuccess) return a->fail(ESRRF_ERR_CUDA, "cudaSetDevice");
    return a->forward(d_frames, fwhm, sensitivity, sigma_b, loss);
}

esrrf_status esrrf_loss_and_grad(esrrf_adjoint* a, const float* d_frames, float fwhm, float sensitivity,
                                 float sigma_b, double* loss, double* grads, float* d_grad_frames) {
    if (!a || !d_frames) return ESRRF_ERR_INVALID;
    if (cudaSetDevice(a->device) != cudaSuccess) return a->fail(ESRRF_ERR_CUDA, "cudaSetDevice");
    esrrf_status r = a->forward(d_frames, fwhm, sensitivity, sigma_b, loss, true);
    if (r != ESRRF_OK) return r;
    return a->backward(d_frames, fwhm, sensitivity, sigma_b, grads, d_grad_frames);
}

const char* esrrf_adjoint_last_error(const esrrf_adjoint* a) {
    if (!a) {
        std::lock_guard<std::mutex> lk(g_adj_mu);
        return g_adj_error.c_str();
    }
    return a->err.c_str();
}

esrrf_status esrrf_adjoint_destroy(esrrf_adjoint* a) {
    if (!a) return ESRRF_ERR_INVALID;
    a->release();
    delete a;
    return ESRRF_OK;
}

}  // extern "C"
