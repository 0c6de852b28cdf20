// rgc_fht_drift.cu -- the fused FHT-path RGC on frames with drift (vibration correction).
//
// The reference applies the per-frame shift of loadDriftXYGPUbuffer (LiveSRRF_CL.java:583-595,
// stored x M) inside calculateRadialGradientConvergence: the centre of output pixel xM is
// xc = xM + 0.5 + shiftX (liveSRRF_noInterpolation.cl:264-268) and the intensity is
// getInterpolatedValue(xM + shiftX, yM + shiftY) when the shift is not zero (:356-357).  The
// plugins set it per SR block (gui/LiveSRRF_optimised_.java:283-305) or once for the whole sweep
// (gui/ParametersSweep_.java:282-290, :452-454).  A shift is uniform over a frame, so here each
// frame of a launch gets its own tap tables (drift_tables_kernel: weights, disc chords, prefix
// sums, the frame's record), and the fused tile kernel (fht_fused.cuh, DRIFT = true) runs on them
// at full tap rate, sampling the shifted intensities from its staged tile.  shift_sample_kernel
// writes whole intensity planes at the shifted positions for the sweep's per-frame mode.
//
// Residual against the reference's per-pixel arithmetic: the reference rounds xc to float per
// pixel, so its centre offsets carry a rounding error of up to half an ulp of xM (6e-5 magnified
// pixels below 2048); the tables use the exact fraction of the shift.  Where that rounding (a
// fraction within rounding of 1) or the truncation of (int)(xc - 0.5) towards zero (left of or
// above the image) moves a pixel's box by one source column or row, the tile kernel corrects that
// pixel's sums by the box's moved edges with the reference's per-tap arithmetic (fht_fused.cuh).
#include <math.h>

#include "device_common.cuh"
#include "esrrf_internal.h"
#include "fht_fused.cuh"

namespace esrrf {

namespace {

// One CTA per frame of the launch.  S <= 32; the tables of a frame are laid out for this S (the
// buffers may have been sized for a larger one).
__global__ void __launch_bounds__(256) drift_tables_kernel(const float* __restrict__ sxp,
                                                           const float* __restrict__ syp, int r0, int S,
                                                           float tSS, float tSO, FhtDriftTables t) {
    __shared__ float sw[32 * 32];            // [jj][ii] weights
    __shared__ float swd[32 * 32];           // [jj][ii] weight / distance
    __shared__ unsigned char sin_[32 * 32];  // [jj][ii] 1: tap inside the disc
    __shared__ int slo[32], shi[32];         // per column: first and last tap row of the disc
    __shared__ double spre[33 * 33];         // [jj][ii] prefix sums
    const int f = blockIdx.x, tid = threadIdx.x;
    const float sxf = sxp[f], syf = syp[f];
    const double flx = floor((double)sxf), fly = floor((double)syf);
    const double fxd = (double)sxf - flx, fyd = (double)syf - fly;
    for (int idx = tid; idx < S * S; idx += blockDim.x) {
        const int ii = idx / S, jj = idx - ii * S;
        // the reference's per-tap arithmetic (liveSRRF_noInterpolation.cl:285-298), no contraction
        const float dx = (float)((double)(r0 + ii) - fxd), dy = (float)((double)(r0 + jj) - fyd);
        const float d = sqrtf(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
        const bool in = d != 0.f && d <= tSO;
        float w = 0.f, wd = 0.f;
        if (in) {
            w = __fmul_rn(d, expf(-__fmul_rn(d, d) / tSS));
            w = __fmul_rn(__fmul_rn(__fmul_rn(w, w), w), w);
            wd = w / d;
        }
        sw[jj * S + ii] = w;
        swd[jj * S + ii] = wd;
        sin_[jj * S + ii] = in ? 1 : 0;
    }
    __syncthreads();
    if (tid < S) {  // column tid: its disc chord (a disc meets a column in one run of rows)
        int lo = S, hi = -1;
        for (int jj = 0; jj < S; ++jj)
            if (sin_[jj * S + tid]) {
                lo = min(lo, jj);
                hi = max(hi, jj);
            }
        slo[tid] = lo;
        shi[tid] = hi;
        t.jr[(long)f * 2 * S + 2 * tid] = lo;
        t.jr[(long)f * 2 * S + 2 * tid + 1] = hi;
    }
    __syncthreads();
    // weights of column ii from its chord's first row on: entry jj' holds tap row lo + jj'
    for (int idx = tid; idx < S * S; idx += blockDim.x) {
        const int ii = idx / S, jq = idx - ii * S, jj = slo[ii] + jq;
        t.wt[(long)f * S * S + idx] = jj <= shi[ii] ? make_float2(sw[jj * S + ii], swd[jj * S + ii])
                                                    : make_float2(0.f, 0.f);
    }
    const int P = S + 1;
    if (tid <= S) {  // row prefix sums: spre[jj + 1][ii + 1] = sum of row jj up to column ii
        if (tid == 0) {
            for (int ii = 0; ii < P; ++ii) spre[ii] = 0.0;
        } else {
            const int jj = tid - 1;
            double s = 0.0;
            spre[tid * P] = 0.0;
            for (int ii = 0; ii < S; ++ii) {
                s += (double)sw[jj * S + ii];
                spre[tid * P + ii + 1] = s;
            }
        }
    }
    __syncthreads();
    if (tid <= S)  // then down each column
        for (int jj = 1; jj < P; ++jj) spre[jj * P + tid] += spre[(jj - 1) * P + tid];
    __syncthreads();
    for (int idx = tid; idx < P * P; idx += blockDim.x) t.pre[(long)f * P * P + idx] = spre[idx];
    if (tid == 0) {
        float ws = 0.f;  // the reference's float sum, j outer, i inner
        for (int jj = 0; jj < S; ++jj)
            for (int ii = 0; ii < S; ++ii)
                if (sin_[jj * S + ii]) ws = __fadd_rn(ws, sw[jj * S + ii]);
        FhtDriftFrame d;
        d.ix = (int)flx;
        d.iy = (int)fly;
        d.fi0 = (float)((double)r0 - fxd);
        d.fj0 = (float)((double)r0 - fyd);
        d.wsum_int = ws;
        d.fx = (float)fxd;
        d.fy = (float)fyd;
        d.zero = sxf == 0.f && syf == 0.f;
        d.sx = sxf;
        d.sy = syf;
        t.fr[f] = d;
    }
}

// Intensity of every pixel of F frames at the frame's shift, as the reference reads it
// (liveSRRF_noInterpolation.cl:355-357).
__global__ void shift_sample_kernel(const float* __restrict__ interp, int W, int H,
                                    const float* __restrict__ sxp, const float* __restrict__ syp,
                                    float* __restrict__ v) {
    const int f = blockIdx.y;
    const long wh = (long)W * H;
    const long pix = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= wh) return;
    const float sx = __ldg(sxp + f), sy = __ldg(syp + f);
    const float* fr = interp + (long)f * wh;
    const int yM = (int)(pix / W), xM = (int)(pix - (long)yM * W);
    v[(long)f * wh + pix] = (sx == 0.f && sy == 0.f)
                                ? __ldg(fr + pix)
                                : dev::sample2d(fr, W, H, (float)xM + sx, (float)yM + sy);
}

}  // namespace

cudaError_t fht_rgc_fused_drift_wide(int S, const fused::FusedParams& fp, const fused::DriftParams& dp,
                                     const FhtRgcArgs& a, cudaStream_t stream);

cudaError_t fht_drift_tables_alloc(int S, int F, long pixels, FhtDriftTables& t) {
    cudaError_t e;
    t.capacity = F;
    t.S = S;
    if ((e = cudaMalloc(&t.fr, sizeof(FhtDriftFrame) * F)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&t.wt, sizeof(float2) * (size_t)F * S * S)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&t.jr, sizeof(int) * (size_t)F * 2 * S)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&t.pre, sizeof(double) * (size_t)F * (S + 1) * (S + 1))) != cudaSuccess) return e;
    if (pixels <= 0) return cudaSuccess;
    return cudaMalloc(&t.v, sizeof(float) * (size_t)F * pixels);
}

void fht_drift_tables_free(FhtDriftTables& t) {
    cudaFree(t.fr);
    cudaFree(t.wt);
    cudaFree(t.jr);
    cudaFree(t.pre);
    cudaFree(t.v);
    t = FhtDriftTables();
}

cudaError_t fht_drift_tables_build(const FhtGeometry& g, const float* sx, const float* sy, int F,
                                   FhtDriftTables& t, cudaStream_t stream) {
    if (F < 1 || F > t.capacity || g.S > t.S || g.S > 32) return cudaErrorInvalidValue;
    drift_tables_kernel<<<F, 256, 0, stream>>>(sx, sy, g.r0, g.S, g.tSS, g.tSO, t);
    return cudaGetLastError();
}

cudaError_t fht_shift_sample(const float* interp, int W, int H, int F, const float* sx, const float* sy,
                             float* v, cudaStream_t stream) {
    const long wh = (long)W * H;
    dim3 grid((unsigned)((wh + 255) / 256), (unsigned)F);
    shift_sample_kernel<<<grid, 256, 0, stream>>>(interp, W, H, sx, sy, v);
    return cudaGetLastError();
}

cudaError_t fht_rgc_fused_drift(const FhtGeometry& g, const FhtDriftTables& t, const FhtRgcArgs& a,
                                cudaStream_t stream) {
    if (a.F > t.capacity || g.S > t.S) return cudaErrorInvalidValue;
    const fused::FusedParams fp{g.r0, g.sensitivity, nullptr, nullptr, nullptr, nullptr};
    const fused::DriftParams dp{t.fr, t.wt, t.jr, t.pre, t.v, g.tSS, g.tSO};
    // tap boxes of 22 .. 32 are instantiated in rgc_fht_drift_wide.cu (compiled in parallel)
    if (g.S >= 22) return fht_rgc_fused_drift_wide(g.S, fp, dp, a, stream);
    return fused::launch_fused_in<true, 4, 20>(g.S, g.r0, g.sensitivity, fp, dp, a, stream);
}

}  // namespace esrrf
