// drift.cu -- frame drift (vibration) estimation by cross-correlation against a reference frame
// (XYShiftCalculator.calculateShiftArray, XYShiftCalculator.java:26-48; ParametersSweep_.java:282-290
// and LiveSRRF_optimised_.java:283-305 feed its result to loadDriftXYGPUbuffer).
//
// The reference takes NanoJ-Core's cross-correlation map of each frame against the block's first
// frame and the sub-pixel position of the map's peak (CrossCorrelationMap,
// EstimateShiftAndTilt.getShiftFromCrossCorrelationPeak; NanoJ-Core is not in the reference tree).
// Restated here:
//   C_f(s) = sum_p (ref(p) - mean ref) frame_f((p + s) mod size)
// the circular cross-correlation (the frame's own mean drops out of a circular sum, and a Pearson
// normalisation is one constant per frame, so neither moves the peak), evaluated directly for the
// lags |sx|, |sy| <= R; its arg-max (first in row-major order on ties); and the stationary point of
// the least-squares quadratic through the 3 x 3 samples around it.  The result d is the displacement
// of the frame's content relative to the reference (frame(p) = ref(p - d)): liveSRRF.cl:263 samples
// frame f at (x + shiftX[f], y + shiftY[f]), which then reads ref(x, y).
//
// Kernels:
//   ref_mean_kernel / ref_center_kernel  the reference frame minus its mean, float
//   corr_kernel   one block = 64 x 64 lags of one frame over one stripe of image row tiles; each
//                 thread 4 x 4 lags, reading float4 rows of the staged frame tile (16 FMAs per 2
//                 shared-memory loads); each row's products summed in FP32, rows and tiles in
//                 FP64; per-stripe partial maps
//   peak_kernel   one block per frame: stripes summed in a fixed order (deterministic), map written
//                 out, arg-max, quadratic fit in FP64
#include <math.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "esrrf.h"

namespace {

constexpr int kLag = 64;              // lags per block side (16 threads x 4)
constexpr int kTX = 32, kTY = 32;     // image tile
constexpr int kGX = kTX + kLag;       // staged frame tile: 96 columns (float4 rows)
constexpr int kGY = kTY + kLag - 1;   // 95 rows

__device__ __forceinline__ float ld(const void* p, int is_u16, long i) {
    return is_u16 ? (float)__ldg((const unsigned short*)p + i) : __ldg((const float*)p + i);
}

__device__ __forceinline__ int wrap(int v, int n) {
    v %= n;
    return v < 0 ? v + n : v;
}

__global__ void ref_mean_kernel(const void* frames, int is_u16, long ref_off, long N, double* sum) {
    double s = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
        s += ld(frames, is_u16, ref_off + i);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, s);
}

__global__ void ref_center_kernel(const void* frames, int is_u16, long ref_off, long N, const double* sum,
                                  float* __restrict__ r) {
    const float mean = (float)(*sum / (double)N);
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
        r[i] = ld(frames, is_u16, ref_off + i) - mean;
}

struct CorrArgs {
    const float* r;      // centred reference, w x h
    const void* frames;  // n x h x w
    int is_u16, w, h, R, side;
    int n_lag;           // lag tiles per side
    int stripes;         // row-tile stripes per frame
    double* part;        // [frame][stripe][side][side]
};

__global__ void __launch_bounds__(256, 3) corr_kernel(CorrArgs a) {
    __shared__ __align__(16) float sg[kGY][kGX];
    __shared__ __align__(16) float sr[kTY][kTX];
    __shared__ int wy[kGY], wx[kGX];
    const int f = blockIdx.y, stripe = blockIdx.z;
    const int lbx = blockIdx.x % a.n_lag, lby = blockIdx.x / a.n_lag;
    const int sxb = lbx * kLag - a.R, syb = lby * kLag - a.R;  // first lag of the block
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const long fo = (long)f * a.w * a.h;
    double dacc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dacc[i][j] = 0.0;
    const int n_rt = (a.h + kTY - 1) / kTY, n_ct = (a.w + kTX - 1) / kTX;
    for (int rt = stripe; rt < n_rt; rt += a.stripes) {
        const int y0 = rt * kTY;
        for (int ct = 0; ct < n_ct; ++ct) {
            const int x0 = ct * kTX;
            __syncthreads();
            if (threadIdx.x < kGY) wy[threadIdx.x] = wrap(y0 + syb + (int)threadIdx.x, a.h);
            if (threadIdx.x < kGX) wx[threadIdx.x] = wrap(x0 + sxb + (int)threadIdx.x, a.w);
            for (int i = threadIdx.x; i < kTY * kTX; i += 256) {
                const int yy = y0 + i / kTX, xx = x0 + i % kTX;
                sr[i / kTX][i % kTX] = (yy < a.h && xx < a.w) ? a.r[(long)yy * a.w + xx] : 0.f;
            }
            __syncthreads();
            for (int i = threadIdx.x; i < kGY * kGX; i += 256) {
                const int rr = i / kGX, cc = i % kGX;
                sg[rr][cc] = ld(a.frames, a.is_u16, fo + (long)wy[rr] * a.w + wx[cc]);
            }
            __syncthreads();
            for (int ly = 0; ly < kTY; ++ly) {
                // one row of the tile: 32 products per lag in FP32, flushed to FP64
                float acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
                const float4* srow = reinterpret_cast<const float4*>(sr[ly]);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    // lags (sy = syb + 4 ty + i, sx = sxb + 4 tx + j) read sg[ly + 4 ty + i][lx + 4 tx + j]
                    const float4* grow = reinterpret_cast<const float4*>(sg[ly + 4 * ty + i]) + tx;
                    float4 lo = grow[0];
#pragma unroll
                    for (int q4 = 0; q4 < kTX / 4; ++q4) {
                        const float4 hi = grow[q4 + 1];
                        const float4 rv = srow[q4];
                        const float g[7] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z};
                        const float rq[4] = {rv.x, rv.y, rv.z, rv.w};
#pragma unroll
                        for (int q = 0; q < 4; ++q)
#pragma unroll
                            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(rq[q], g[q + j], acc[i][j]);
                        lo = hi;
                    }
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) dacc[i][j] += (double)acc[i][j];
            }
        }
    }
    double* out = a.part + ((long)f * a.stripes + stripe) * a.side * a.side;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int ly = lby * kLag + 4 * ty + i;  // = sy + R
        if (ly >= a.side) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int lx = lbx * kLag + 4 * tx + j;
            if (lx < a.side) out[(long)ly * a.side + lx] = dacc[i][j];
        }
    }
}

// One block per frame: C = sum over stripes (fixed order), optional float copy, arg-max, fit.
__global__ void __launch_bounds__(256) peak_kernel(double* part, int stripes, int side, int R,
                                                    float* __restrict__ ccm_out, float* __restrict__ shifts) {
    const int f = blockIdx.x;
    const long M = (long)side * side;
    double* base = part + (long)f * stripes * M;  // stripe 0 receives the sum
    double best = -INFINITY;
    long bi = 0x7fffffffffffffffL;
    for (long i = threadIdx.x; i < M; i += blockDim.x) {
        double v = base[i];
        for (int s = 1; s < stripes; ++s) v += base[(long)s * M + i];
        base[i] = v;
        if (ccm_out) ccm_out[(long)f * M + i] = (float)v;
        if (v > best) {  // ascending i: the first maximum of this thread's lags
            best = v;
            bi = i;
        }
    }
    __shared__ double sv[256];
    __shared__ long si[256];
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            const double v2 = sv[threadIdx.x + o];
            const long i2 = si[threadIdx.x + o];
            if (v2 > sv[threadIdx.x] || (v2 == sv[threadIdx.x] && i2 < si[threadIdx.x])) {
                sv[threadIdx.x] = v2;
                si[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const long b = si[0] < M ? si[0] : 0;
    const int py = (int)(b / side), px = (int)(b % side);
    double ox = 0.0, oy = 0.0;
    if (px > 0 && px < side - 1 && py > 0 && py < side - 1) {
        // least-squares quadratic a + b x + c y + d x^2 + e x y + f y^2 through the 3 x 3 samples
        // (x, y in -1..1): the normal equations separate into b = Sx/6, c = Sy/6, e = Sxy/4,
        // d = Sxx/2 - S/3, f = Syy/2 - S/3; stationary point clamped to [-1, 1]
        double S = 0, Sx = 0, Sy = 0, Sxy = 0, Sxx = 0, Syy = 0;
        for (int j = -1; j <= 1; ++j)
            for (int i = -1; i <= 1; ++i) {
                const double z = base[(long)(py + j) * side + px + i];
                S += z;
                Sx += i * z;
                Sy += j * z;
                Sxy += i * j * z;
                Sxx += i * i * z;
                Syy += j * j * z;
            }
        const double cb = Sx / 6.0, cc = Sy / 6.0, ce = Sxy / 4.0;
        const double cd = Sxx / 2.0 - S / 3.0, cf = Syy / 2.0 - S / 3.0;
        const double det = 4.0 * cd * cf - ce * ce;
        if (det != 0.0) {
            ox = (-2.0 * cf * cb + ce * cc) / det;
            oy = (-2.0 * cd * cc + ce * cb) / det;
        }
        ox = fmax(-1.0, fmin(1.0, ox));
        oy = fmax(-1.0, fmin(1.0, oy));
    }
    shifts[2 * f] = (float)(px - R + ox);
    shifts[2 * f + 1] = (float)(py - R + oy);
}

std::mutex g_mu;
std::string g_err;

struct Workspace {
    void* p = nullptr;
    size_t bytes = 0;
};
std::mutex g_ws_mu;
std::map<int, Workspace> g_ws;

esrrf_status fail(const std::string& m, esrrf_status s = ESRRF_ERR_INVALID) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_err = m;
    return s;
}

}  // namespace

extern "C" {

const char* esrrf_drift_last_error(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_err.c_str();
}

esrrf_status esrrf_drift_window(int width, int height, int max_shift, int* radius) {
    if (!radius) return fail("null argument");
    if (width < 3 || height < 3) return fail("need frames of at least 3 x 3 pixels");
    const int lim = (std::min(width, height) - 1) / 2;
    const int R = max_shift > 0 ? max_shift : 31;
    *radius = std::max(1, std::min(R, lim));
    return ESRRF_OK;
}

esrrf_status esrrf_estimate_drift(const void* d_frames, int is_u16, int n_frames, int width, int height,
                                  int ref_frame, int max_shift, float* shift_x, float* shift_y,
                                  float* d_ccm, void* stream) {
    if (!d_frames || !shift_x || !shift_y) return fail("null argument");
    if (n_frames < 1) return fail("need at least one frame");
    if (ref_frame < 0 || ref_frame >= n_frames) return fail("ref_frame outside the frames");
    int R = 0;
    if (esrrf_drift_window(width, height, max_shift, &R) != ESRRF_OK) return ESRRF_ERR_INVALID;
    if ((long)width * height > (1L << 30)) return fail("frame too large");
    cudaStream_t st = (cudaStream_t)stream;
    const long N = (long)width * height;
    const int side = 2 * R + 1;
    const int n_lag = (side + kLag - 1) / kLag;
    const int n_rt = (height + kTY - 1) / kTY;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail("no current CUDA device", ESRRF_ERR_CUDA);
    // one block per (lag tile, frame, image row tile) -- the finest split measured fastest on a
    // B200 (100 frames of 512 x 512: 4.7 ms against 5.2 ms for 4 row tiles per block) -- unless the
    // per-stripe partial maps would pass 1 GB
    const long per_stripe = (long)n_frames * side * side * (long)sizeof(double);
    const int stripes = (int)std::max<long>(1, std::min<long>(n_rt, (1L << 30) / std::max(1L, per_stripe)));
    if (n_frames > 65535) return fail("at most 65535 frames per call");
    // one cached workspace per device, grown on demand (calls on a device are serialised)
    const size_t off_part = 0, off_r = off_part + (size_t)per_stripe * stripes;
    const size_t off_sum = (off_r + sizeof(float) * N + 255) / 256 * 256;
    const size_t off_sh = off_sum + 256, need = off_sh + sizeof(float) * 2 * n_frames;
    std::lock_guard<std::mutex> ws_lock(g_ws_mu);
    Workspace& ws = g_ws[dev];
#define DK(call)                                                 \
    do {                                                         \
        cudaError_t _e = (call);                                 \
        if (_e != cudaSuccess) return fail(cudaGetErrorString(_e), ESRRF_ERR_CUDA); \
    } while (0)
    if (ws.bytes < need) {
        if (ws.p) DK(cudaFree(ws.p));
        ws.p = nullptr;
        ws.bytes = 0;
        DK(cudaMalloc(&ws.p, need));
        ws.bytes = need;
    }
    char* base = (char*)ws.p;
    double* part = (double*)(base + off_part);
    float* r = (float*)(base + off_r);
    double* sum = (double*)(base + off_sum);
    float* shifts = (float*)(base + off_sh);
    DK(cudaMemsetAsync(sum, 0, sizeof(double), st));
    const long ref_off = (long)ref_frame * N;
    ref_mean_kernel<<<128, 256, 0, st>>>(d_frames, is_u16, ref_off, N, sum);
    ref_center_kernel<<<256, 256, 0, st>>>(d_frames, is_u16, ref_off, N, sum, r);
    CorrArgs a{r, d_frames, is_u16, width, height, R, side, n_lag, stripes, part};
    corr_kernel<<<dim3(n_lag * n_lag, n_frames, stripes), 256, 0, st>>>(a);
    peak_kernel<<<n_frames, 256, 0, st>>>(part, stripes, side, R, d_ccm, shifts);
    DK(cudaGetLastError());
    std::vector<float> h(2 * (size_t)n_frames);
    DK(cudaMemcpyAsync(h.data(), shifts, sizeof(float) * h.size(), cudaMemcpyDeviceToHost, st));
    DK(cudaStreamSynchronize(st));
#undef DK
    for (int f = 0; f < n_frames; ++f) {
        shift_x[f] = h[2 * f];
        shift_y[f] = h[2 * f + 1];
    }
    return ESRRF_OK;
}

}  // extern "C"
