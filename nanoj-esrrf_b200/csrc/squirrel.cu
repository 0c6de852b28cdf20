// squirrel.cu -- resolution-scaled error (RSE), resolution-scaled Pearson coefficient (RSP) and
// error maps of many super-resolved images against their references, on the GPU
// (ErrorMapLiveSRRF.java:81-193, as ParametersSweep_.java:468-519 applies it to every sweep
// reconstruction: SR = the AVG, VAR or TAC2 slice, reference = the INT slice of the same block).
//
// For each image: optionally crop a border of `crop` input pixels (x M) from both images; find the
// blur sigma in [0, 4 / 2.35482 M] that minimises RMSE(ref, G_sigma * (alpha SR + beta)), with
// alpha, beta the least-squares fit of ref to (G_sigma * SR, G_sigma * 1) for that sigma
// (calculateAlphaBeta, :206-239; Brent search, :119-125); then RSE = that RMSE, RSP = the
// Pearson correlation of G_sigma * (alpha SR + beta) with ref, and the error map
// |ref - G_sigma * (alpha SR + beta)|.
//
// The blur restates ImageJ's Gaussian blur as the reference calls it (FloatProcessor.blurGaussian,
// accuracy 0.01: kernel radius ceil(sigma sqrt(-2 ln 0.01)) + 1, normalised, edge pixels
// replicated).  With replicated edges G * 1 = 1 and G * (alpha X + beta) = alpha G * X + beta, so
// every objective evaluation needs only the blurred SR image's sums (sum B, sum B^2, sum B ref),
// accumulated in FP64; all images' Brent searches advance in lockstep, one batched blur per step.
// (ImageJ additionally smooths the kernel's last few taps and down-samples for large sigma; those
// refinements are not restated.)
#include <math.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "esrrf.h"

namespace {

constexpr int kMaxRadius = 255;   // kernel radius limit (sigma up to ~80 pixels)
constexpr int kRowTile = 64;      // rows per column-pass block

struct Img {
    size_t sr_off, ref_off;       // floats from the base pointers to the image's first pixel
    float sigma;                  // current blur
    int radius;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ void make_kernel(float sigma, int r, float* k) {
    // k[0..r]: exp(-x^2 / 2 sigma^2), normalised over -r..r (r = 0: identity)
    if (threadIdx.x <= r) k[threadIdx.x] = r == 0 ? 1.f : expf(-0.5f * (float)(threadIdx.x * threadIdx.x) / (sigma * sigma));
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = k[0];
        for (int i = 1; i <= r; ++i) s += 2.f * k[i];
        const float inv = 1.f / s;
        for (int i = 0; i <= r; ++i) k[i] *= inv;
    }
    __syncthreads();
}

// Row pass: tmp[i][y][x] = sum_t k[t] SR[y][clamp(x + t)] over the cropped window.
__global__ void __launch_bounds__(256) row_pass_kernel(const float* __restrict__ base, const Img* __restrict__ imgs,
                                                       int W, int x0, int y0, int Wc, int Hc,
                                                       float* __restrict__ tmp) {
    extern __shared__ float sm[];  // [kMaxRadius + 1] kernel, then the row
    const Img im = imgs[blockIdx.y];
    const int r = im.radius;
    float* k = sm;
    float* row = sm + kMaxRadius + 1;
    make_kernel(im.sigma, r, k);
    const int y = blockIdx.x;
    const float* src = base + im.sr_off + (long)(y0 + y) * W + x0;
    for (int i = threadIdx.x; i < Wc + 2 * r; i += blockDim.x) row[i] = src[clampi(i - r, 0, Wc - 1)];
    __syncthreads();
    float* dst = tmp + ((long)blockIdx.y * Hc + y) * Wc;
    for (int x = threadIdx.x; x < Wc; x += blockDim.x) {
        float s = k[0] * row[x + r];
        for (int t = 1; t <= r; ++t) s = fmaf(k[t], row[x + r - t] + row[x + r + t], s);
        dst[x] = s;
    }
}

// Column pass on a 32-column x kRowTile-row block, then the block's FP64 sums of B, B^2 and
// B ref (and, with `map`, the error map for the given alpha, beta).
__global__ void __launch_bounds__(256) col_pass_kernel(const float* __restrict__ base, const Img* __restrict__ imgs,
                                                       const float* __restrict__ tmp, int W, int x0, int y0,
                                                       int Wc, int Hc, double* __restrict__ sums,
                                                       const float* __restrict__ ab, float* __restrict__ map) {
    extern __shared__ float sm[];  // kernel, then [(kRowTile + 2r)][32]
    const int i = blockIdx.z;
    const Img im = imgs[i];
    const int r = im.radius;
    float* k = sm;
    float* col = sm + kMaxRadius + 1;
    make_kernel(im.sigma, r, k);
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const int x = blockIdx.x * 32 + lane, ys = blockIdx.y * kRowTile;
    const float* t = tmp + (long)i * Hc * Wc;
    const int xc = min(x, Wc - 1);
    for (int j = wq; j < kRowTile + 2 * r; j += 8) col[j * 32 + lane] = t[(long)clampi(ys + j - r, 0, Hc - 1) * Wc + xc];
    __syncthreads();
    double sb = 0.0, sbb = 0.0, sbr = 0.0;
    for (int j = wq; j < kRowTile; j += 8) {
        const int y = ys + j;
        if (x >= Wc || y >= Hc) continue;
        float b = k[0] * col[(j + r) * 32 + lane];
        for (int q = 1; q <= r; ++q) b = fmaf(k[q], col[(j + r - q) * 32 + lane] + col[(j + r + q) * 32 + lane], b);
        const float rv = base[im.ref_off + (long)(y0 + y) * W + x0 + x];
        if (map) {
            map[((long)i * Hc + y) * Wc + x] = fabsf(rv - fmaf(ab[2 * i], b, ab[2 * i + 1]));
            continue;
        }
        sb += b;
        sbb += (double)b * b;
        sbr += (double)b * rv;
    }
    if (map) return;
    __shared__ double red[3][8];
    for (int o = 16; o > 0; o >>= 1) {
        sb += __shfl_xor_sync(0xffffffffu, sb, o);
        sbb += __shfl_xor_sync(0xffffffffu, sbb, o);
        sbr += __shfl_xor_sync(0xffffffffu, sbr, o);
    }
    if (lane == 0) {
        red[0][wq] = sb;
        red[1][wq] = sbb;
        red[2][wq] = sbr;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) s += red[threadIdx.x][w];
        atomicAdd(sums + 3 * i + threadIdx.x, s);
    }
}

// Sum and sum of squares of each cropped reference (independent of sigma).
__global__ void __launch_bounds__(256) ref_stats_kernel(const float* __restrict__ base, const Img* __restrict__ imgs,
                                                        int W, int x0, int y0, int Wc, int Hc,
                                                        double* __restrict__ sums) {
    const Img im = imgs[blockIdx.y];
    double s = 0.0, ss = 0.0;
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < (long)Wc * Hc; p += (long)gridDim.x * blockDim.x) {
        const float v = base[im.ref_off + (long)(y0 + p / Wc) * W + x0 + p % Wc];
        s += v;
        ss += (double)v * v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        ss += __shfl_xor_sync(0xffffffffu, ss, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(sums + 2 * blockIdx.y, s);
        atomicAdd(sums + 2 * blockIdx.y + 1, ss);
    }
}

int kernel_radius(double sigma) {
    // ImageJ GaussianBlur.makeGaussianKernel: ceil(sigma sqrt(-2 ln accuracy)) + 1, accuracy 0.01
    if (!(sigma > 0.0)) return 0;
    return std::min(kMaxRadius, (int)std::ceil(sigma * std::sqrt(-2.0 * std::log(0.01))) + 1);
}

// Brent's minimisation without derivatives (R. P. Brent, 1973, procedure localmin), started at the
// interval's midpoint with stopping tolerance rel |x| + abs, as commons-math3's BrentOptimizer
// applies it; written as a state machine so that many searches can share one evaluation batch.
struct Brent {
    double a, b, x, w, v, fx, fw, fv, d = 0.0, e = 0.0, u = 0.0;
    double best_x, best_f;
    double rel = 1e-10, abs_tol = 1e-14;
    int evals = 0, max_evals = 1000;
    bool started = false, done = false;
    Brent(double lo, double hi) : a(lo), b(hi), x(0.5 * (lo + hi)), w(x), v(x) {}
    // the next abscissa to evaluate, or false when converged
    bool propose(double& out) {
        if (done) return false;
        if (!started) {
            out = x;
            return true;
        }
        const double c = 0.5 * (3.0 - std::sqrt(5.0));
        const double m = 0.5 * (a + b);
        const double tol1 = rel * std::fabs(x) + abs_tol, tol2 = 2.0 * tol1;
        if (std::fabs(x - m) <= tol2 - 0.5 * (b - a) || evals >= max_evals) {
            done = true;
            return false;
        }
        bool golden = true;
        if (std::fabs(e) > tol1) {
            double r = (x - w) * (fx - fv), q = (x - v) * (fx - fw), p = (x - v) * q - (x - w) * r;
            q = 2.0 * (q - r);
            if (q > 0.0)
                p = -p;
            else
                q = -q;
            r = e;
            e = d;
            if (std::fabs(p) < std::fabs(0.5 * q * r) && p > q * (a - x) && p < q * (b - x)) {
                d = p / q;
                u = x + d;
                if (u - a < tol2 || b - u < tol2) d = x <= m ? tol1 : -tol1;
                golden = false;
            }
        }
        if (golden) {
            e = x < m ? b - x : a - x;
            d = c * e;
        }
        u = x + (std::fabs(d) >= tol1 ? d : (d > 0.0 ? tol1 : -tol1));
        out = u;
        return true;
    }
    void tell(double f) {
        ++evals;
        if (!started) {
            started = true;
            fx = fw = fv = f;
            best_x = x;
            best_f = f;
            return;
        }
        if (f < best_f) {
            best_f = f;
            best_x = u;
        }
        if (f <= fx) {
            if (u < x)
                b = x;
            else
                a = x;
            v = w;
            fv = fw;
            w = x;
            fw = fx;
            x = u;
            fx = f;
        } else {
            if (u < x)
                a = u;
            else
                b = u;
            if (f <= fw || w == x) {
                v = w;
                fv = fw;
                w = u;
                fw = f;
            } else if (f <= fv || v == x || v == w) {
                v = u;
                fv = f;
            }
        }
    }
};

struct Fit {
    double alpha, beta, rmse, ppmcc;
};

// calculateAlphaBeta and the RMSE / Pearson coefficient of alpha B + beta against the reference,
// from the sums (blurred ones are exactly one with replicated edges, so N = the pixel count).
Fit fit_from_sums(double n, double sb, double sbb, double sbr, double sr, double srr) {
    Fit f{};
    const double den = n * sbb - sb * sb;
    f.alpha = den != 0.0 ? (n * sbr - sr * sb) / den : 0.0;
    f.beta = sr / n - f.alpha * (sb / n);
    const double a = f.alpha, b = f.beta;
    const double sse = a * a * sbb + 2.0 * a * b * sb + n * b * b - 2.0 * a * sbr - 2.0 * b * sr + srr;
    f.rmse = std::sqrt(std::max(sse, 0.0) / n);
    const double vr = n * srr - sr * sr;
    const double cov = n * sbr - sb * sr;
    f.ppmcc = (den > 0.0 && vr > 0.0) ? (a < 0.0 ? -1.0 : 1.0) * cov / std::sqrt(den * vr) : 0.0;
    return f;
}

std::mutex g_err_mu;
std::string g_err;

esrrf_status fail(const std::string& m, esrrf_status s = ESRRF_ERR_INVALID) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err = m;
    return s;
}

// Scratch of esrrf_squirrel, kept per device between calls (grow-only): allocating and freeing
// the up-to-1 GB blur buffer on every call made the call's time vary by a factor of two.  A call
// holds its device's lock throughout, so concurrent calls on one device run one after the other.
struct SquirrelScratch {
    std::mutex mu;
    float* tmp = nullptr;
    size_t tmp_floats = 0;
    void* img = nullptr;  // Img[batch]
    double* sums = nullptr;
    float* ab = nullptr;
    int batch = 0;
};
SquirrelScratch g_sq[64];

}  // namespace

extern "C" {

const char* esrrf_squirrel_last_error(void) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    return g_err.c_str();
}

esrrf_status esrrf_squirrel(const esrrf_squirrel_params* p, int n, const float* d_base,
                            const size_t* sr_offsets, const size_t* ref_offsets, float* sigma,
                            float* alpha, float* beta, float* rse, float* rsp, float* d_error_maps) {
    if (!p || !d_base || !sr_offsets || !ref_offsets || n < 0) return fail("null argument");
    if (n == 0) return ESRRF_OK;
    const int W = p->width, H = p->height, M = p->magnification;
    if (W < 1 || H < 1 || M < 1) return fail("width, height and magnification must be positive");
    const int cb = p->crop > 0 ? p->crop * M : 0;
    const int Wc = W - 2 * cb, Hc = H - 2 * cb;
    if (Wc < 1 || Hc < 1) return fail("crop leaves no pixels");
    const double smax = (double)((4.0f / 2.35482f) * (float)M);  // maxSigmaBoundary, Nyquist assumed
    const double sfix = (double)(p->fixed_sigma * (float)M);
    if (kernel_radius(p->fix_sigma ? sfix : smax) >= kMaxRadius) return fail("sigma too large for the blur kernel");
    cudaStream_t st = (cudaStream_t)p->stream;
    const int batch = std::max(1, std::min(n, (int)(((size_t)1 << 30) / ((size_t)Wc * Hc * sizeof(float)))));
    const size_t colsmem = sizeof(float) * (kMaxRadius + 1 + (size_t)(kRowTile + 2 * kMaxRadius) * 32);
    const size_t rowsmem = sizeof(float) * (kMaxRadius + 1 + (size_t)Wc + 2 * kMaxRadius);
    if (rowsmem > 200 * 1024) return fail("image too wide");
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(col_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)colsmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(row_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rowsmem)) != cudaSuccess)
        return fail(cudaGetErrorString(e), ESRRF_ERR_CUDA);
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return fail(cudaGetErrorString(e), ESRRF_ERR_CUDA);
    if (dev < 0 || dev >= 64) return fail("device ordinal out of range");
    SquirrelScratch& sc = g_sq[dev];
    std::lock_guard<std::mutex> lk(sc.mu);
#define SQ(call)                                                     \
    do {                                                             \
        cudaError_t _e = (call);                                     \
        if (_e != cudaSuccess) return fail(cudaGetErrorString(_e), ESRRF_ERR_CUDA); \
    } while (0)
    const size_t need = (size_t)batch * Wc * Hc;
    if (sc.tmp_floats < need) {
        SQ(cudaStreamSynchronize(st));
        cudaFree(sc.tmp);
        sc.tmp = nullptr;
        sc.tmp_floats = 0;
        SQ(cudaMalloc(&sc.tmp, sizeof(float) * need));
        sc.tmp_floats = need;
    }
    if (sc.batch < batch) {
        SQ(cudaStreamSynchronize(st));
        cudaFree(sc.img);
        cudaFree(sc.sums);
        cudaFree(sc.ab);
        sc.img = nullptr;
        sc.sums = nullptr;
        sc.ab = nullptr;
        sc.batch = 0;
        SQ(cudaMalloc(&sc.img, sizeof(Img) * batch));
        SQ(cudaMalloc(&sc.sums, sizeof(double) * 3 * batch));
        SQ(cudaMalloc(&sc.ab, sizeof(float) * 2 * batch));
        sc.batch = batch;
    }
    float* tmp = sc.tmp;
    Img* d_img = static_cast<Img*>(sc.img);
    double* d_sums = sc.sums;
    float* d_ab = sc.ab;
    const double npx = (double)Wc * Hc;
    std::vector<Img> hi(batch);
    std::vector<double> hs(3 * batch);
    // blur the listed images at their sigmas and return (sum B, sum B^2, sum B ref) each
    auto evaluate = [&](int cnt, bool map, float* map_out) -> cudaError_t {
        cudaError_t ee;
        if ((ee = cudaMemcpyAsync(d_img, hi.data(), sizeof(Img) * cnt, cudaMemcpyHostToDevice, st)) != cudaSuccess) return ee;
        if ((ee = cudaMemsetAsync(d_sums, 0, sizeof(double) * 3 * cnt, st)) != cudaSuccess) return ee;
        int rmax = 0;
        for (int i = 0; i < cnt; ++i) rmax = std::max(rmax, hi[i].radius);
        row_pass_kernel<<<dim3(Hc, cnt), 256, sizeof(float) * (kMaxRadius + 1 + Wc + 2 * rmax), st>>>(
            d_base, d_img, W, cb, cb, Wc, Hc, tmp);
        col_pass_kernel<<<dim3((Wc + 31) / 32, (Hc + kRowTile - 1) / kRowTile, cnt), 256,
                          sizeof(float) * (kMaxRadius + 1 + (size_t)(kRowTile + 2 * rmax) * 32), st>>>(
            d_base, d_img, tmp, W, cb, cb, Wc, Hc, d_sums, d_ab, map ? map_out : nullptr);
        if ((ee = cudaGetLastError()) != cudaSuccess) return ee;
        if (!map && (ee = cudaMemcpyAsync(hs.data(), d_sums, sizeof(double) * 3 * cnt, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return ee;
        return cudaStreamSynchronize(st);
    };
    for (int b0 = 0; b0 < n; b0 += batch) {
        const int cnt = std::min(batch, n - b0);
        // reference sums
        std::vector<double> rs(2 * cnt);
        for (int i = 0; i < cnt; ++i) hi[i] = Img{sr_offsets[b0 + i], ref_offsets[b0 + i], 0.f, 0};
        SQ(cudaMemcpyAsync(d_img, hi.data(), sizeof(Img) * cnt, cudaMemcpyHostToDevice, st));
        SQ(cudaMemsetAsync(d_sums, 0, sizeof(double) * 2 * cnt, st));
        ref_stats_kernel<<<dim3(64, cnt), 256, 0, st>>>(d_base, d_img, W, cb, cb, Wc, Hc, d_sums);
        SQ(cudaGetLastError());
        SQ(cudaMemcpyAsync(rs.data(), d_sums, sizeof(double) * 2 * cnt, cudaMemcpyDeviceToHost, st));
        SQ(cudaStreamSynchronize(st));
        std::vector<double> best(cnt);
        if (p->fix_sigma) {
            for (int i = 0; i < cnt; ++i) best[i] = sfix;
        } else {
            std::vector<Brent> br(cnt, Brent(0.0, smax));
            std::vector<int> act;
            std::vector<double> xs;
            for (;;) {
                act.clear();
                xs.clear();
                for (int i = 0; i < cnt; ++i) {
                    double x;
                    if (br[i].propose(x)) {
                        act.push_back(i);
                        xs.push_back(x);
                    }
                }
                if (act.empty()) break;
                for (size_t q = 0; q < act.size(); ++q) {
                    const int i = act[q];
                    hi[q] = Img{sr_offsets[b0 + i], ref_offsets[b0 + i], (float)xs[q], kernel_radius((float)xs[q])};
                }
                SQ(evaluate((int)act.size(), false, nullptr));
                for (size_t q = 0; q < act.size(); ++q) {
                    const int i = act[q];
                    const Fit f = fit_from_sums(npx, hs[3 * q], hs[3 * q + 1], hs[3 * q + 2], rs[2 * i], rs[2 * i + 1]);
                    br[i].tell(f.rmse);
                }
            }
            for (int i = 0; i < cnt; ++i) best[i] = br[i].best_x;
        }
        // final fit at the chosen sigma, then the error maps
        for (int i = 0; i < cnt; ++i)
            hi[i] = Img{sr_offsets[b0 + i], ref_offsets[b0 + i], (float)best[i], kernel_radius((float)best[i])};
        SQ(evaluate(cnt, false, nullptr));
        std::vector<float> ab(2 * cnt);
        for (int i = 0; i < cnt; ++i) {
            const Fit f = fit_from_sums(npx, hs[3 * i], hs[3 * i + 1], hs[3 * i + 2], rs[2 * i], rs[2 * i + 1]);
            if (sigma) sigma[b0 + i] = (float)best[i];
            if (alpha) alpha[b0 + i] = (float)f.alpha;
            if (beta) beta[b0 + i] = (float)f.beta;
            if (rse) rse[b0 + i] = (float)f.rmse;
            if (rsp) rsp[b0 + i] = (float)f.ppmcc;
            ab[2 * i] = (float)f.alpha;
            ab[2 * i + 1] = (float)f.beta;
        }
        if (d_error_maps) {
            SQ(cudaMemcpyAsync(d_ab, ab.data(), sizeof(float) * 2 * cnt, cudaMemcpyHostToDevice, st));
            SQ(evaluate(cnt, true, d_error_maps + (size_t)b0 * Wc * Hc));
        }
    }
#undef SQ
    return ESRRF_OK;
}

}  // extern "C"
