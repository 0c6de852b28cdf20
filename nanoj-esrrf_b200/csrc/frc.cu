// frc.cu -- Fourier ring correlation and FIRE resolution of image pairs (the sweep's odd/even
// reconstructions, gui/ParametersSweep_.java:403-447: FRC.calculateFireNumber(odd, even,
// FIXED_1_OVER_7) x the output pixel size).
//
// NanoJ-Core's FRC class is not in the reference tree, so the published method (Nieuwenhuizen et
// al., Nat. Methods 10:557, 2013) is restated with these choices, identical in the oracle:
//   1. each image minus its mean, times a separable Tukey window (cosine tapers over the outer
//      TAPER/2 of each axis), placed at the origin of an N x N zero plane, N the next power of
//      two >= max(width, height, 32);
//   2. F = 2-D DFT (own radix-2 FFT: rows in shared memory, a tiled transpose, rows again -- the
//      ring sums are symmetric in the two axes, so the spectrum is used transposed);
//   3. ring r holds the frequencies (u, v), |u|, |v| <= N/2 (signed), with round(sqrt(u^2 + v^2))
//      = r, decided exactly in integers; r = 0 .. N/2;
//   4. FRC(r) = sum Re(F1 conj F2) / sqrt(sum |F1|^2 sum |F2|^2) (FP64 sums);
//   5. FIRE: the first ring r >= 1 with FRC(r) < 1/7; for r >= 2 the crossing q is interpolated
//      linearly between rings r - 1 and r and the resolution is N / q pixels x pixel_size; NaN when
//      FRC(1) is already below 1/7 or the curve never drops below it (ring 0, the mean, is not used).
#include <math.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "esrrf.h"

namespace {

constexpr int kMaxLogN = 12;  // N <= 4096
constexpr float kTaper = 0.25f;

std::mutex g_mu;
std::string g_err;

esrrf_status fail(const std::string& m, esrrf_status s = ESRRF_ERR_INVALID) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_err = m;
    return s;
}

int padded_size(int w, int h) {
    int n = 32;  // at least one 32 x 32 transpose tile
    while (n < std::max(w, h)) n <<= 1;
    return n;
}

__device__ __forceinline__ float tukey(int i, int n) {
    // 1 inside, 0.5 (1 - cos(pi x / a)) over the outer a = TAPER (n - 1) / 2 samples
    const float a = kTaper * (float)(n - 1) * 0.5f;
    const float x = fminf((float)i, (float)(n - 1 - i));
    if (a <= 0.f || x >= a) return 1.f;
    return 0.5f * (1.f - cospif(x / a));
}

// image means, FP64, one block per image
__global__ void mean_kernel(const float* __restrict__ base, const size_t* __restrict__ offs, int w, int h,
                            double* __restrict__ mean) {
    const float* img = base + offs[blockIdx.x];
    double s = 0.0;
    for (long i = threadIdx.x; i < (long)w * h; i += blockDim.x) s += img[i];
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) mean[blockIdx.x] = s / ((double)w * h);
    }
}

// tapered, zero-padded complex rows (image at the origin); grid (N, images)
__global__ void load_kernel(const float* __restrict__ base, const size_t* __restrict__ offs, int w, int h, int N,
                            const double* __restrict__ mean, float2* __restrict__ out) {
    const int img = blockIdx.y, y = blockIdx.x;
    float2* row = out + ((long)img * N + y) * N;
    const float* src = base + offs[img];
    const float m = (float)mean[img];
    const float wy = y < h ? tukey(y, h) : 0.f;
    for (int x = threadIdx.x; x < N; x += blockDim.x) {
        float v = 0.f;
        if (y < h && x < w) v = (src[(long)y * w + x] - m) * wy * tukey(x, w);
        row[x] = make_float2(v, 0.f);
    }
}

// one row of length N = 2^logN per block: bit-reversed load, radix-2 stages, twiddles from a
// per-block table exp(-2 pi i k / N)
__global__ void fft_rows_kernel(float2* __restrict__ data, int logN) {
    extern __shared__ float2 sm[];
    const int N = 1 << logN;
    float2* s = sm;
    float2* tw = sm + N;
    float2* row = data + (long)blockIdx.x * N;
    for (int k = threadIdx.x; k < N / 2; k += blockDim.x) {
        float sn, cs;
        sincospif(-2.f * (float)k / (float)N, &sn, &cs);
        tw[k] = make_float2(cs, sn);
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) s[__brev((unsigned)i) >> (32 - logN)] = row[i];
    __syncthreads();
    for (int ls = 0; ls < logN; ++ls) {
        const int half = 1 << ls;
        for (int j = threadIdx.x; j < N / 2; j += blockDim.x) {
            const int pos = j & (half - 1);
            const int i0 = ((j >> ls) << (ls + 1)) + pos, i1 = i0 + half;
            const float2 t = tw[pos << (logN - 1 - ls)];
            const float2 a = s[i0], b = s[i1];
            const float2 bt = make_float2(b.x * t.x - b.y * t.y, b.x * t.y + b.y * t.x);
            s[i0] = make_float2(a.x + bt.x, a.y + bt.y);
            s[i1] = make_float2(a.x - bt.x, a.y - bt.y);
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) row[i] = s[i];
}

// out[img][x][y] = in[img][y][x]; grid (N/32, N/32, images), 32 x 8 threads
__global__ void transpose_kernel(const float2* __restrict__ in, float2* __restrict__ out, int N) {
    __shared__ float2 t[32][33];
    const long off = (long)blockIdx.z * N * N;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += 8) t[j][threadIdx.x] = in[off + (long)(y0 + j) * N + x0 + threadIdx.x];
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) out[off + (long)(x0 + j) * N + y0 + threadIdx.x] = t[threadIdx.x][j];
}

// ring of (u, v): round(sqrt(u^2 + v^2)) in integers (r^2 - r + 1 <= k <= r^2 + r)
__device__ __forceinline__ int ring_of(int u, int v) {
    const int k = u * u + v * v;
    int r = (int)sqrtf((float)k);
    while (r * r > k) --r;
    while ((r + 1) * (r + 1) <= k) ++r;
    return k > r * r + r ? r + 1 : r;
}

// per (pair, chunk of rows): partial ring sums [3][R] in FP64; images 2p and 2p+1 of the batch
__global__ void ring_kernel(const float2* __restrict__ F, int N, int rows_per_chunk, int chunks,
                            double* __restrict__ part) {
    extern __shared__ double acc[];  // [3][R]
    const int R = N / 2 + 1;
    const int pair = blockIdx.y, chunk = blockIdx.x;
    for (int i = threadIdx.x; i < 3 * R; i += blockDim.x) acc[i] = 0.0;
    __syncthreads();
    const float2* A = F + (long)(2 * pair) * N * N;
    const float2* B = A + (long)N * N;
    const int r0 = chunk * rows_per_chunk, r1 = min(N, r0 + rows_per_chunk);
    for (long i = (long)r0 * N + threadIdx.x; i < (long)r1 * N; i += blockDim.x) {
        const int a = (int)(i / N), b = (int)(i - (long)a * N);
        const int u = a < N / 2 ? a : a - N, v = b < N / 2 ? b : b - N;
        const int r = ring_of(u, v);
        if (r >= R) continue;
        const float2 p = A[i], q = B[i];
        atomicAdd(&acc[r], (double)p.x * q.x + (double)p.y * q.y);
        atomicAdd(&acc[R + r], (double)p.x * p.x + (double)p.y * p.y);
        atomicAdd(&acc[2 * R + r], (double)q.x * q.x + (double)q.y * q.y);
    }
    __syncthreads();
    double* out = part + ((long)pair * chunks + chunk) * 3 * R;
    for (int i = threadIdx.x; i < 3 * R; i += blockDim.x) out[i] = acc[i];
}

// per pair (one thread): chunks summed in order, curve, FIRE
__global__ void fire_kernel(const double* __restrict__ part, int chunks, int N, int npairs, float pixel_size,
                            float* __restrict__ curves, float* __restrict__ fire) {
    const int pair = blockIdx.x * blockDim.x + threadIdx.x;
    if (pair >= npairs) return;
    const int R = N / 2 + 1;
    const double* p = part + (long)pair * chunks * 3 * R;
    double prev = 0.0;
    float res = NAN;
    bool found = false;
    for (int r = 0; r < R; ++r) {
        double c = 0.0, a = 0.0, b = 0.0;
        for (int k = 0; k < chunks; ++k) {
            c += p[(long)k * 3 * R + r];
            a += p[(long)k * 3 * R + R + r];
            b += p[(long)k * 3 * R + 2 * R + r];
        }
        const double frc = (a > 0.0 && b > 0.0) ? c / sqrt(a * b) : 0.0;
        if (curves) curves[(long)pair * R + r] = (float)frc;
        if (!found && r >= 1 && frc < 1.0 / 7.0) {
            found = true;
            if (r >= 2) {
                const double q = (r - 1) + (prev - 1.0 / 7.0) / (prev - frc);
                res = (float)((double)N / q * (double)pixel_size);
            }
        }
        prev = frc;
    }
    fire[pair] = res;
}

// Buffers of esrrf_frc, kept per device between calls (grow-only), as the SQUIRREL scratch: a
// call holds its device's lock throughout, so concurrent calls on one device run one after the
// other.
struct FrcScratch {
    std::mutex mu;
    void* buf[7] = {};
    size_t cap[7] = {};
};
FrcScratch g_frc[64];

// buffer i of the device's scratch with at least `bytes` (reallocated, after the stream drained,
// when it is smaller)
cudaError_t frc_buffer(FrcScratch& sc, int i, size_t bytes, cudaStream_t st, void** out) {
    if (sc.cap[i] < bytes) {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
        cudaFree(sc.buf[i]);
        sc.buf[i] = nullptr;
        sc.cap[i] = 0;
        if ((e = cudaMalloc(&sc.buf[i], bytes)) != cudaSuccess) return e;
        sc.cap[i] = bytes;
    }
    *out = sc.buf[i];
    return cudaSuccess;
}

}  // namespace

extern "C" {

const char* esrrf_frc_last_error(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_err.c_str();
}

esrrf_status esrrf_frc_size(int width, int height, int* padded, int* n_rings) {
    if (width < 2 || height < 2) return fail("images must be at least 2 x 2");
    const int N = padded_size(width, height);
    if (N > (1 << kMaxLogN)) return fail("images larger than 4096 pixels a side");
    if (padded) *padded = N;
    if (n_rings) *n_rings = N / 2 + 1;
    return ESRRF_OK;
}

esrrf_status esrrf_frc(const esrrf_frc_params* p, int n, const float* d_base, const size_t* a_offsets,
                       const size_t* b_offsets, float* fire, float* curves) {
    if (!p || !d_base || !a_offsets || !b_offsets || !fire) return fail("null argument");
    if (n < 0) return fail("negative pair count");
    int N = 0, R = 0;
    if (esrrf_frc_size(p->width, p->height, &N, &R) != ESRRF_OK) return ESRRF_ERR_INVALID;
    if (n == 0) return ESRRF_OK;
    int logN = 0;
    while ((1 << logN) < N) ++logN;
    cudaStream_t st = (cudaStream_t)p->stream;
    // pairs per batch: two N x N complex planes each in two buffers, within ~1 GB and the grid's
    // y limit (2 images per pair)
    const size_t plane = (size_t)N * N * sizeof(float2);
    const int batch = (int)std::max<size_t>(
        1, std::min<size_t>({(size_t)n, (1ull << 30) / (4 * plane), (size_t)16384}));
    const int rows_per_chunk = std::max(1, std::min(N, (1 << 16) / N));
    const int chunks = (N + rows_per_chunk - 1) / rows_per_chunk;
#define FK(call)                                                                   \
    do {                                                                           \
        cudaError_t _e = (call);                                                   \
        if (_e != cudaSuccess) return fail(cudaGetErrorString(_e), ESRRF_ERR_CUDA); \
    } while (0)
    int dev = 0;
    FK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail("device ordinal out of range");
    FrcScratch& sc = g_frc[dev];
    std::lock_guard<std::mutex> lk(sc.mu);
    void* bp[7] = {};
    FK(frc_buffer(sc, 0, 2 * plane * batch, st, &bp[0]));
    FK(frc_buffer(sc, 1, 2 * plane * batch, st, &bp[1]));
    FK(frc_buffer(sc, 2, sizeof(double) * 2 * batch, st, &bp[2]));
    FK(frc_buffer(sc, 3, sizeof(double) * 3 * R * (size_t)chunks * batch, st, &bp[3]));
    FK(frc_buffer(sc, 4, sizeof(size_t) * 2 * batch, st, &bp[4]));
    FK(frc_buffer(sc, 5, sizeof(float) * batch, st, &bp[5]));
    if (curves) FK(frc_buffer(sc, 6, sizeof(float) * R * (size_t)batch, st, &bp[6]));
    float2* F = static_cast<float2*>(bp[0]);
    float2* G = static_cast<float2*>(bp[1]);
    double* mean = static_cast<double*>(bp[2]);
    double* part = static_cast<double*>(bp[3]);
    size_t* d_offs = static_cast<size_t*>(bp[4]);
    float* d_fire = static_cast<float*>(bp[5]);
    float* d_curves = static_cast<float*>(bp[6]);
    const size_t fft_smem = sizeof(float2) * (N + N / 2);
    FK(cudaFuncSetAttribute(fft_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fft_smem));
    const size_t ring_smem = sizeof(double) * 3 * R;
    FK(cudaFuncSetAttribute(ring_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ring_smem));
    const int fft_threads = std::min(512, std::max(32, N / 2));
    std::vector<size_t> offs(2 * batch);
    for (int b0 = 0; b0 < n; b0 += batch) {
        const int nb = std::min(batch, n - b0);
        for (int i = 0; i < nb; ++i) {
            offs[2 * i] = a_offsets[b0 + i];
            offs[2 * i + 1] = b_offsets[b0 + i];
        }
        FK(cudaMemcpyAsync(d_offs, offs.data(), sizeof(size_t) * 2 * nb, cudaMemcpyHostToDevice, st));
        mean_kernel<<<2 * nb, 256, 0, st>>>(d_base, d_offs, p->width, p->height, mean);
        load_kernel<<<dim3(N, 2 * nb), 256, 0, st>>>(d_base, d_offs, p->width, p->height, N, mean, F);
        fft_rows_kernel<<<2 * nb * N, fft_threads, fft_smem, st>>>(F, logN);
        transpose_kernel<<<dim3(N / 32, N / 32, 2 * nb), dim3(32, 8), 0, st>>>(F, G, N);
        fft_rows_kernel<<<2 * nb * N, fft_threads, fft_smem, st>>>(G, logN);
        ring_kernel<<<dim3(chunks, nb), 256, ring_smem, st>>>(G, N, rows_per_chunk, chunks, part);
        fire_kernel<<<(nb + 127) / 128, 128, 0, st>>>(part, chunks, N, nb, p->pixel_size, d_curves, d_fire);
        FK(cudaGetLastError());
        FK(cudaMemcpyAsync(fire + b0, d_fire, sizeof(float) * nb, cudaMemcpyDeviceToHost, st));
        if (curves)
            FK(cudaMemcpyAsync(curves + (size_t)b0 * R, d_curves, sizeof(float) * R * nb, cudaMemcpyDeviceToHost, st));
        FK(cudaStreamSynchronize(st));
    }
#undef FK
    return ESRRF_OK;
}

}  // extern "C"
