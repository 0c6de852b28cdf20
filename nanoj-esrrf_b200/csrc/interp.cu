// interp.cu -- Fourier (Hartley) interpolation of frames by the magnification on the GPU.
//
// Replaces the per-frame CPU loop FourierInterpolation.fhtSpaceInterpolation
// (FourierInterpolation.java:12-73) that LiveSRRF_CL.prepareDataFHT_SRRF runs before every
// upload (LiveSRRF_CL.java:598-617).  The reference's transform is nanoj.core2.NanoJFHT
// (NanoJ-Core, not vendored); this file implements the map that its call sites define -- mirror
// padding to a power-of-two square (FourierInterpolation.java:118-172), forward 2-D Hartley
// transform, spectral index remap p -> p (p < N/2) or p + (M-1) N (:33-42), inverse transform on
// the magnified canvas, crop (:49-56) -- in closed form: a separable Dirichlet-kernel product
// (two batched GEMMs) plus four rank-one terms from the Hartley spectrum's unpaired Nyquist row
// and column.
#include <math.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "esrrf_internal.h"

namespace esrrf {

namespace {

// Power-of-two size that mirrorPaddingEvenSquare pads to (FourierInterpolation.java:125-130).
int pow2_ceil_java(int n) {
    int b = (int)std::ceil(std::log((double)n) / std::log(2.0));
    return (int)std::pow(2.0, (double)b);
}

// Source index along one axis of padded position c (mirror tiling with an odd number of tiles,
// centre tile unflipped, then a centred crop of length out_dim; FourierInterpolation.java:138-171).
int mirror_src(int c, int n, int out_dim) {
    int scale = (int)std::ceil((double)out_dim / n);
    if (scale % 2 == 0) scale += 1;
    const int roi = (scale * n - out_dim) / 2;
    const int pos = c + roi;
    const int tile = pos / n;
    const int i = pos - tile * n;
    const int rel = tile - (scale - 1) / 2;
    return (rel % 2 == 0) ? i : n - 1 - i;
}

// N-1-term Dirichlet kernel sum_{|k| < N/2} cos(k a), a = 2 pi j / NM, j in [0, NM).
double dirichlet(long j, int N, long NM) {
    if (j == 0) return (double)(N - 1);
    const double a = 2.0 * M_PI * (double)j / (double)NM;
    return std::sin((N - 1) * a / 2.0) / std::sin(a / 2.0);
}

template <class T>
cudaError_t upload(T** dptr, const std::vector<T>& host) {
    cudaError_t e = cudaMalloc((void**)dptr, sizeof(T) * host.size());
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dptr, host.data(), sizeof(T) * host.size(), cudaMemcpyHostToDevice);
}

__device__ __forceinline__ float load_raw(const void* raw, bool is_u16, long idx) {
    return is_u16 ? (float)__ldg((const unsigned short*)raw + idx) : __ldg((const float*)raw + idx);
}

// Alternating sums of the padded frame: wy[y] = sum_x (-1)^x X[y][x] and
// wx[x] = sum_y (-1)^y X[y][x].  Grid (ceil(N/32), frames), 32 warps: each CTA owns 32 rows (one
// per warp, lanes across the row) and 32 columns (lane = column, the warps splitting the rows),
// so that many independent loads are in flight (the sums are latency bound, not bandwidth bound).
__global__ void __launch_bounds__(1024) alt_sums_kernel(const void* raw, int is_u16, int w, int h,
                                                        int N, const int* __restrict__ srcx,
                                                        const int* __restrict__ srcy,
                                                        float* __restrict__ alt) {
    const int f = blockIdx.y;
    const void* frame = is_u16 ? (const void*)((const unsigned short*)raw + (long)f * w * h)
                               : (const void*)((const float*)raw + (long)f * w * h);
    float* out = alt + (long)f * (3 * N + 1);
    __shared__ double red[32][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int base = blockIdx.x * 32;
    {
        const int y = base + warp;
        if (y < N) {
            const long rowoff = (long)srcy[y] * w;
            double acc = 0.0, tot = 0.0;
#pragma unroll 8
            for (int x = lane; x < N; x += 32) {
                const float v = load_raw(frame, is_u16, rowoff + srcx[x]);
                acc += (x & 1) ? -(double)v : (double)v;
                tot += (double)v;
            }
            for (int o = 16; o > 0; o >>= 1) {
                acc += __shfl_xor_sync(0xffffffffu, acc, o);
                tot += __shfl_xor_sync(0xffffffffu, tot, o);
            }
            if (lane == 0) {
                out[y] = (float)acc;
                out[2 * N + 1 + y] = (float)tot;  // plain row sum, for the frame mean
            }
        }
    }
    const int x = base + lane;
    double acc = 0.0;
    if (x < N) {
        const int sx = srcx[x];
#pragma unroll 8
        for (int y = warp; y < N; y += 32) {
            const float v = load_raw(frame, is_u16, (long)srcy[y] * w + sx);
            acc += (y & 1) ? -(double)v : (double)v;
        }
    }
    red[warp][lane] = acc;
    __syncthreads();
    if (warp == 0 && x < N) {
        double t = 0.0;
        for (int i = 0; i < 32; ++i) t += red[i][lane];
        out[N + x] = (float)t;
    }
}

// Rank-one correction vectors per frame:
//   P = s_axis Dy wy,  T = s_axis Dy flip(wy) + s q cy,
//   Q = s_axis Dx wx + s q cx,  R = s_axis Dx flip(wx) + s q (cx + ux),
// flip(w)[m] = w[(N - m) mod N].  Dy, Dx already carry s_axis.
__global__ void __launch_bounds__(256) rank1_vectors_kernel(
    const float* __restrict__ alt, const float* __restrict__ dyT, const float* __restrict__ dxT,
    const float* __restrict__ cx, const float* __restrict__ ux, const float* __restrict__ cy,
    int N, int HM, int WM, float s_axis, float s, float* __restrict__ vec) {
    // grid ((HM + WM + 31) / 32, frames): 32 outputs per CTA (lane = output), the 8 warps each
    // summing every 8th term, partial sums combined in warp order
    extern __shared__ float wsh[];  // [2N]: wy then wx
    __shared__ float qred[8], mred[8];
    __shared__ float part[2][8][33];
    const int f = blockIdx.y;
    const float* a = alt + (long)f * (3 * N + 1);
    float qp = 0.f, mp = 0.f;  // q = sum_y (-1)^y wy[y]; frame sum from the row sums
    for (int i = threadIdx.x; i < 2 * N; i += blockDim.x) {
        const float v = a[i];
        wsh[i] = v;
        if (i < N) {
            qp += (i & 1) ? -v : v;
            mp += a[2 * N + 1 + i];
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        qp += __shfl_xor_sync(0xffffffffu, qp, o);
        mp += __shfl_xor_sync(0xffffffffu, mp, o);
    }
    if ((threadIdx.x & 31) == 0) {
        qred[threadIdx.x >> 5] = qp;
        mred[threadIdx.x >> 5] = mp;
    }
    __syncthreads();
    float q = 0.f, msum = 0.f;
    for (int i = 0; i < 8; ++i) {
        q += qred[i];
        msum += mred[i];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int e = blockIdx.x * 32 + lane;
    float* v = vec + (long)f * (2 * HM + 2 * WM + 1);
    // The dense passes interpolate X - c (c = frame mean) and add c s N^2 back: the map sends a
    // constant to (s N^2) times it, and the alternating sums of a constant vanish (N even), so
    // this only shrinks the GEMM summands.
    if (blockIdx.x == 0 && threadIdx.x == 0) v[2 * HM + 2 * WM] = msum / ((float)N * (float)N);
    float d0 = 0.f, d1 = 0.f;
    if (e < HM) {
#pragma unroll 4
        for (int y = warp; y < N; y += 8) {
            const float dv = dyT[(long)y * HM + e];
            d0 = fmaf(dv, wsh[y], d0);
            d1 = fmaf(dv, wsh[(N - y) & (N - 1)], d1);
        }
    } else if (e < HM + WM) {
        const int n = e - HM;
#pragma unroll 4
        for (int x = warp; x < N; x += 8) {
            const float dv = dxT[(long)x * WM + n];
            d0 = fmaf(dv, wsh[N + x], d0);
            d1 = fmaf(dv, wsh[N + ((N - x) & (N - 1))], d1);
        }
    }
    part[0][warp][lane] = d0;
    part[1][warp][lane] = d1;
    __syncthreads();
    if (warp != 0) return;
    d0 = 0.f;
    d1 = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        d0 += part[0][k][lane];
        d1 += part[1][k][lane];
    }
    if (e < HM) {
        v[e] = s_axis * d0;
        v[HM + e] = s_axis * d1 + s * q * cy[e];
    } else if (e < HM + WM) {
        const int n = e - HM;
        v[2 * HM + n] = s_axis * d0 + s * q * cx[n];
        v[2 * HM + WM + n] = s_axis * d1 + s * q * (cx[n] + ux[n]);
    }
}

// --------------------------------------------------------------------------------------------
// Batched FP32 GEMM, 128x128x8 CTA tile, 256 threads, 8x8 outputs per thread (two 4x4 quads
// 64 apart in each direction so that shared-memory reads are conflict free).
//   PASS 1: C[f] (N x WM)  = X_f (N x N, gathered through the padding tables) . dxT (N x WM)
//   PASS 2: C[f] (HM x WM) = dy (HM x N) . rowT[f] (N x WM) + rank-one epilogue
//   PASS 3: C[f] = A (shared, row-major Mr x K) . B[f] (K x Nc)           (adjoint, columns)
//   PASS 4: C[f] = A[f] (row-major Mr x K) . B (shared, K x Nc)           (adjoint, rows)
// --------------------------------------------------------------------------------------------
struct GemmArgs {
    int Mr, Nc, K;
    const void* raw;  // pass 1
    int is_u16, w, h;
    const int* srcx;
    const int* srcy;
    const float* A;   // pass 2: dy
    const float* B;   // pass 1: dxT; pass 2: rowT
    float* C;
    const float* vec; // pass 2 epilogue
    const float* cx;
    const float* ux;
    const float* cy;
    const float* uy;
    int HM, WM;
    float cscale;      // pass 2: s N^2 (1 for the mean-preserving scale)
};

template <int PASS>
__global__ void __launch_bounds__(256) gemm_kernel(GemmArgs g) {
    __shared__ __align__(16) float As[2][8][128];
    __shared__ __align__(16) float Bs[2][8][128];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int f = blockIdx.z;
    const int m0 = blockIdx.y * 128, n0 = blockIdx.x * 128;
    const float* Bf = (PASS == 1 || PASS == 4) ? g.B : g.B + (long)f * g.K * g.Nc;
    const float* Af = (PASS == 4) ? g.A + (long)f * g.Mr * g.K : g.A;
    const void* rawf = nullptr;
    float cmean = 0.f;
    if (PASS == 1) {
        rawf = g.is_u16 ? (const void*)((const unsigned short*)g.raw + (long)f * g.w * g.h)
                        : (const void*)((const float*)g.raw + (long)f * g.w * g.h);
        cmean = g.vec[(long)f * (2 * g.HM + 2 * g.WM + 1) + 2 * g.HM + 2 * g.WM];
    }

    // global-load mapping
    const int a_row = tid >> 1, a_k = (tid & 1) * 4;   // A: 128 rows x 8 k
    const int b_k = tid >> 5, b_col = (tid & 31) * 4;  // B: 8 k x 128 cols
    float ra[4], rb[4];

    auto load_tiles = [&](int k0) {
        const int m = m0 + a_row;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int k = k0 + a_k + i;
            float v = 0.f;
            if (m < g.Mr && k < g.K) {
                if (PASS == 1)
                    v = load_raw(rawf, g.is_u16, (long)__ldg(g.srcy + m) * g.w + __ldg(g.srcx + k)) - cmean;
                else
                    v = __ldg(Af + (long)m * g.K + k);
            }
            ra[i] = v;
        }
        const int kb = k0 + b_k;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int n = n0 + b_col + i;
            rb[i] = (kb < g.K && n < g.Nc) ? __ldg(Bf + (long)kb * g.Nc + n) : 0.f;
        }
    };
    auto store_tiles = [&](int buf) {
#pragma unroll
        for (int i = 0; i < 4; ++i) As[buf][a_k + i][a_row] = ra[i];
        *reinterpret_cast<float4*>(&Bs[buf][b_k][b_col]) = make_float4(rb[0], rb[1], rb[2], rb[3]);
    };

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

    load_tiles(0);
    store_tiles(0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < g.K; k0 += 8) {
        const bool more = k0 + 8 < g.K;
        if (more) load_tiles(k0 + 8);
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            float a[8], b[8];
            const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][64 + tx * 4]);
            a[0] = a0.x; a[1] = a0.y; a[2] = a0.z; a[3] = a0.w;
            a[4] = a1.x; a[5] = a1.y; a[6] = a1.z; a[7] = a1.w;
            b[0] = b0.x; b[1] = b0.y; b[2] = b0.z; b[3] = b0.w;
            b[4] = b1.x; b[5] = b1.y; b[6] = b1.z; b[7] = b1.w;
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        if (more) {
            store_tiles(buf ^ 1);
            __syncthreads();
            buf ^= 1;
        }
    }

    float* Cf = g.C + (long)f * g.Mr * g.Nc;
    const float* vec = (PASS == 2) ? g.vec + (long)f * (2 * g.HM + 2 * g.WM + 1) : nullptr;
    const float cback = (PASS == 2) ? vec[2 * g.HM + 2 * g.WM] * g.cscale : 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int m = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        if (m >= g.Mr) continue;
        float pm = 0.f, tm = 0.f, cym = 0.f, uym = 0.f;
        if (PASS == 2) {
            pm = vec[m];
            tm = vec[g.HM + m];
            cym = g.cy[m];
            uym = g.uy[m];
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int n = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
            if (n >= g.Nc) continue;
            float v = acc[i][j];
            if (PASS == 2) {
                const float qn = vec[2 * g.HM + n], rn = vec[2 * g.HM + g.WM + n];
                v += pm * g.cx[n] + cym * qn - uym * rn - tm * g.ux[n] + cback;
            }
            Cf[(long)m * g.Nc + n] = v;
        }
    }
}

// Adjoint of the rank-one terms, step 1: per frame, G c_x and G u_x (rows of G = dL/dI'),
// G^T c_y and G^T u_y (columns).  Grid (ceil((HM+WM)/8), F), one warp per row or column.
__global__ void __launch_bounds__(256) adj_proj_kernel(const float* __restrict__ G, int HM, int WM,
                                                       const float* __restrict__ cx,
                                                       const float* __restrict__ ux,
                                                       const float* __restrict__ cy,
                                                       const float* __restrict__ uy,
                                                       float* __restrict__ proj) {
    const int f = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const int e = blockIdx.x * 8 + (threadIdx.x >> 5);
    const float* Gf = G + (long)f * HM * WM;
    float* pr = proj + (long)f * (2 * HM + 2 * WM);
    if (e < HM) {
        float a = 0.f, b = 0.f;
        for (int x = lane; x < WM; x += 32) {
            const float g = Gf[(long)e * WM + x];
            a = fmaf(g, cx[x], a);
            b = fmaf(g, ux[x], b);
        }
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (lane == 0) {
            pr[e] = a;
            pr[HM + e] = b;
        }
    } else if (e < HM + WM) {
        const int x = e - HM;
        float a = 0.f, b = 0.f;
        for (int y = lane; y < HM; y += 32) {
            const float g = Gf[(long)y * WM + x];
            a = fmaf(g, cy[y], a);
            b = fmaf(g, uy[y], b);
        }
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (lane == 0) {
            pr[2 * HM + x] = a;
            pr[2 * HM + WM + x] = b;
        }
    }
}

// Adjoint of the rank-one terms, step 2 (forward: P = s_a Dy wy, T = s_a Dy flip(wy) + s q cy,
// Q = s_a Dx wx + s q cx, R = s_a Dx flip(wx) + s q (cx + ux); I' += P cx' + cy Q' - uy R' - T ux'):
//   dwy[m] = s_a (Dy' Gc)[m] - s_a (Dy' Gu)[(N-m)%N]
//   dwx[m] = s_a (Dx' Gtc)[m] - s_a (Dx' Gtu)[(N-m)%N]
//   dq     = s (cy.Gc - uy.(Gc + Gu) - cy.Gu)
// Grid (ceil(2N/32), F); output m < N is dwy[m], N <= m < 2N is dwx[m - N]; block 0 also
// reduces dq.  dx is Dx row-major [WM][N] (scaled like dxT).
__global__ void __launch_bounds__(256) adj_rank1_kernel(const float* __restrict__ proj,
                                                        const float* __restrict__ dy,
                                                        const float* __restrict__ dx, int N, int HM,
                                                        int WM, const float* __restrict__ cy,
                                                        const float* __restrict__ uy, float s_axis,
                                                        float s, float* __restrict__ dvec) {
    // 32 outputs per block (one per lane); the 8 warps split the rows and reduce in shared memory
    const int f = blockIdx.y;
    const float* pr = proj + (long)f * (2 * HM + 2 * WM);
    float* dv = dvec + (long)f * (2 * N + 1);
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const int m = blockIdx.x * 32 + lane;
    __shared__ float ra[8][32], rb[8][32];
    float a = 0.f, b = 0.f;
    if (m < N) {
        const int mf = (N - m) & (N - 1);
        for (int y = wq; y < HM; y += 8) {
            a = fmaf(dy[(long)y * N + m], pr[y], a);
            b = fmaf(dy[(long)y * N + mf], pr[HM + y], b);
        }
    } else if (m < 2 * N) {
        const int mm = m - N, mf = (N - mm) & (N - 1);
        for (int x = wq; x < WM; x += 8) {
            a = fmaf(dx[(long)x * N + mm], pr[2 * HM + x], a);
            b = fmaf(dx[(long)x * N + mf], pr[2 * HM + WM + x], b);
        }
    }
    ra[wq][lane] = a;
    rb[wq][lane] = b;
    __syncthreads();
    if (wq == 0 && m < 2 * N) {
        float A = 0.f, B = 0.f;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            A += ra[i][lane];
            B += rb[i][lane];
        }
        dv[m] = s_axis * (A - B);  // dv[m] (m < N) or dv[N + mm]
    }
    if (blockIdx.x == 0) {
        __shared__ float red[8];
        float q = 0.f;
        for (int y = threadIdx.x; y < HM; y += blockDim.x)
            q += cy[y] * pr[y] - uy[y] * (pr[y] + pr[HM + y]) - cy[y] * pr[HM + y];
        for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = q;
        __syncthreads();
        if (threadIdx.x == 0) {
            float t = 0.f;
            for (int i = 0; i < 8; ++i) t += red[i];
            dv[2 * N] = s * t;
        }
    }
}

// dL/draw: padded-frame gradient (dense part + rank-one part) scattered through the mirror
// padding tables, plus the frame-average term dF / T.  Grid (ceil(N/256), N, F).
__global__ void adj_scatter_kernel(const float* __restrict__ gX, const float* __restrict__ dvec,
                                   int N, int w, int h, const int* __restrict__ srcx,
                                   const int* __restrict__ srcy, int identity,
                                   float* __restrict__ graw) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const long f = blockIdx.z;
    if (x >= N) return;
    const float* dv = dvec + f * (2 * N + 1);
    const float vx = (x & 1) ? -1.f : 1.f, vy = (y & 1) ? -1.f : 1.f;
    const float val = gX[(f * N + y) * (long)N + x] + dv[y] * vx + vy * dv[N + x] + dv[2 * N] * vx * vy;
    float* dst = graw + f * (long)w * h + (long)srcy[y] * w + srcx[x];
    if (identity)
        *dst += val;
    else
        atomicAdd(dst, val);
}

}  // namespace

cudaError_t interp_adjoint_run(const InterpPlan& p, const float* dx, const float* gI, int F,
                               float* T1, float* gX, float* proj, float* dvec, float* graw,
                               cudaStream_t stream) {
    // graw must hold the frame-average term (or zeros) on entry; this adds L^T gI.
    const int N = p.N;
    GemmArgs g{};
    g.Mr = N;
    g.K = p.HM;
    g.Nc = p.WM;
    g.A = p.dyT;   // [N][HM]
    g.B = gI;      // [F][HM][WM]
    g.C = T1;      // [F][N][WM]
    gemm_kernel<3><<<dim3((g.Nc + 127) / 128, (g.Mr + 127) / 128, F), 256, 0, stream>>>(g);
    g.Mr = N;
    g.K = p.WM;
    g.Nc = N;
    g.A = T1;      // [F][N][WM]
    g.B = dx;      // [WM][N]
    g.C = gX;      // [F][N][N]
    gemm_kernel<4><<<dim3((g.Nc + 127) / 128, (g.Mr + 127) / 128, F), 256, 0, stream>>>(g);
    adj_proj_kernel<<<dim3((p.HM + p.WM + 7) / 8, F), 256, 0, stream>>>(gI, p.HM, p.WM, p.cx, p.ux,
                                                                         p.cy, p.uy, proj);
    adj_rank1_kernel<<<dim3((2 * N + 31) / 32, F), 256, 0, stream>>>(
        proj, p.dy, dx, N, p.HM, p.WM, p.cy, p.uy, (float)p.s_axis, (float)p.s, dvec);
    adj_scatter_kernel<<<dim3((N + 255) / 256, N, F), 256, 0, stream>>>(
        gX, dvec, N, p.w, p.h, p.srcx, p.srcy, p.identity_pad ? 1 : 0, graw);
    return cudaGetLastError();
}

cudaError_t interp_plan_create(InterpPlan& p, int w, int h, int M, int scale_mode) {
    p.w = w;
    p.h = h;
    p.M = M;
    const int bw = pow2_ceil_java(w), bh = pow2_ceil_java(h);
    p.N = std::max(bw, bh);
    const int N = p.N;
    const long NM = (long)N * M;
    p.WM = w * M;
    p.HM = h * M;
    p.xroi = (int)((NM - p.WM) / 2);
    p.yroi = (int)((NM - p.HM) / 2);
    p.identity_pad = (w == N && h == N);
    p.s_axis = scale_mode == 0 ? 1.0 / N : 1.0 / (double)NM;
    p.s = p.s_axis * p.s_axis;

    std::vector<int> sx(N), sy(N);
    for (int c = 0; c < N; ++c) {
        sx[c] = mirror_src(c, w, N);
        sy[c] = mirror_src(c, h, N);
    }
    std::vector<float> dxT((size_t)N * p.WM), dy((size_t)p.HM * N), dyT((size_t)N * p.HM);
    for (int n = 0; n < p.WM; ++n)
        for (int m = 0; m < N; ++m) {
            long j = ((long)m * M - (n + p.xroi)) % NM;
            if (j < 0) j += NM;
            dxT[(size_t)m * p.WM + n] = (float)(dirichlet(j, N, NM) * p.s_axis);
        }
    for (int n = 0; n < p.HM; ++n)
        for (int m = 0; m < N; ++m) {
            long j = ((long)m * M - (n + p.yroi)) % NM;
            if (j < 0) j += NM;
            const float v = (float)(dirichlet(j, N, NM) * p.s_axis);
            dy[(size_t)n * N + m] = v;
            dyT[(size_t)m * p.HM + n] = v;
        }
    std::vector<float> cx(p.WM), ux(p.WM), cy(p.HM), uy(p.HM);
    for (int n = 0; n < p.WM; ++n) {
        const double a = M_PI * (double)(n + p.xroi) / M;
        cx[n] = (float)std::cos(a);
        ux[n] = (float)std::sin(a);
    }
    for (int n = 0; n < p.HM; ++n) {
        const double a = M_PI * (double)(n + p.yroi) / M;
        cy[n] = (float)std::cos(a);
        uy[n] = (float)std::sin(a);
    }
    cudaError_t e;
    if ((e = upload(&p.dxT, dxT)) != cudaSuccess) return e;
    if ((e = upload(&p.dy, dy)) != cudaSuccess) return e;
    if ((e = upload(&p.dyT, dyT)) != cudaSuccess) return e;
    if ((e = upload(&p.cx, cx)) != cudaSuccess) return e;
    if ((e = upload(&p.ux, ux)) != cudaSuccess) return e;
    if ((e = upload(&p.cy, cy)) != cudaSuccess) return e;
    if ((e = upload(&p.uy, uy)) != cudaSuccess) return e;
    if ((e = upload(&p.srcx, sx)) != cudaSuccess) return e;
    if ((e = upload(&p.srcy, sy)) != cudaSuccess) return e;
    // Tensor-core passes on compute capability 10.x unless ESRRF_INTERP_GEMM=simt selects the
    // FP32 SIMT kernels.
    const char* sel = std::getenv("ESRRF_INTERP_GEMM");
    int dev = 0, major = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev)) != cudaSuccess)
        return e;
    p.tc = major == 10 && tc_interp_supported(p) && !(sel && std::strcmp(sel, "simt") == 0);
    if (p.tc) return tc_plan_tables(p, dxT, dy);
    return cudaSuccess;
}

void interp_plan_destroy(InterpPlan& p) {
    cudaFree(p.dxT);
    cudaFree(p.dy);
    cudaFree(p.dyT);
    cudaFree(p.cx);
    cudaFree(p.ux);
    cudaFree(p.cy);
    cudaFree(p.uy);
    cudaFree(p.srcx);
    cudaFree(p.srcy);
    cudaFree(p.dxp);
    cudaFree(p.dyp);
    cudaFree(p.tc_err);
    p = InterpPlan();
}

cudaError_t interp_run(const InterpPlan& p, InterpScratch& sc, const void* raw, bool is_u16, int F,
                       float* out, cudaStream_t stream, int* launches) {
    if (F <= 0) return cudaSuccess;
    if (F > sc.capacity) return cudaErrorInvalidValue;
    const int N = p.N;
    alt_sums_kernel<<<dim3((N + 31) / 32, F), 1024, 0, stream>>>(raw, is_u16 ? 1 : 0, p.w, p.h, N,
                                                               p.srcx, p.srcy, sc.alt);
    {
        dim3 grid((p.HM + p.WM + 31) / 32, F);
        rank1_vectors_kernel<<<grid, 256, sizeof(float) * 2 * N, stream>>>(
            sc.alt, p.dyT, p.dxT, p.cx, p.ux, p.cy, N, p.HM, p.WM, (float)p.s_axis, (float)p.s,
            sc.vec);
    }
    if (p.tc) {
        if (launches) *launches += 5;  // sums, rank-one vectors, split operands, two passes
        cudaError_t e = cudaGetLastError();
        return e != cudaSuccess ? e : tc_interp_passes(p, sc, raw, is_u16, F, out, stream);
    }
    GemmArgs g{};
    g.raw = raw;
    g.is_u16 = is_u16 ? 1 : 0;
    g.w = p.w;
    g.h = p.h;
    g.srcx = p.srcx;
    g.srcy = p.srcy;
    g.HM = p.HM;
    g.WM = p.WM;
    g.vec = sc.vec;
    g.cscale = (float)(p.s * (double)N * (double)N);
    // pass 1: rows of the padded frame times dxT
    g.Mr = N;
    g.Nc = p.WM;
    g.K = N;
    g.B = p.dxT;
    g.C = sc.rowT;
    {
        dim3 grid((g.Nc + 127) / 128, (g.Mr + 127) / 128, F);
        gemm_kernel<1><<<grid, 256, 0, stream>>>(g);
    }
    // pass 2: dy times the first-pass rows, plus the rank-one epilogue
    g.Mr = p.HM;
    g.Nc = p.WM;
    g.K = N;
    g.A = p.dy;
    g.B = sc.rowT;
    g.C = out;
    g.vec = sc.vec;
    g.cx = p.cx;
    g.ux = p.ux;
    g.cy = p.cy;
    g.uy = p.uy;
    {
        dim3 grid((g.Nc + 127) / 128, (g.Mr + 127) / 128, F);
        gemm_kernel<2><<<grid, 256, 0, stream>>>(g);
    }
    if (launches) *launches += 4;
    return cudaGetLastError();
}

}  // namespace esrrf

namespace esrrf {

// Same tables as interp_plan_create, laid out in caller-provided device memory from `base`
// (each piece 256-byte aligned) instead of fresh allocations.  With base == nullptr only the
// byte count is computed.  Host tables are staged by pageable cudaMemcpyAsync on `stream`,
// which copies them out before returning.
cudaError_t interp_plan_place(InterpPlan& p, int w, int h, int M, int scale_mode,
                              unsigned char* base, size_t* bytes, cudaStream_t stream) {
    p.w = w;
    p.h = h;
    p.M = M;
    p.N = std::max(pow2_ceil_java(w), pow2_ceil_java(h));
    const int N = p.N;
    const long NM = (long)N * M;
    p.WM = w * M;
    p.HM = h * M;
    p.xroi = (int)((NM - p.WM) / 2);
    p.yroi = (int)((NM - p.HM) / 2);
    p.identity_pad = (w == N && h == N);
    p.s_axis = scale_mode == 0 ? 1.0 / N : 1.0 / (double)NM;
    p.s = p.s_axis * p.s_axis;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t n_dxT = (size_t)N * p.WM, n_dy = (size_t)p.HM * N;
    size_t off = 0;
    const size_t o_dxT = off; off += al(sizeof(float) * n_dxT);
    const size_t o_dy = off;  off += al(sizeof(float) * n_dy);
    const size_t o_dyT = off; off += al(sizeof(float) * n_dy);
    const size_t o_cx = off;  off += al(sizeof(float) * p.WM);
    const size_t o_ux = off;  off += al(sizeof(float) * p.WM);
    const size_t o_cy = off;  off += al(sizeof(float) * p.HM);
    const size_t o_uy = off;  off += al(sizeof(float) * p.HM);
    const size_t o_sx = off;  off += al(sizeof(int) * N);
    const size_t o_sy = off;  off += al(sizeof(int) * N);
    *bytes = off;
    if (!base) return cudaSuccess;
    p.dxT = (float*)(base + o_dxT);
    p.dy = (float*)(base + o_dy);
    p.dyT = (float*)(base + o_dyT);
    p.cx = (float*)(base + o_cx);
    p.ux = (float*)(base + o_ux);
    p.cy = (float*)(base + o_cy);
    p.uy = (float*)(base + o_uy);
    p.srcx = (int*)(base + o_sx);
    p.srcy = (int*)(base + o_sy);
    std::vector<int> sx(N), sy(N);
    for (int c = 0; c < N; ++c) {
        sx[c] = mirror_src(c, w, N);
        sy[c] = mirror_src(c, h, N);
    }
    std::vector<float> dxT(n_dxT), dy(n_dy), dyT(n_dy);
    for (int n = 0; n < p.WM; ++n)
        for (int m = 0; m < N; ++m) {
            long j = ((long)m * M - (n + p.xroi)) % NM;
            if (j < 0) j += NM;
            dxT[(size_t)m * p.WM + n] = (float)(dirichlet(j, N, NM) * p.s_axis);
        }
    for (int n = 0; n < p.HM; ++n)
        for (int m = 0; m < N; ++m) {
            long j = ((long)m * M - (n + p.yroi)) % NM;
            if (j < 0) j += NM;
            const float v = (float)(dirichlet(j, N, NM) * p.s_axis);
            dy[(size_t)n * N + m] = v;
            dyT[(size_t)m * p.HM + n] = v;
        }
    std::vector<float> cx(p.WM), ux(p.WM), cy(p.HM), uy(p.HM);
    for (int n = 0; n < p.WM; ++n) {
        const double a = M_PI * (double)(n + p.xroi) / M;
        cx[n] = (float)std::cos(a);
        ux[n] = (float)std::sin(a);
    }
    for (int n = 0; n < p.HM; ++n) {
        const double a = M_PI * (double)(n + p.yroi) / M;
        cy[n] = (float)std::cos(a);
        uy[n] = (float)std::sin(a);
    }
    cudaError_t e;
    const cudaMemcpyKind k = cudaMemcpyHostToDevice;
    if ((e = cudaMemcpyAsync(p.dxT, dxT.data(), sizeof(float) * n_dxT, k, stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(p.dy, dy.data(), sizeof(float) * n_dy, k, stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(p.dyT, dyT.data(), sizeof(float) * n_dy, k, stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(p.cx, cx.data(), sizeof(float) * p.WM, k, stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(p.ux, ux.data(), sizeof(float) * p.WM, k, stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(p.cy, cy.data(), sizeof(float) * p.HM, k, stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(p.uy, uy.data(), sizeof(float) * p.HM, k, stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(p.srcx, sx.data(), sizeof(int) * N, k, stream)) != cudaSuccess) return e;
    return cudaMemcpyAsync(p.srcy, sy.data(), sizeof(int) * N, k, stream);
}

}  // namespace esrrf
