// rgc_bic.cu -- the 2-D bicubic ("BIC") path: what LiveSRRF_CL runs with doFHTinterpolation off
// (prepareBuffersBICinterpolation loads liveSRRF.cl, LiveSRRF_CL.java:266-459), and the
// macro-pixel (MP) map correction shared with the 3-D path.
//
// Per frame: 2-point gradient on the raw frame (liveSRRF.cl:187-214), Catmull-Rom 2x resampling
// of the gradient (:217-233), RGC on the 2x gradient grid with bicubic intensity (:238-401).
// Each output pixel is one thread that walks the frames of a launch with its cumulants in
// registers; the reference instead relaunches per frame and read-modify-writes global memory.
#include <math.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "esrrf_internal.h"

namespace esrrf {

namespace {

using dev::cglh_power;
using dev::load_px;
using dev::sample2d;

__global__ void bic_grad_kernel(const void* raw, int is_u16, int w, int h, float* __restrict__ fraw,
                                float* __restrict__ gx, float* __restrict__ gy) {
    const int x1 = blockIdx.x * blockDim.x + threadIdx.x;
    const int y1 = blockIdx.y;
    const long f = blockIdx.z;
    if (x1 >= w) return;
    const long base = f * (long)w * h;
    const int x0 = max(x1 - 1, 0), y0 = max(y1 - 1, 0);
    const float p = load_px(raw, is_u16, base + (long)y1 * w + x1);
    fraw[base + (long)y1 * w + x1] = p;
    gx[base + (long)y1 * w + x1] = p - load_px(raw, is_u16, base + (long)y1 * w + x0);
    gy[base + (long)y1 * w + x1] = p - load_px(raw, is_u16, base + (long)y0 * w + x1);
}

// Generic 2x lateral resampling of `planes` consecutive [h][w] planes into [2h][2w].
__global__ void grad2x_kernel(const float* __restrict__ g, int w, int h, float* __restrict__ gi) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const long pl = blockIdx.z;
    if (x >= 2 * w) return;
    gi[pl * 4L * w * h + (long)y * 2 * w + x] =
        sample2d(g + pl * (long)w * h, w, h, (float)x / 2.0f, (float)y / 2.0f);
}

__global__ void __launch_bounds__(256) bic_rgc_kernel(BicRgcArgs a) {
    const long pix = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int WM = a.w * a.M, HM = a.h * a.M;
    const long whM = (long)WM * HM;
    if (pix >= whM) return;
    const int yM = (int)(pix / WM), xM = (int)(pix - (long)yM * WM);
    const int w2 = 2 * a.w, h2 = 2 * a.h;
    const int r0 = -(int)(2.0f * a.radius), r1 = (int)(2.0f * a.radius + 1);
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    float prev = a.st.prev[pix];
    for (int f = 0; f < a.F; ++f) {
        const float* gxi = a.gxi + (long)f * w2 * h2;
        const float* gyi = a.gyi + (long)f * w2 * h2;
        const float* fr = a.fraw + (long)f * a.w * a.h;
        // drift is stored x M by the host and used as raw-pixel units (liveSRRF.cl:263-264)
        const float sx = a.shift[f], sy = a.shift[a.F + f];
        const float xc = (float)(((double)xM + 0.5) / a.M + (double)sx);
        const float yc = (float)(((double)yM + 0.5) / a.M + (double)sy);
        const int kx = (int)(2.0f * xc), ky = (int)(2.0f * yc);
        float cglh = 0.f, wsum = 0.f;
        for (int j = r0; j <= r1; ++j) {
            const float vy = ((float)ky + (float)j) / 2.0f;
            if (!(vy > 0 && vy < (float)a.h)) continue;
            for (int i = r0; i <= r1; ++i) {
                const float vx = ((float)kx + (float)i) / 2.0f;
                if (!(vx > 0 && vx < (float)a.w)) continue;
                const float dx = vx - xc, dy = vy - yc;
                const float d = sqrtf(dx * dx + dy * dy);
                if (!(d != 0.f && d <= a.tSO)) continue;
                const int ax = min(max((int)(2 * ((double)vx - 0.5)), 0), w2 - 1);
                const int ay = min(max((int)(2 * ((double)vy - 0.5)), 0), h2 - 1);
                const int ax1 = min(max((int)(2 * ((double)vx - 0.5) + 1), 0), w2 - 1);
                const int ay1 = min(max((int)(2 * ((double)vy - 0.5) + 1), 0), h2 - 1);
                const float Gx = __ldg(gxi + (long)ay * w2 + ax1);
                const float Gy = __ldg(gyi + (long)ay1 * w2 + ax);
                float wt = d * expf(-(d * d) / a.tSS);
                wt = wt * wt * wt * wt;
                wsum += wt;
                if (Gx * dx + Gy * dy < 0) {
                    const float gm = sqrtf(Gx * Gx + Gy * Gy);
                    float dk = fabsf(Gy * dx - Gx * dy) / gm;
                    if (isnan(dk)) dk = d;
                    dk = 1 - dk / d;
                    cglh += dk * wt;
                }
            }
        }
        const float cg = cglh_power(cglh / wsum, a.sens);
        const float v = sample2d(fr, a.w, a.h, (float)xM / (float)a.M + sx - 0.5f,
                                 (float)yM / (float)a.M + sy - 0.5f);
        const float x = a.int_weighting ? v * cg : cg;
        s0 += x;
        s1 += (double)x * x;
        if (a.t0 + f > 0) s2 += (double)x * prev;
        s3 += v;
        prev = x;
    }
    a.st.acc[pix] += s0;
    a.st.acc[whM + pix] += s1;
    a.st.acc[2 * whM + pix] += s2;
    a.st.acc[3 * whM + pix] += s3;
    a.st.prev[pix] = prev;
}

// Mean of each sub-pixel phase of AVG, VAR and TAC2 over all macro-pixels
// (kernelCalculateMPmap, liveSRRF.cl:464-487, live3DSRRF.cl:561-588).  One CTA per phase.
__global__ void mp_map_kernel(const float* __restrict__ out, int w, int h, int P, int M, int is3d,
                              float* __restrict__ map) {
    const int phases = is3d ? M * M * M : M * M;
    const int idx = blockIdx.x;  // c * phases + phase
    const int c = idx / phases, ph = idx - c * phases;
    const int pz = is3d ? ph / (M * M) : 0;
    const int py = (ph - pz * M * M) / M;
    const int px = ph - pz * M * M - py * M;
    const long WM = (long)w * M, HM = (long)h * M, PM = is3d ? (long)P * M : 1;
    const long plane4 = WM * HM * PM;
    const long cells = (long)w * h * (is3d ? P : 1);
    double s = 0.0;
    for (long i = threadIdx.x; i < cells; i += blockDim.x) {
        const long z = i / ((long)w * h);
        const long r = i - z * w * h;
        const long y = r / w, x = r - (r / w) * w;
        const long zz = is3d ? pz + z * M : 0;
        s += out[c * plane4 + zz * WM * HM + (py + y * M) * WM + px + x * M];
    }
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) map[idx] = (float)(red[0] / (double)cells);
}

// Divide AVG, VAR, TAC2 by their phase means, then the readback's NaN->0
// (kernelCorrectMPmap, liveSRRF.cl:490-505, live3DSRRF.cl:591-611).
__global__ void mp_correct_kernel(float* __restrict__ out, int w, int h, int P, int M, int is3d,
                                  const float* __restrict__ map) {
    const long WM = (long)w * M, HM = (long)h * M, PM = is3d ? (long)P * M : 1;
    const long plane4 = WM * HM * PM;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 3 * plane4) return;
    const int c = (int)(idx / plane4);
    const long r = idx - c * plane4;
    const long zM = r / (WM * HM);
    const long yM = (r - zM * WM * HM) / WM;
    const long xM = r - zM * WM * HM - yM * WM;
    const int phases = is3d ? M * M * M : M * M;
    const int ph = (int)((is3d ? (zM % M) * M * M : 0) + (yM % M) * M + (xM % M));
    const float v = out[idx] / map[c * phases + ph];
    out[idx] = isnan(v) ? 0.f : v;
}

// Unit gradient on the 2x grid into the padded field, columns split by parity (column ax of
// parity ax & 1 at ax >> 1), so 32 consecutive cells of one phase read 32 consecutive entries.
// The reference reads Gx at (ay, ax + 1) and Gy at (ay + 1, ax) for a tap at ax = 2 (vx - 0.5)
// and takes the tap only if 0 < vx < w, i.e. 0 <= ax <= 2w - 2 (liveSRRF.cl:271-290): the last
// column and row hold a zero gradient, never inward, so out-of-range taps add nothing.
__global__ void unit_grad2d_kernel(const float* __restrict__ gxi, const float* __restrict__ gyi,
                                   int w, int h, int padx, int pady, int W2p, int H2p,
                                   float2* __restrict__ U) {
    const int ax = blockIdx.x * blockDim.x + threadIdx.x;
    const int ay = blockIdx.y;
    const long f = blockIdx.z;
    const int w2 = 2 * w, h2 = 2 * h;
    if (ax >= w2) return;
    float2 u = make_float2(0.f, 0.f);
    if (ax < w2 - 1 && ay < h2 - 1) {
        const long pl = f * w2 * h2;
        const float Gx = __ldg(gxi + pl + (long)ay * w2 + ax + 1);
        const float Gy = __ldg(gyi + pl + (long)(ay + 1) * w2 + ax);
        const float n2 = Gx * Gx + Gy * Gy;
        if (n2 > 0.f) {
            const float inv = rsqrtf(n2);
            u = make_float2(Gx * inv, Gy * inv);
        }
    }
    const int xp = ax + padx;  // padx is even: same parity as ax
    U[(f * H2p + ay + pady) * W2p + (xp & 1) * (W2p / 2) + (xp >> 1)] = u;
}

// Sum of weights over each output pixel's in-range taps (the reference's sum of w, in its tap
// order), once per handle: it depends on the pixel's phase and on how close it is to the edges.
__global__ void wsum2d_kernel(BicTables t, int w, int h, int M, float* __restrict__ out) {
    const int WM = w * M, HM = h * M;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)WM * HM) return;
    const int yM = (int)(idx / WM), xM = (int)(idx - (long)yM * WM);
    const int qx = xM / M, qy = yM / M;
    const int phase = (yM % M) * M + xM % M;
    float ws = 0.f;
    for (int k = t.start[phase]; k < t.start[phase + 1]; ++k) {
        const int2 s = t.node[k];
        const int ax = 2 * qx + s.x, ay = 2 * qy + s.y;
        if (ax < 0 || ax > 2 * w - 2 || ay < 0 || ay > 2 * h - 2) continue;
        ws += t.tw[k];
    }
    out[idx] = ws;
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
    // 8-byte asynchronous copy; valid = false writes zeros and reads nothing
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(valid ? 8 : 0)
                 : "memory");
}

// One thread per output pixel; a CTA is 32 x 8 input cells of one sub-pixel phase, so the whole
// CTA walks the same tap list (broadcast from shared memory).  Per frame the CTA's slab of the
// unit-gradient field (its 8 cell rows' 2x-grid rows plus the tap reach, both parity halves of
// its 32 cell columns plus the reach) is copied with cp.async into one of two buffers while the
// taps of the previous frame run.  Per tap: inward test g . d < 0, then Dk w = w - (w / d) |g x d|
// (liveSRRF.cl:293-339 with the gradient normalised once per node; a zero gradient is never
// inward, where the reference's NaN guard gives Dk = 0).  Sum of weights from the per-pixel
// table; intensity, cumulants and the (n - 1) bookkeeping as bic_rgc_kernel.  A launch's frames
// are summed in FP32 and folded into the block's FP64 accumulators once.
__global__ void __launch_bounds__(256, 4) bic_tab_kernel(BicTabArgs a) {
    extern __shared__ float4 smb[];
    const int M = a.M;
    // phase fastest: the M^2 CTAs that stage the same slab run together and share it through L2
    const int lp = blockIdx.x, px = lp % M, py = lp / M;
    const int bx = blockIdx.y, by = blockIdx.z;
    const int t0 = a.tab.start[lp], n = a.tab.start[lp + 1] - t0;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int row2 = 2 * a.tab.sl_nx;        // float2s per slab row
    const int slab = a.tab.sl_rows * row2;   // float2s per slab
    float4* stab = smb;                                                   // [max_taps]
    float* sw = reinterpret_cast<float*>(smb + a.tab.max_taps);          // [max_taps]
    float2* sbuf = reinterpret_cast<float2*>(smb + a.tab.max_taps + (a.tab.max_taps + 3) / 4);  // [2][slab]
    for (int i = tid; i < n; i += 256) {
        stab[i] = a.tab.tab[t0 + i];
        sw[i] = a.tab.tw[t0 + i];
    }
    const int qx_raw = bx * 32 + threadIdx.x, qy_raw = by * 8 + threadIdx.y;
    const bool valid = qx_raw < a.w && qy_raw < a.h;
    const int qx = min(qx_raw, a.w - 1), qy = min(qy_raw, a.h - 1);
    const int xM = qx * M + px, yM = qy * M + py;
    const int WM = a.w * M;
    const long pix = (long)yM * WM + xM;
    const long whM = (long)WM * a.h * M;
    const long fstride = (long)a.tab.H2p * a.tab.W2p;
    const long pl = (long)a.w * a.h;
    const int half = a.tab.W2p / 2;
    const int row0 = 16 * by + a.tab.pady + a.tab.sl_symin;
    const int cin0 = a.tab.padx / 2 + 32 * bx + a.tab.sl_fxmin;
    const int tbase = 2 * threadIdx.y * row2 + threadIdx.x;  // this thread's cell in the slab
    // the intensity is sampled at the same position in every frame
    const dev::Sample2dAt sp = dev::sample2d_at(a.w, a.h, (float)xM / (float)M - 0.5f, (float)yM / (float)M - 0.5f);
    const float wsum = a.tab.wsum[pix];
    const bool emit = a.cg_out != nullptr;
    float prev = valid && !emit ? a.st.prev[pix] : 0.f;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    // slab staging: warp ty copies rows ty, ty + 8, ...; lane tx the positions tx + 32 q of each
    // row, whose source column offsets (parity half + column; -1 beyond the field) are the same
    // for every row and frame (row2 <= 4 x 32, checked when the tables are built)
    int coff[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int rem = threadIdx.x + 32 * q;
        const int par = rem >= a.tab.sl_nx ? 1 : 0, cin = cin0 + rem - par * a.tab.sl_nx;
        coff[q] = rem < row2 && cin < half ? par * half + cin : -1;
    }
    auto stage = [&](int f) {
        const float2* Uf = a.U + f * fstride;
        float2* dst = sbuf + (f & 1) * slab;
        for (int ly = threadIdx.y; ly < a.tab.sl_rows; ly += 8) {
            const int row = row0 + ly;
            const bool rin = row < a.tab.H2p;
            const float2* src = Uf + (long)row * a.tab.W2p;
            float2* d = dst + ly * row2 + threadIdx.x;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if ((int)threadIdx.x + 32 * q >= row2) break;
                const bool in = rin && coff[q] >= 0;
                cp_async8(d + 32 * q, in ? (const void*)(src + coff[q]) : (const void*)a.U, in);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (a.F > 0) stage(0);
    for (int f = 0; f < a.F; ++f) {
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();  // slab f landed everywhere; buffer (f + 1) & 1 is no longer read
        if (f + 1 < a.F) stage(f + 1);
        const float2* sl = sbuf + (f & 1) * slab + tbase;
        float cg = 0.f;
        for (int t = 0; t < n; ++t) {
            const float4 e = stab[t];
            const float2 u = sl[__float_as_int(e.x)];
            const float dot = fmaf(u.x, e.y, u.y * e.z);
            // the term is computed for every tap so that only the add depends on the inward test
            const float cr = fmaf(u.y, e.y, -u.x * e.z);  // gy dx - gx dy
            const float term = fmaf(-fabsf(cr), e.w, sw[t]);
            if (dot < 0.f) cg += term;
        }
        const float v = dev::sample2d_apply(a.fraw + f * pl, a.w, sp);
        if (emit) {
            if (valid) {
                a.cg_out[(long)f * whM + pix] = cg / wsum;
                a.v_out[(long)f * whM + pix] = v;
            }
            continue;
        }
        const float c = cglh_power(cg / wsum, a.sens);
        const float x = a.int_weighting ? v * c : c;
        s0 += x;
        s1 = fmaf(x, x, s1);
        if (a.t0 + f > 0) s2 = fmaf(x, prev, s2);
        s3 += v;
        prev = x;
    }
    if (!valid || emit) return;
    a.st.acc[pix] += (double)s0;
    a.st.acc[whM + pix] += (double)s1;
    a.st.acc[2 * whM + pix] += (double)s2;
    a.st.acc[3 * whM + pix] += (double)s3;
    a.st.prev[pix] = prev;
}

}  // namespace

cudaError_t bic_tables_build(const BicGeometry& g, int M, int w, int h, BicTables& t, bool& built,
                             cudaStream_t stream) {
    // Tap geometry of bic_rgc_kernel with zero shift, for the pixel of each phase in the first
    // input cell (Java float arithmetic as the reference: xc = (float)((xM + 0.5) / M)); the
    // offsets from (kx, ky) and the distances repeat in every cell (exactly so for M a power of
    // two, whose phase centres are exact in FP32).
    built = false;
    const int r0 = -(int)(2.0f * g.radius), r1 = (int)(2.0f * g.radius + 1);
    struct Tap {
        int sx, sy;
        float dx, dy, d, wt;
    };
    std::vector<Tap> taps;
    std::vector<int> start(M * M + 1, 0);
    int sxmin = 0, sxmax = 0, symin = 0, symax = 0, maxn = 0;
    for (int py = 0; py < M; ++py)
        for (int px = 0; px < M; ++px) {
            const int phase = py * M + px;
            start[phase] = (int)taps.size();
            const float xc = (float)(((double)px + 0.5) / M);
            const float yc = (float)(((double)py + 0.5) / M);
            const int kx = (int)(2.0f * xc), ky = (int)(2.0f * yc);
            for (int j = r0; j <= r1; ++j) {
                const float vy = ((float)ky + (float)j) / 2.0f;
                for (int i = r0; i <= r1; ++i) {
                    const float vx = ((float)kx + (float)i) / 2.0f;
                    const float dx = vx - xc, dy = vy - yc;
                    const float d = sqrtf(dx * dx + dy * dy);
                    if (!(d != 0.f && d <= g.tSO)) continue;
                    float wt = d * expf(-(d * d) / g.tSS);
                    wt = wt * wt * wt * wt;
                    const Tap tp{kx + i - 1, ky + j - 1, dx, dy, d, wt};
                    sxmin = std::min(sxmin, tp.sx);
                    sxmax = std::max(sxmax, tp.sx);
                    symin = std::min(symin, tp.sy);
                    symax = std::max(symax, tp.sy);
                    taps.push_back(tp);
                }
            }
            maxn = std::max(maxn, (int)taps.size() - start[phase]);
        }
    start[M * M] = (int)taps.size();
    if (taps.empty()) return cudaSuccess;
    // zero halo: node column ax = 2 qx + sx in [sxmin, 2w - 2 + sxmax], rows likewise
    t.padx = std::max(-sxmin, std::max(sxmax - 1, 0));
    t.padx += t.padx & 1;
    t.pady = std::max(-symin, std::max(symax - 1, 0));
    t.W2p = 2 * w + 2 * t.padx;
    t.H2p = 2 * h + 2 * t.pady;
    const int fxmin = sxmin >> 1, fxmax = sxmax >> 1;
    t.sl_symin = symin;
    t.sl_fxmin = fxmin;
    t.sl_rows = 2 * 7 + symax - symin + 1;
    t.sl_nx = 31 + fxmax - fxmin + 1;
    t.max_taps = maxn;
    t.smem = sizeof(float4) * ((size_t)maxn + (maxn + 3) / 4) + sizeof(float2) * 2 * (size_t)t.sl_rows * 2 * t.sl_nx;
    // the kernel stages a slab row with at most 4 x 32 lanes' positions
    if (t.smem > 200 * 1024 || 2 * t.sl_nx > 128) return cudaSuccess;
    std::vector<float4> A;
    std::vector<float> Wt;
    std::vector<int2> node;
    for (const Tap& tp : taps) {
        const int off = (tp.sy - symin) * 2 * t.sl_nx + (tp.sx & 1) * t.sl_nx + ((tp.sx >> 1) - fxmin);
        float offf;
        std::memcpy(&offf, &off, 4);
        A.push_back(make_float4(offf, tp.dx, tp.dy, tp.wt / tp.d));
        Wt.push_back(tp.wt);
        node.push_back(make_int2(tp.sx, tp.sy));
    }
    auto up = [](auto** d, const auto& v) -> cudaError_t {
        cudaError_t e = cudaMalloc((void**)d, sizeof(v[0]) * v.size());
        if (e != cudaSuccess) return e;
        return cudaMemcpy(*d, v.data(), sizeof(v[0]) * v.size(), cudaMemcpyHostToDevice);
    };
    cudaError_t e;
    if ((e = up(&t.tab, A)) != cudaSuccess || (e = up(&t.tw, Wt)) != cudaSuccess ||
        (e = up(&t.node, node)) != cudaSuccess || (e = up(&t.start, start)) != cudaSuccess)
        return e;
    const long total = (long)w * M * h * M;
    if ((e = cudaMalloc((void**)&t.wsum, sizeof(float) * total)) != cudaSuccess) return e;
    wsum2d_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(t, w, h, M, t.wsum);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
    built = true;
    return cudaSuccess;
}

void bic_tables_free(BicTables& t) {
    cudaFree(t.tab);
    cudaFree(t.tw);
    cudaFree(t.node);
    cudaFree(t.start);
    cudaFree(t.wsum);
    t = BicTables();
}

size_t bic_field_float2s(const BicTables& t, int F) { return (size_t)F * t.H2p * t.W2p; }

cudaError_t unit_grad2d(const float* gxi, const float* gyi, int w, int h, int F, const BicTables& t,
                        float2* U, cudaStream_t stream) {
    unit_grad2d_kernel<<<dim3((2 * w + 127) / 128, 2 * h, F), 128, 0, stream>>>(
        gxi, gyi, w, h, t.padx, t.pady, t.W2p, t.H2p, U);
    return cudaGetLastError();
}

cudaError_t bic_rgc_tab(const BicTabArgs& a, cudaStream_t stream) {
    if (!a.tab.tab || a.tab.smem > 200 * 1024) return cudaErrorInvalidValue;
    static unsigned long long configured = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && !(configured & (1ull << dev))) {
        if ((e = cudaFuncSetAttribute(bic_tab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      200 * 1024)) != cudaSuccess)
            return e;
        configured |= 1ull << dev;
    }
    if ((a.w + 31) / 32 > 65535 || (a.h + 7) / 8 > 65535) return cudaErrorInvalidValue;
    const dim3 grid(a.M * a.M, (a.w + 31) / 32, (a.h + 7) / 8);
    bic_tab_kernel<<<grid, dim3(32, 8), a.tab.smem, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t bic_prepare(const void* raw, int is_u16, int w, int h, int F, float* fraw, float* gx,
                        float* gy, float* gxi, float* gyi, cudaStream_t stream) {
    bic_grad_kernel<<<dim3((w + 127) / 128, h, F), 128, 0, stream>>>(raw, is_u16, w, h, fraw, gx, gy);
    grad2x_kernel<<<dim3((2 * w + 127) / 128, 2 * h, F), 128, 0, stream>>>(gx, w, h, gxi);
    grad2x_kernel<<<dim3((2 * w + 127) / 128, 2 * h, F), 128, 0, stream>>>(gy, w, h, gyi);
    return cudaGetLastError();
}

cudaError_t grad2x(const float* g, int w, int h, int planes, float* gi, cudaStream_t stream) {
    grad2x_kernel<<<dim3((2 * w + 127) / 128, 2 * h, planes), 128, 0, stream>>>(g, w, h, gi);
    return cudaGetLastError();
}

cudaError_t bic_rgc(const BicRgcArgs& a, cudaStream_t stream) {
    const long whM = (long)a.w * a.M * a.h * a.M;
    bic_rgc_kernel<<<(unsigned)((whM + 255) / 256), 256, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t mp_correct(float* out, int w, int h, int P, int M, int is3d, float* map,
                       cudaStream_t stream) {
    const int phases = is3d ? M * M * M : M * M;
    mp_map_kernel<<<3 * phases, 256, 0, stream>>>(out, w, h, P, M, is3d, map);
    const long plane4 = (long)w * M * h * M * (is3d ? (long)P * M : 1);
    mp_correct_kernel<<<(unsigned)((3 * plane4 + 255) / 256), 256, 0, stream>>>(out, w, h, P, M, is3d, map);
    return cudaGetLastError();
}

}  // namespace esrrf
