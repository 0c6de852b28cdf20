/*
 * esrrf_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference eSRRF hot path.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it, as the checker; the product never routes through it.
 *
 * Parity status: the RGC, gradient, cumulant, MP-map and 3-D stages are pinned against the
 * reference's own OpenCL C kernels compiled on the host (oracle/_ref, fixtures under
 * tests/golden/).  The Fourier-interpolation stage restates FourierInterpolation.java, whose
 * transform lives in the un-vendored nanoj.core2.NanoJFHT (NanoJ-Core, version unpinned); it is
 * evaluated here from the definition of the 2-D discrete Hartley transform, so that stage is
 * "parity unpinned" against the reference itself.
 */
#include "esrrf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <tgmath.h>

#define ORC_F32 1
#define REAL float
#define SFX _f32
#include "esrrf_oracle_impl.h"
#undef ORC_F32
#undef REAL
#undef SFX

#define ORC_F32 0
#define REAL double
#define SFX _f64
#include "esrrf_oracle_impl.h"
#undef ORC_F32
#undef REAL
#undef SFX

void orc_robx_f32(const float* img, int width, int height, float* gx, float* gy) {
    robx_f32(img, width, height, gx, gy);
}

/* ------------------------------------------------------------------------------------------ */
/* Fourier interpolation (FourierInterpolation.java:12-73, 118-172).                           */
/* ------------------------------------------------------------------------------------------ */

/* Index of the padded-canvas pixel (along one axis) in the source image, following the mirror
 * tiling of mirrorPaddingEvenSquare: tile s of size n, centre tile unflipped, neighbours
 * alternately flipped, then a centred crop of length `out_dim`.  Returns the source index for
 * canvas position c in [0, out_dim). */
static int mirror_src(int c, int n, int out_dim) {
    int scale = (int)ceil((double)out_dim / n);
    if (scale % 2 == 0) scale += 1;
    const int roi = (scale * n - out_dim) / 2;
    const int pos = c + roi;
    const int tile = pos / n;
    const int i = pos - tile * n;
    const int rel = tile - (scale - 1) / 2; /* Java `%` keeps the sign; parity is what matters */
    return (rel % 2 == 0) ? i : n - 1 - i;
}

static int pow2_ceil(int n) {
    int b = (int)ceil(log((double)n) / log(2.0));
    return (int)pow(2.0, (double)b);
}

int orc_fht_interpolate(const float* raw, int n_frames, int w, int h, int M, int scale_mode,
                        float* out) {
    if (n_frames < 1 || w < 2 || h < 2 || M < 1) return -1;
    const int bw = pow2_ceil(w), bh = pow2_ceil(h);
    const int N = bw > bh ? bw : bh; /* padded square size */
    const int NM = N * M;            /* magnified canvas size */
    const int WM = w * M, HM = h * M;
    const int xroi = (NM - WM) / 2, yroi = (NM - HM) / 2;
    const double scale = scale_mode == 0 ? 1.0 / ((double)N * N) : 1.0 / ((double)NM * NM);
    const double twopi = 6.283185307179586476925286766559;
    const double tw = twopi / N, twM = twopi / NM;

    int* srcx = (int*)malloc(sizeof(int) * N);
    int* srcy = (int*)malloc(sizeof(int) * N);
    double* pad = (double*)malloc(sizeof(double) * N * N);
    double* c1 = (double*)malloc(sizeof(double) * N * N); /* sum_x f cos, [kx][y] */
    double* s1 = (double*)malloc(sizeof(double) * N * N); /* sum_x f sin, [kx][y] */
    double* H = (double*)malloc(sizeof(double) * N * N);  /* DHT, [ky][kx] */
    double* a2 = (double*)malloc(sizeof(double) * N * WM); /* [ky][nx] */
    double* b2 = (double*)malloc(sizeof(double) * N * WM);
    int* kmap = (int*)malloc(sizeof(int) * N);
    if (!srcx || !srcy || !pad || !c1 || !s1 || !H || !a2 || !b2 || !kmap) return -2;
    for (int c = 0; c < N; ++c) {
        srcx[c] = mirror_src(c, w, N);
        srcy[c] = mirror_src(c, h, N);
    }
    /* Spectrum remap (FourierInterpolation.java:33-42): p < N/2 keeps its index, the rest move
     * to p + (M-1) N, i.e. index p is the signed frequency p (p < N/2) or p - N. */
    for (int p = 0; p < N; ++p) kmap[p] = p < N / 2 ? p : p + (M - 1) * N;

    for (int f = 0; f < n_frames; ++f) {
        const float* img = raw + (long)f * w * h;
        for (int y = 0; y < N; ++y)
            for (int x = 0; x < N; ++x) pad[(long)y * N + x] = img[(long)srcy[y] * w + srcx[x]];
        /* Forward 2-D DHT H(kx,ky) = sum f(x,y) cas(tw (kx x + ky y)), via
         * cas(a + b) = cos a cas b + sin a cas(-b). */
#pragma omp parallel for schedule(static)
        for (int kx = 0; kx < N; ++kx)
            for (int y = 0; y < N; ++y) {
                double sc = 0, ss = 0;
                for (int x = 0; x < N; ++x) {
                    const double ang = tw * (double)(((long)kx * x) % N);
                    sc += pad[(long)y * N + x] * cos(ang);
                    ss += pad[(long)y * N + x] * sin(ang);
                }
                c1[(long)kx * N + y] = sc;
                s1[(long)kx * N + y] = ss;
            }
#pragma omp parallel for schedule(static)
        for (int ky = 0; ky < N; ++ky)
            for (int kx = 0; kx < N; ++kx) {
                double acc = 0;
                for (int y = 0; y < N; ++y) {
                    const double ang = tw * (double)(((long)ky * y) % N);
                    const double cp = cos(ang) + sin(ang), cm = cos(ang) - sin(ang);
                    acc += c1[(long)kx * N + y] * cp + s1[(long)kx * N + y] * cm;
                }
                H[(long)ky * N + kx] = acc;
            }
        /* Inverse DHT on the NM x NM canvas of the remapped spectrum, evaluated only at the
         * cropped output pixels: x'(nx,ny) = scale sum H(K) cas(twM (Kx nx + Ky ny)). */
#pragma omp parallel for schedule(static)
        for (int ky = 0; ky < N; ++ky)
            for (int ox = 0; ox < WM; ++ox) {
                const long nx = ox + xroi;
                double sa = 0, sb = 0;
                for (int kx = 0; kx < N; ++kx) {
                    const double ang = twM * (double)(((long)kmap[kx] * nx) % NM);
                    sa += H[(long)ky * N + kx] * cos(ang);
                    sb += H[(long)ky * N + kx] * sin(ang);
                }
                a2[(long)ky * WM + ox] = sa;
                b2[(long)ky * WM + ox] = sb;
            }
        float* o = out + (long)f * WM * HM;
#pragma omp parallel for schedule(static)
        for (int oy = 0; oy < HM; ++oy) {
            const long ny = oy + yroi;
            for (int ox = 0; ox < WM; ++ox) {
                double acc = 0;
                for (int ky = 0; ky < N; ++ky) {
                    const double ang = twM * (double)(((long)kmap[ky] * ny) % NM);
                    const double cp = cos(ang) + sin(ang), cm = cos(ang) - sin(ang);
                    acc += a2[(long)ky * WM + ox] * cp + b2[(long)ky * WM + ox] * cm;
                }
                o[(long)oy * WM + ox] = (float)(acc * scale);
            }
        }
    }
    free(srcx);
    free(srcy);
    free(pad);
    free(c1);
    free(s1);
    free(H);
    free(a2);
    free(b2);
    free(kmap);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* MFM reshape (LiveSRRF_CL.java:963-994).                                                     */
/* ------------------------------------------------------------------------------------------ */

int orc_mfm_reshape(const float* frames, int n_frames, int width, int height, int n_planes,
                    const float* roi, const float* coeff, float background, float* planes) {
    const int nsplit = 3;
    const int ws = width / nsplit, hs = height / nsplit;
    if (n_frames < 1 || ws < 1 || hs < 1 || n_planes < 1) return -1;
    for (int f = 0; f < n_frames; ++f) {
        const float* img = frames + (long)f * width * height;
        for (int z = 0; z < n_planes; ++z) {
            const int i = ((int)roi[z]) % 3;
            const int j = ((int)(roi[z] - (float)i)) / 3;
            /* Math.round(float) = floor(x + 0.5f) */
            const int x0 = (int)floorf((float)width / nsplit * i + 0.5f);
            const int y0 = (int)floorf((float)height / nsplit * j + 0.5f);
            for (int y = 0; y < hs; ++y)
                for (int x = 0; x < ws; ++x) {
                    const float p = img[(long)(y0 + y) * width + (x0 + x)];
                    planes[(((long)f * n_planes + z) * hs + y) * ws + x] = (p - background) / coeff[z];
                }
        }
    }
    return 0;
}
