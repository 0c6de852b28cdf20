/*
 * esrrf_oracle_impl.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Precision-generic body of the restatement; esrrf_oracle.c includes it twice, with
 * REAL=float/SFX=_f32 (reference expression order, the parity target) and
 * REAL=double/SFX=_f64 (the same algorithm in double precision).
 *
 * Parameters derived on the Java host (sigma, radius, 2 sigma^2, 2 sigma + 1) are always
 * computed in float exactly as LiveSRRF_CL.java does, because they define the algorithm;
 * only the per-pixel arithmetic changes precision.
 */
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

/* Catmull-Rom kernel, a = 0.5 (liveSRRF.cl:26-35). */
static REAL FN(cubic)(REAL x) {
    const REAL a = (REAL)0.5;
    if (x < 0) x = -x;
    REAL z = 0;
    if (x < 1)
        z = x * x * (x * (-a + (REAL)2) + (a - (REAL)3)) + (REAL)1;
    else if (x < 2)
        z = -a * x * x * x + (REAL)5 * a * x * x - (REAL)8 * a * x + (REAL)4 * a;
    return z;
}

/* Bicubic sample when the 4x4 support is interior, else bilinear with extrapolation
 * (liveSRRF.cl:39-133, liveSRRF_noInterpolation.cl:29-75, live3DSRRF.cl:42-140). */
static REAL FN(sample2d)(const REAL* a, int w, int h, REAL x, REAL y) {
    const int u0 = (int)floor((double)x);
    const int v0 = (int)floor((double)y);
    if (u0 > 0 && u0 < w - 2 && v0 > 0 && v0 < h - 2) {
        REAL q = 0;
        for (int j = 0; j <= 3; ++j) {
            int v = v0 - 1 + j;
            v = v < 0 ? 0 : (v > h - 1 ? h - 1 : v);
            REAL p = 0;
            for (int i = 0; i <= 3; ++i) {
                int u = u0 - 1 + i;
                u = u < 0 ? 0 : (u > w - 1 ? w - 1 : u);
                p = p + a[(long)v * w + u] * FN(cubic)(x - (REAL)u);
            }
            q = q + p * FN(cubic)(y - (REAL)v);
        }
        return q;
    }
    REAL xc = x > 0 ? x : 0, yc = y > 0 ? y : 0;
    const int xb = (int)((REAL)(w - 2) < xc ? (REAL)(w - 2) : xc);
    const int yb = (int)((REAL)(h - 2) < yc ? (REAL)(h - 2) : yc);
    const REAL xf = x - (REAL)xb, yf = y - (REAL)yb;
    const REAL ll = a[(long)yb * w + xb], lr = a[(long)yb * w + xb + 1];
    const REAL ur = a[(long)(yb + 1) * w + xb + 1], ul = a[(long)(yb + 1) * w + xb];
    const REAL upper = ul + xf * (ur - ul);
    const REAL lower = ll + xf * (lr - ll);
    return lower + yf * (upper - lower);
}

static int FN(clampi)(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* Temporal cumulant accumulator for one output pixel (liveSRRF_noInterpolation.cl:359-389,
 * liveSRRF.cl:363-393, live3DSRRF.cl:459-490).  In the f32 variant each frame's term is divided
 * by n (or n-1) before it is added, in the reference's order; the f64 variant sums in double
 * and divides once at the end. `tac_div2` reproduces the 2-D bicubic path, which stores the
 * previous value already divided by (n-1) and divides the product again (liveSRRF.cl:374,377). */
typedef struct {
    REAL avg, x2, tac, in, prev;
} FN(cumul);

static void FN(cumul_add)(FN(cumul) * c, int t, int n, REAL v, REAL cglh, int intw, int tac_div2) {
    const REAL x = intw ? v * cglh : cglh;
#if ORC_F32
    if (t == 0) {
        c->avg = intw ? v * cglh / n : cglh / n;
        c->x2 = intw ? v * cglh * v * cglh / n : cglh * cglh / n;
        c->tac = 0;
        c->in = v / n;
    } else {
        c->avg = c->avg + (intw ? v * cglh / n : cglh / n);
        c->x2 = c->x2 + (intw ? v * cglh * v * cglh / n : cglh * cglh / n);
        c->tac = c->tac + (intw ? v * cglh * c->prev / (n - 1) : cglh * c->prev / (n - 1));
        c->in = c->in + v / n;
    }
    c->prev = tac_div2 ? x / (n - 1) : x;
#else
    if (t == 0) {
        c->avg = x;
        c->x2 = x * x;
        c->tac = 0;
        c->in = v;
    } else {
        c->avg += x;
        c->x2 += x * x;
        c->tac += x * c->prev;
        c->in += v;
    }
    c->prev = x;
#endif
}

/* kernelCalculateVar then the readback's NaN->0 (liveSRRF_noInterpolation.cl:419-428). */
static void FN(cumul_store)(const FN(cumul) * c, int n, int tac_div2, long plane, long off,
                            float* out) {
#if ORC_F32
    const REAL avg = c->avg, av2 = avg * avg;
    REAL out4[4] = {avg, c->x2 - av2, c->tac - av2, c->in};
    (void)tac_div2;
#else
    const REAL avg = c->avg / n, av2 = avg * avg;
    REAL tac = n > 1 ? c->tac / (n - 1) : 0;
    if (tac_div2 && n > 1) tac /= (n - 1);
    REAL out4[4] = {avg, c->x2 / n - av2, tac - av2, c->in / n};
#endif
    for (int k = 0; k < 4; ++k) {
        float o = (float)out4[k];
        out[k * plane + off] = isnan(o) ? 0.0f : o;
    }
}

/* CGLH normalisation and sensitivity (liveSRRF_noInterpolation.cl:349-353). */
static REAL FN(cglh_finish)(REAL cglh, REAL wsum, float sensitivity) {
    cglh /= wsum;
    if (cglh >= 0)
        cglh = pow(cglh, (REAL)sensitivity); /* tgmath: powf in the f32 variant */
    else
        cglh = 0;
    return cglh;
}

/* ------------------------------------------------------------------------------------------ */
/* FHT path: Roberts cross on the interpolated frame, RGC with integer tap geometry.           */
/* ------------------------------------------------------------------------------------------ */

static void FN(robx)(const float* p, int w, int h, REAL* gx, REAL* gy) {
    for (int y1 = 0; y1 < h; ++y1) {
        const int y0 = y1 - 1 > 0 ? y1 - 1 : 0;
        for (int x1 = 0; x1 < w; ++x1) {
            const int x0 = x1 - 1 > 0 ? x1 - 1 : 0;
            const REAL a = p[(long)y0 * w + x1], b = p[(long)y1 * w + x0];
            const REAL c = p[(long)y1 * w + x1], d = p[(long)y0 * w + x0];
            gx[(long)y1 * w + x1] = a - b + c - d;
            gy[(long)y1 * w + x1] = -a + b + c - d;
        }
    }
}

int FN(orc_fht_block)(const float* interp, int n, int W, int H, int M, float fwhm, int sens,
                      int intw, const float* drift_x, const float* drift_y, float* out) {
    if (n < 1 || W < 2 || H < 2 || M < 1) return -1;
    const float sigma = fwhm / 2.354f;
    const float Mf = (float)M;
    const float tSS = 2 * sigma * Mf * sigma * Mf;
    const float tSO = (2 * sigma + 1) * Mf;
    const float R = Mf * ((float)((int)(2 * sigma)) + 1);
    const int r0 = -(int)R, r1 = (int)(R + 1);
    const long wh = (long)W * H;
    REAL* gx = (REAL*)malloc(sizeof(REAL) * wh);
    REAL* gy = (REAL*)malloc(sizeof(REAL) * wh);
    FN(cumul)* acc = (FN(cumul)*)calloc(wh, sizeof(FN(cumul)));
    REAL* fimg = (REAL*)malloc(sizeof(REAL) * wh);
    if (!gx || !gy || !acc || !fimg) return -2;

    for (int t = 0; t < n; ++t) {
        const float* fr = interp + (long)t * wh;
        const float sx = Mf * (drift_x ? drift_x[t] : 0.0f);
        const float sy = Mf * (drift_y ? drift_y[t] : 0.0f);
        FN(robx)(fr, W, H, gx, gy);
        for (long k = 0; k < wh; ++k) fimg[k] = fr[k];
#pragma omp parallel for schedule(dynamic, 4)
        for (int yM = 0; yM < H; ++yM) {
            for (int xM = 0; xM < W; ++xM) {
                const float xc = (float)((double)xM + 0.5 + (double)sx);
                const float yc = (float)((double)yM + 0.5 + (double)sy);
                const int bx = (int)((double)xc - 0.5), by = (int)((double)yc - 0.5);
                REAL cglh = 0, wsum = 0;
                for (int j = r0; j <= r1; ++j) {
                    const float vy = (float)((double)((float)by + (float)j) + 0.5);
                    if (!(vy > 0 && vy < (float)H)) continue;
                    for (int i = r0; i <= r1; ++i) {
                        const float vx = (float)((double)((float)bx + (float)i) + 0.5);
                        if (!(vx > 0 && vx < (float)W)) continue;
                        const REAL dx = (REAL)vx - (REAL)xc, dy = (REAL)vy - (REAL)yc;
                        const REAL d = sqrt(dx * dx + dy * dy);
                        if (!(d != 0 && d <= (REAL)tSO)) continue;
                        const int gxx = FN(clampi)((int)((double)vx - 0.5 + 1), 0, W - 1);
                        const int gxy = FN(clampi)((int)((double)vy - 0.5), 0, H - 1);
                        const int gyx = FN(clampi)((int)((double)vx - 0.5), 0, W - 1);
                        const int gyy = FN(clampi)((int)((double)vy - 0.5 + 1), 0, H - 1);
                        const REAL Gx = gx[(long)gxy * W + gxx], Gy = gy[(long)gyy * W + gyx];
                        REAL wgt = d * exp(-(d * d) / (REAL)tSS);
                        wgt = wgt * wgt * wgt * wgt;
                        wsum += wgt;
                        if (Gx * dx + Gy * dy < 0) {
                            const REAL gm = sqrt(Gx * Gx + Gy * Gy);
                            REAL dk = fabs(Gy * dx - Gx * dy) / gm;
                            if (isnan(dk)) dk = d;
                            dk = 1 - dk / d;
                            cglh += dk * wgt;
                        }
                    }
                }
                cglh = FN(cglh_finish)(cglh, wsum, (float)sens);
                REAL v;
                if (sx == 0 && sy == 0)
                    v = fr[(long)yM * W + xM];
                else
                    v = FN(sample2d)(fimg, W, H, (REAL)xM + (REAL)sx, (REAL)yM + (REAL)sy);
                FN(cumul_add)(&acc[(long)yM * W + xM], t, n, v, cglh, intw, 0);
            }
        }
    }
    for (long k = 0; k < wh; ++k) FN(cumul_store)(&acc[k], n, 0, wh, k, out);
    free(gx);
    free(gy);
    free(acc);
    free(fimg);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* 2-D bicubic path.                                                                           */
/* ------------------------------------------------------------------------------------------ */

/* Magnification-phase correction of AVG/VAR/TAC2 (liveSRRF.cl:464-505). */
static void FN(mp_correct)(float* out, int WM, int HM, int planesM, int w, int h, int planes,
                           int M, int is3d) {
    const long whM = (long)WM * HM;
    const long plane4 = whM * planesM;
    const int nz = is3d ? M : 1;
    const long cells = (long)w * h * planes;
    for (int c = 0; c < 3; ++c) {
        for (int pz = 0; pz < nz; ++pz)
            for (int py = 0; py < M; ++py)
                for (int px = 0; px < M; ++px) {
                    REAL s = 0;
                    for (long i = 0; i < cells; ++i) {
                        const long z = i / ((long)w * h);
                        const long y = (i - z * w * h) / w;
                        const long x = i - y * w - z * w * h;
                        const long zz = is3d ? (pz + z * M) : 0;
                        s += out[c * plane4 + zz * whM + (py + y * M) * WM + px + x * M];
                    }
                    const REAL map = s / (REAL)cells;
                    for (long i = 0; i < cells; ++i) {
                        const long z = i / ((long)w * h);
                        const long y = (i - z * w * h) / w;
                        const long x = i - y * w - z * w * h;
                        const long zz = is3d ? (pz + z * M) : 0;
                        float* o = &out[c * plane4 + zz * whM + (py + y * M) * WM + px + x * M];
                        *o = (float)((REAL)(*o) / map);
                    }
                }
    }
}

int FN(orc_bic_block)(const float* frames, int n, int W, int H, int M, float fwhm, int sens,
                      int intw, int mp, const float* drift_x, const float* drift_y, float* out) {
    if (n < 1 || W < 4 || H < 4 || M < 1) return -1;
    const int gm = 2;
    const float sigma = fwhm / 2.354f;
    const float radius = ((float)((int)(gm * 2 * sigma))) / gm + 1;
    const float tSS = 2 * sigma * sigma, tSO = 2 * sigma + 1;
    const int r0 = -(int)((float)gm * radius), r1 = (int)((float)gm * radius + 1);
    const int WM = W * M, HM = H * M, W2 = 2 * W, H2 = 2 * H;
    const long wh = (long)W * H, whM = (long)WM * HM, wh2 = (long)W2 * H2;
    REAL* img = (REAL*)malloc(sizeof(REAL) * wh);
    REAL* gx = (REAL*)malloc(sizeof(REAL) * wh);
    REAL* gy = (REAL*)malloc(sizeof(REAL) * wh);
    REAL* gxi = (REAL*)malloc(sizeof(REAL) * wh2);
    REAL* gyi = (REAL*)malloc(sizeof(REAL) * wh2);
    FN(cumul)* acc = (FN(cumul)*)calloc(whM, sizeof(FN(cumul)));
    if (!img || !gx || !gy || !gxi || !gyi || !acc) return -2;

    for (int t = 0; t < n; ++t) {
        const float* p = frames + (long)t * wh;
        /* Drift is stored x magnification by the host but used in raw-pixel units by this
         * kernel (LiveSRRF_CL.java:587-588 vs liveSRRF.cl:263-264); reproduced as is. */
        const float sx = (float)M * (drift_x ? drift_x[t] : 0.0f);
        const float sy = (float)M * (drift_y ? drift_y[t] : 0.0f);
        for (long k = 0; k < wh; ++k) img[k] = p[k];
        /* 2-point gradient (liveSRRF.cl:187-214). */
        for (int y1 = 0; y1 < H; ++y1)
            for (int x1 = 0; x1 < W; ++x1) {
                const int x0 = x1 - 1 > 0 ? x1 - 1 : 0, y0 = y1 - 1 > 0 ? y1 - 1 : 0;
                gx[(long)y1 * W + x1] = img[(long)y1 * W + x1] - img[(long)y1 * W + x0];
                gy[(long)y1 * W + x1] = img[(long)y1 * W + x1] - img[(long)y0 * W + x1];
            }
        /* 2x gradient interpolation (liveSRRF.cl:217-233). */
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H2; ++y)
            for (int x = 0; x < W2; ++x) {
                gxi[(long)y * W2 + x] = FN(sample2d)(gx, W, H, (REAL)((float)x / 2.0f), (REAL)((float)y / 2.0f));
                gyi[(long)y * W2 + x] = FN(sample2d)(gy, W, H, (REAL)((float)x / 2.0f), (REAL)((float)y / 2.0f));
            }
        /* RGC on the 2x gradient grid (liveSRRF.cl:238-401). */
#pragma omp parallel for schedule(dynamic, 4)
        for (int yM = 0; yM < HM; ++yM) {
            for (int xM = 0; xM < WM; ++xM) {
                const float xc = (float)(((double)xM + 0.5) / M + (double)sx);
                const float yc = (float)(((double)yM + 0.5) / M + (double)sy);
                const int kx = (int)((float)gm * xc), ky = (int)((float)gm * yc);
                REAL cglh = 0, wsum = 0;
                for (int j = r0; j <= r1; ++j) {
                    const float vy = ((float)ky + (float)j) / (float)gm;
                    if (!(vy > 0 && vy < (float)H)) continue;
                    for (int i = r0; i <= r1; ++i) {
                        const float vx = ((float)kx + (float)i) / (float)gm;
                        if (!(vx > 0 && vx < (float)W)) continue;
                        const REAL dx = (REAL)vx - (REAL)xc, dy = (REAL)vy - (REAL)yc;
                        const REAL d = sqrt(dx * dx + dy * dy);
                        if (!(d != 0 && d <= (REAL)tSO)) continue;
                        const int ax = (int)(gm * ((double)vx - 0.5)), ay = (int)(gm * ((double)vy - 0.5));
                        const int gxx = FN(clampi)((int)(gm * ((double)vx - 0.5) + 1), 0, W2 - 1);
                        const int gyy = FN(clampi)((int)(gm * ((double)vy - 0.5) + 1), 0, H2 - 1);
                        const REAL Gx = gxi[(long)FN(clampi)(ay, 0, H2 - 1) * W2 + gxx];
                        const REAL Gy = gyi[(long)gyy * W2 + FN(clampi)(ax, 0, W2 - 1)];
                        REAL wgt = d * exp(-(d * d) / (REAL)tSS);
                        wgt = wgt * wgt * wgt * wgt;
                        wsum += wgt;
                        if (Gx * dx + Gy * dy < 0) {
                            const REAL gmg = sqrt(Gx * Gx + Gy * Gy);
                            REAL dk = fabs(Gy * dx - Gx * dy) / gmg;
                            if (isnan(dk)) dk = d;
                            dk = 1 - dk / d;
                            cglh += dk * wgt;
                        }
                    }
                }
                cglh = FN(cglh_finish)(cglh, wsum, (float)sens);
                const REAL v = FN(sample2d)(img, W, H, (REAL)((float)xM / (float)M + sx - 0.5f),
                                            (REAL)((float)yM / (float)M + sy - 0.5f));
                FN(cumul_add)(&acc[(long)yM * WM + xM], t, n, v, cglh, intw, 1);
            }
        }
    }
    for (long k = 0; k < whM; ++k) {
        /* store without the NaN clean-up first: the MP correction runs before the readback */
        FN(cumul_store)(&acc[k], n, 1, whM, k, out);
    }
    if (mp) FN(mp_correct)(out, WM, HM, 1, W, H, 1, M, 0);
    for (long k = 0; k < 4 * whM; ++k)
        if (isnan(out[k])) out[k] = 0.0f;
    free(img);
    free(gx);
    free(gy);
    free(gxi);
    free(gyi);
    free(acc);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* 3-D path.                                                                                   */
/* ------------------------------------------------------------------------------------------ */

int FN(orc_3d_block)(const float* planes, int n, int P, int W, int H, int M, float fwhm,
                     int sens, int intw, int mp, const float* theta_deg, const float* shift_x,
                     const float* shift_y, const float* drift_x, const float* drift_y, float* out) {
    if (n < 1 || P < 2 || W < 4 || H < 4 || M < 1) return -1;
    const int gm = 2;
    const float sigma = fwhm / 2.354f;
    const float radius = ((float)((int)(gm * 2 * sigma))) / gm + 1;
    const float tSS = 2 * sigma * sigma, tSO = 2 * sigma + 1;
    const int r0 = -(int)((float)gm * radius), r1 = (int)((float)gm * radius + 1);
    const int k0 = -(int)radius, k1 = (int)radius + 1;
    const int WM = W * M, HM = H * M, PM = P * M, W2 = 2 * W, H2 = 2 * H;
    const long wh = (long)W * H, single = wh * P, whM = (long)WM * HM, whdM = whM * PM;
    const long wh2 = (long)W2 * H2;
    REAL* apx = (REAL*)malloc(sizeof(REAL) * single);
    REAL* raw = (REAL*)malloc(sizeof(REAL) * single);
    REAL* g[3];
    REAL* gi[3];
    for (int c = 0; c < 3; ++c) {
        g[c] = (REAL*)malloc(sizeof(REAL) * single);
        gi[c] = (REAL*)malloc(sizeof(REAL) * wh2 * P);
    }
    FN(cumul)* acc = (FN(cumul)*)calloc(whdM, sizeof(FN(cumul)));
    float* th = (float*)malloc(sizeof(float) * P);
    for (int z = 0; z < P; ++z) th[z] = (float)(-(double)theta_deg[z] * 3.141592653589793 / 180.0);

    for (int t = 0; t < n; ++t) {
        const float* p = planes + (long)t * single;
        const float dX = (float)M * (drift_x ? drift_x[t] : 0.0f);
        const float dY = (float)M * (drift_y ? drift_y[t] : 0.0f);
        for (long k = 0; k < single; ++k) raw[k] = p[k];
        /* Per-plane rotation about the centre and shift (live3DSRRF.cl:204-224). */
        for (int z = 0; z < P; ++z)
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x) {
                    const float ct = cosf(th[z]), st = sinf(th[z]);
                    const float xa = ((float)x - (float)(W - 1) / 2.0f) * ct -
                                     ((float)y - (float)(H - 1) / 2.0f) * st + (float)(W - 1) / 2.0f -
                                     shift_x[z];
                    const float ya = ((float)x - (float)(W - 1) / 2.0f) * st +
                                     ((float)y - (float)(H - 1) / 2.0f) * ct + (float)(H - 1) / 2.0f -
                                     shift_y[z];
                    apx[z * wh + (long)y * W + x] = FN(sample2d)(raw + z * wh, W, H, (REAL)xa, (REAL)ya);
                }
        /* 3-D 2-point gradient (live3DSRRF.cl:229-279). */
        for (int z = 0; z < P; ++z)
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x) {
                    const int x0 = x > 0 ? x - 1 : 0, y0 = y > 0 ? y - 1 : 0, z0 = z > 0 ? z - 1 : 0;
                    const long o = z * wh + (long)y * W + x;
                    g[0][o] = apx[o] - apx[z * wh + (long)y * W + x0];
                    g[1][o] = apx[o] - apx[z * wh + (long)y0 * W + x];
                    g[2][o] = apx[o] - apx[z0 * wh + (long)y * W + x];
                }
        /* Lateral 2x interpolation of the three components (live3DSRRF.cl:282-320). */
#pragma omp parallel for schedule(static)
        for (int z = 0; z < P; ++z)
            for (int y = 0; y < H2; ++y)
                for (int x = 0; x < W2; ++x)
                    for (int c = 0; c < 3; ++c)
                        gi[c][z * wh2 + (long)y * W2 + x] =
                            FN(sample2d)(g[c] + z * wh, W, H, (REAL)((float)x / 2.0f), (REAL)((float)y / 2.0f));
        /* 3-D RGC (live3DSRRF.cl:325-498). */
#pragma omp parallel for schedule(dynamic, 4)
        for (int zy = 0; zy < PM * HM; ++zy) {
            const int zM = zy / HM, yM = zy % HM;
            for (int xM = 0; xM < WM; ++xM) {
                const float xc = (float)(((double)xM + 0.5) / M + (double)dX);
                const float yc = (float)(((double)yM + 0.5) / M + (double)dY);
                const float zc = (float)(((double)zM + 0.5) / M);
                const int kx = (int)((float)gm * xc), ky = (int)((float)gm * yc);
                REAL cglh = 0, wsum = 0;
                for (int j = r0; j <= r1; ++j) {
                    const float vy = ((float)ky + (float)j) / (float)gm;
                    if (!(vy > 0 && vy < (float)H)) continue;
                    for (int i = r0; i <= r1; ++i) {
                        const float vx = ((float)kx + (float)i) / (float)gm;
                        if (!(vx > 0 && vx < (float)W)) continue;
                        for (int k = k0; k <= k1; ++k) {
                            const float vz = (float)((int)zc) + (float)k;
                            if (!(vz > 0 && vz < (float)P)) continue;
                            const REAL dx = (REAL)vx - (REAL)xc, dy = (REAL)vy - (REAL)yc;
                            const REAL dz = (REAL)vz - (REAL)zc;
                            const REAL d = sqrt(dx * dx + dy * dy + dz * dz);
                            if (!(d != 0 && d <= (REAL)tSO)) continue;
                            const int ax = FN(clampi)((int)(gm * ((double)vx - 0.5)), 0, W2 - 1);
                            const int ay = FN(clampi)((int)(gm * ((double)vy - 0.5)), 0, H2 - 1);
                            const int ax1 = FN(clampi)((int)(gm * ((double)vx - 0.5) + 1), 0, W2 - 1);
                            const int ay1 = FN(clampi)((int)(gm * ((double)vy - 0.5) + 1), 0, H2 - 1);
                            const int az = FN(clampi)((int)vz, 0, P - 1);
                            const REAL Gx = gi[0][az * wh2 + (long)ay * W2 + ax1];
                            const REAL Gy = gi[1][az * wh2 + (long)ay1 * W2 + ax];
                            const REAL Gz = gi[2][az * wh2 + (long)ay * W2 + ax];
                            REAL wgt = d * exp(-(d * d) / (REAL)tSS);
                            wgt = wgt * wgt * wgt * wgt;
                            wsum += wgt;
                            if (Gx * dx + Gy * dy + Gz * dz < 0) {
                                const REAL gmg = sqrt(Gx * Gx + Gy * Gy + Gz * Gz);
                                const REAL c1 = dy * Gz - dz * Gy, c2 = dz * Gx - dx * Gz;
                                const REAL c3 = dx * Gy - dy * Gx;
                                REAL dk = sqrt(c1 * c1 + c2 * c2 + c3 * c3) / gmg;
                                if (isnan(dk)) dk = d;
                                dk = 1 - dk / d;
                                cglh += dk * wgt;
                            }
                        }
                    }
                }
                cglh = FN(cglh_finish)(cglh, wsum, (float)sens);
                /* Cubic z interpolation of bicubic xy samples (live3DSRRF.cl:434-456); the
                 * fourth plane repeats z0+1, as in the reference. */
                int z0;
                const float zcof = zc - 0.5f;
                if (zcof < 0)
                    z0 = 0;
                else if (zcof >= (float)(P - 1))
                    z0 = P - 2;
                else
                    z0 = (int)floor((double)zcof);
                const REAL sxp = (REAL)((float)xM / (float)M + dX - 0.5f);
                const REAL syp = (REAL)((float)yM / (float)M + dY - 0.5f);
                const int zm1 = z0 - 1 > 0 ? z0 - 1 : 0;
                const int zp2 = z0 + 1 < P - 1 ? z0 + 1 : P - 1;
                const REAL v_1 = FN(sample2d)(apx + zm1 * wh, W, H, sxp, syp);
                const REAL v0 = FN(sample2d)(apx + z0 * wh, W, H, sxp, syp);
                const REAL v1 = FN(sample2d)(apx + (z0 + 1) * wh, W, H, sxp, syp);
                const REAL v2 = FN(sample2d)(apx + zp2 * wh, W, H, sxp, syp);
                const REAL z01 = (REAL)zc - (REAL)((float)z0 + 0.5f);
                const REAL a = (REAL)-0.5 * v_1 + (REAL)1.5 * v0 - (REAL)1.5 * v1 + (REAL)0.5 * v2;
                const REAL b = v_1 - (REAL)2.5 * v0 + (REAL)2.0 * v1 - (REAL)0.5 * v2;
                const REAL c = (REAL)-0.5 * v_1 + (REAL)0.5 * v1;
                const REAL v = a * z01 * z01 * z01 + b * z01 * z01 + c * z01 + v0;
                FN(cumul_add)(&acc[(long)zM * whM + (long)yM * WM + xM], t, n, v, cglh, intw, 0);
            }
        }
    }
    for (long k = 0; k < whdM; ++k) FN(cumul_store)(&acc[k], n, 0, whdM, k, out);
    if (mp) FN(mp_correct)(out, WM, HM, PM, W, H, P, M, 1);
    for (long k = 0; k < 4 * whdM; ++k)
        if (isnan(out[k])) out[k] = 0.0f;
    free(apx);
    free(raw);
    for (int c = 0; c < 3; ++c) {
        free(g[c]);
        free(gi[c]);
    }
    free(acc);
    free(th);
    return 0;
}

#undef FN
#undef CAT
#undef CAT2
