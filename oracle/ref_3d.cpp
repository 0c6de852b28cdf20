/*
 * ref_3d.cpp -- TEST INFRASTRUCTURE ONLY (oracle/_ref build).
 *
 * Compiles the reference's 3-D kernel source resources/live3DSRRF.cl unchanged (included from
 * the reference tree at build time, never copied) and replays the host launch order of
 * nanoj/liveSRRF/LiveSRRF_CL.java for one SR block with a 3-D calibration:
 *   initialise (3-D branch, nPlanes, nPlanesM)       LiveSRRF_CL.java:159-264
 *   prepareBuffersBICinterpolation + ShiftXYTheta3D   LiveSRRF_CL.java:266-459
 *   calculateSRRF (align, 2-point 3-D gradient, xy 2x gradient interpolation, 3-D RGC)
 *                                                     LiveSRRF_CL.java:636-746
 *   readSRRFbuffer (VAR, MP^3 map + correction, NaN->0) LiveSRRF_CL.java:749-794
 * Input frames are the planes after the host-side MFM reshape (reshapeImageStack3D,
 * LiveSRRF_CL.java:963-994): [n][nPlanes][h][w] float.
 */
#include "ref_common.h"

namespace ref_3d {
static double $SENSITIVITY$, $TWOSIGSQUARE$, $TWOSIGpONE$, $RADIUS$, $VXY_OFFSET$, $DIMRATIO$;
static int $MAGNIFICATION$, $GXGYMAGNIFICATION$, $WIDTH$, $HEIGHT$, $WH$, $WINT$, $HINT$,
    $WHINT$, $WM$, $HM$, $WHM$, $WHDM$, $NFRAMEFORSRRF$, $INTWEIGHTING$, $NPLANES$, $WHD$,
    $VXY_ARRAYSHIFT$;
#include REF_3D_CL
#include "ref_undef.h"
}  // namespace ref_3d

extern "C" int ref_3d_block(const float* planes, int n_frames, int n_planes, int width,
                            int height, int magnification, float fwhm, int sensitivity,
                            int frames_per_load, int int_weighting, int mp_correction,
                            const float* theta_deg, const float* shift_x, const float* shift_y,
                            float dim_ratio, const float* drift_x, const float* drift_y,
                            float* out /* [4][nPlanes*M][H*M][W*M] */) {
    using namespace ref_3d;
    if (n_frames < 1 || width < 4 || height < 4 || magnification < 1 || n_planes < 2) return -1;
    if (frames_per_load < 1) frames_per_load = n_frames;
    const int gradientMag = 2;
    const int M = magnification;

    const float sigma = fwhm / 2.354f;
    const float radius = ((float)((int)(gradientMag * 2 * sigma))) / gradientMag + 1;
    $MAGNIFICATION$ = M;
    $SENSITIVITY$ = refcommon::java_float_literal((float)sensitivity);
    $GXGYMAGNIFICATION$ = gradientMag;
    $TWOSIGSQUARE$ = refcommon::java_float_literal(2 * sigma * sigma);
    $TWOSIGpONE$ = refcommon::java_float_literal(2 * sigma + 1);
    $RADIUS$ = refcommon::java_float_literal(radius);
    $WIDTH$ = width;
    $HEIGHT$ = height;
    $WH$ = width * height;
    $WM$ = width * M;
    $HM$ = height * M;
    $WHM$ = width * height * M * M;
    $WINT$ = gradientMag * width;
    $HINT$ = gradientMag * height;
    $WHINT$ = gradientMag * width * gradientMag * height;
    $VXY_OFFSET$ = refcommon::java_float_literal(0.5f);
    $VXY_ARRAYSHIFT$ = 1;
    $NFRAMEFORSRRF$ = n_frames;
    $INTWEIGHTING$ = int_weighting ? 1 : 0;
    $NPLANES$ = n_planes;
    $DIMRATIO$ = refcommon::java_float_literal(dim_ratio);
    $WHD$ = width * height * n_planes;
    $WHDM$ = width * height * n_planes * M * M * M;

    const long single = (long)width * height * n_planes;
    const long whdM = single * M * M * M;
    std::vector<float> px((size_t)frames_per_load * single), apx(px.size());
    std::vector<float> gx(px.size()), gy(px.size()), gz(px.size());
    std::vector<float> gxi((size_t)frames_per_load * 4 * single), gyi(gxi.size()), gzi(gxi.size());
    std::vector<float> prev(whdM, 0.0f), outbuf(4 * whdM, 0.0f), driftXY(2 * n_frames, 0.0f);
    std::vector<float> mpmap(3 * M * M * M, 0.0f), sxyt(3 * n_planes);
    int cur[2] = {0, 0};

    /* ShiftXYTheta3D upload (LiveSRRF_CL.java:438-457): -theta in radians, then x, y shifts. */
    for (int i = 0; i < n_planes; ++i) {
        sxyt[i] = (float)(-(double)theta_deg[i] * 3.141592653589793 / 180.0);
        sxyt[i + n_planes] = shift_x[i];
        sxyt[i + 2 * n_planes] = shift_y[i];
    }
    for (int i = 0; i < n_frames; ++i) {
        driftXY[i] = M * (drift_x ? drift_x[i] : 0.0f);
        driftXY[i + n_frames] = M * (drift_y ? drift_y[i] : 0.0f);
    }
    kernelResetFramePosition(cur);

    for (int start = 0; start < n_frames; start += frames_per_load) {
        int nLoad = std::min(frames_per_load, n_frames - start);
        std::memcpy(px.data(), planes + (size_t)start * single, sizeof(float) * nLoad * single);
        refcommon::range1d(single * nLoad,
                           [&] { kernelAlignPixels(px.data(), apx.data(), sxyt.data()); });
        refcommon::range1d(single * nLoad, [&] {
            calculateGradient_2point(apx.data(), gx.data(), gy.data(), gz.data(), cur);
        });
        refcommon::range1d(4 * single * nLoad, [&] {
            calculateGradientInterpolation(gx.data(), gy.data(), gz.data(), gxi.data(), gyi.data(),
                                           gzi.data());
        });
        for (int f = 0; f < nLoad; ++f) {
            refcommon::range1d(whdM, [&] {
                calculateRadialGradientConvergence(apx.data(), gxi.data(), gyi.data(), gzi.data(),
                                                   prev.data(), outbuf.data(), driftXY.data(), cur);
            });
            for (int i = 0; i < 2; ++i) {
                clshim::gid[0] = i;
                kernelIncrementFramePosition(cur);
            }
        }
    }
    refcommon::range1d(whdM, [&] { kernelCalculateVar(outbuf.data()); });
    if (mp_correction) {
        refcommon::range1d(3L * M * M * M, [&] { kernelCalculateMPmap(outbuf.data(), mpmap.data()); });
        refcommon::range1d(3L * whdM, [&] { kernelCorrectMPmap(outbuf.data(), mpmap.data()); });
    }
    refcommon::nan_to_zero(outbuf.data(), 4 * whdM);
    std::memcpy(out, outbuf.data(), sizeof(float) * 4 * whdM);
    return 0;
}
