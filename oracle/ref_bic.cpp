/*
 * ref_bic.cpp -- TEST INFRASTRUCTURE ONLY (oracle/_ref build).
 *
 * Compiles the reference's 2-D bicubic-path kernel source resources/liveSRRF.cl unchanged
 * (included from the reference tree at build time, never copied) and replays the host launch
 * order of nanoj/liveSRRF/LiveSRRF_CL.java for one SR block with doFHTinterpolation=false:
 *   initialise / prepareBuffersBICinterpolation    LiveSRRF_CL.java:159-264, 266-459
 *   loadDriftXYGPUbuffer (drift x magnification)    LiveSRRF_CL.java:583-595
 *   calculateSRRF (2-point gradient, 2x gradient interpolation, RGC per frame)
 *                                                    LiveSRRF_CL.java:636-746
 *   readSRRFbuffer (VAR, MP map + correction, NaN->0) LiveSRRF_CL.java:749-794
 */
#include "ref_common.h"

namespace ref_bic {
static double $SENSITIVITY$, $TWOSIGSQUARE$, $TWOSIGpONE$, $RADIUS$, $VXY_OFFSET$;
static int $MAGNIFICATION$, $GXGYMAGNIFICATION$, $WIDTH$, $HEIGHT$, $WH$, $WINT$, $HINT$,
    $WHINT$, $WM$, $HM$, $WHM$, $NFRAMEFORSRRF$, $INTWEIGHTING$, $VXY_ARRAYSHIFT$;
#include REF_BIC_CL
#include "ref_undef.h"
}  // namespace ref_bic

extern "C" int ref_bic_block(const float* frames, int n_frames, int width, int height,
                             int magnification, float fwhm, int sensitivity, int frames_per_load,
                             int int_weighting, int mp_correction, const float* drift_x,
                             const float* drift_y, float* out /* [4][H*M][W*M] */,
                             float* mpmap_out /* [3][M][M] or null */) {
    using namespace ref_bic;
    if (n_frames < 1 || width < 4 || height < 4 || magnification < 1) return -1;
    if (frames_per_load < 1) frames_per_load = n_frames;
    const int gradientMag = 2;
    const int M = magnification;

    /* prepareBuffersBICinterpolation (LiveSRRF_CL.java:301-342), Java float arithmetic. */
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

    const long wh = (long)width * height;
    const long whM = wh * M * M;
    std::vector<float> px((size_t)frames_per_load * wh), gx(px.size()), gy(px.size());
    std::vector<float> gxi((size_t)frames_per_load * 4 * wh), gyi(gxi.size());
    std::vector<float> prev(whM, 0.0f), outbuf(4 * whM, 0.0f), driftXY(2 * n_frames, 0.0f);
    std::vector<float> mpmap(3 * M * M, 0.0f);
    int cur[2] = {0, 0};

    for (int i = 0; i < n_frames; ++i) {
        driftXY[i] = M * (drift_x ? drift_x[i] : 0.0f);
        driftXY[i + n_frames] = M * (drift_y ? drift_y[i] : 0.0f);
    }
    kernelResetFramePosition(cur);

    for (int start = 0; start < n_frames; start += frames_per_load) {
        int nLoad = std::min(frames_per_load, n_frames - start);
        std::memcpy(px.data(), frames + (size_t)start * wh, sizeof(float) * nLoad * wh);
        refcommon::range3d(width, height, nLoad,
                           [&] { calculateGradient_2point(px.data(), gx.data(), gy.data(), cur); });
        refcommon::range3d(gradientMag * width, gradientMag * height, nLoad, [&] {
            calculateGradientInterpolation(gx.data(), gy.data(), gxi.data(), gyi.data());
        });
        for (int f = 0; f < nLoad; ++f) {
            refcommon::range1d(whM, [&] {
                calculateRadialGradientConvergence(px.data(), gxi.data(), gyi.data(), prev.data(),
                                                   outbuf.data(), driftXY.data(), cur);
            });
            for (int i = 0; i < 2; ++i) {
                clshim::gid[0] = i;
                kernelIncrementFramePosition(cur);
            }
        }
    }
    refcommon::range1d(whM, [&] { kernelCalculateVar(outbuf.data()); });
    if (mp_correction) {
        refcommon::range1d(3L * M * M, [&] { kernelCalculateMPmap(outbuf.data(), mpmap.data()); });
        refcommon::range1d(3L * whM, [&] { kernelCorrectMPmap(outbuf.data(), mpmap.data()); });
    }
    refcommon::nan_to_zero(outbuf.data(), 4 * whM);
    std::memcpy(out, outbuf.data(), sizeof(float) * 4 * whM);
    if (mpmap_out) std::memcpy(mpmap_out, mpmap.data(), sizeof(float) * 3 * M * M);
    return 0;
}
