/*
 * ref_fht.cpp -- TEST INFRASTRUCTURE ONLY (oracle/_ref build).
 *
 * Compiles the reference's FHT-path kernel source resources/liveSRRF_noInterpolation.cl
 * unchanged (included from the reference tree at build time, never copied) and replays the
 * host launch order of nanoj/liveSRRF/LiveSRRF_CL.java for one SR block:
 *   initialise / prepareBuffersFHTinterpolation   LiveSRRF_CL.java:159-264, 462-579
 *   loadDriftXYGPUbuffer (drift x magnification)   LiveSRRF_CL.java:583-595
 *   prepareDataFHT_SRRF + calculateSRRF             LiveSRRF_CL.java:598-632, 636-746
 *   readSRRFbuffer (VAR, NaN->0)                     LiveSRRF_CL.java:749-794
 * Frames arrive already Fourier-interpolated ([n][HM][WM] float); the interpolation itself is
 * the un-vendored NanoJFHT, restated separately in esrrf_oracle.c.
 */
#include "ref_common.h"

namespace ref_fht {
static double $SENSITIVITY$, $TWOSIGSQUARE$, $TWOSIGpONE$, $RADIUS$, $VXY_OFFSET$;
static int $WIDTH$, $HEIGHT$, $WH$, $NFRAMEFORSRRF$, $INTWEIGHTING$, $VXY_ARRAYSHIFT$;
#include REF_FHT_CL
#include "ref_undef.h"
}  // namespace ref_fht

extern "C" int ref_fht_block(const float* frames_interp, int n_frames, int widthM, int heightM,
                             int magnification, float fwhm, int sensitivity, int frames_per_load,
                             int int_weighting, const float* drift_x, const float* drift_y,
                             float* out /* [4][HM][WM] */) {
    using namespace ref_fht;
    if (n_frames < 1 || widthM < 2 || heightM < 2 || magnification < 1) return -1;
    if (frames_per_load < 1) frames_per_load = n_frames;

    /* prepareBuffersFHTinterpolation (LiveSRRF_CL.java:486-509), Java float arithmetic. */
    const float M = (float)magnification;
    const float sigma = fwhm / 2.354f;
    const float analysisRadius = (float)((int)(2 * sigma)) + 1;
    $SENSITIVITY$ = refcommon::java_float_literal((float)sensitivity);
    $TWOSIGSQUARE$ = refcommon::java_float_literal(2 * sigma * M * sigma * M);
    $TWOSIGpONE$ = refcommon::java_float_literal((2 * sigma + 1) * M);
    $RADIUS$ = refcommon::java_float_literal(M * analysisRadius);
    $WIDTH$ = widthM;
    $HEIGHT$ = heightM;
    $WH$ = widthM * heightM;
    $VXY_OFFSET$ = refcommon::java_float_literal(0.5f);
    $VXY_ARRAYSHIFT$ = 1;
    $NFRAMEFORSRRF$ = n_frames;
    $INTWEIGHTING$ = int_weighting ? 1 : 0;

    const long wh = (long)widthM * heightM;
    std::vector<float> px((size_t)frames_per_load * wh), gx(px.size()), gy(px.size());
    std::vector<float> prev(wh, 0.0f), outbuf(4 * wh, 0.0f), driftXY(2 * n_frames, 0.0f);
    int cur[2] = {0, 0};

    /* loadDriftXYGPUbuffer: stored in magnified-pixel units (LiveSRRF_CL.java:586-589). */
    for (int i = 0; i < n_frames; ++i) {
        driftXY[i] = magnification * (drift_x ? drift_x[i] : 0.0f);
        driftXY[i + n_frames] = magnification * (drift_y ? drift_y[i] : 0.0f);
    }
    /* resetFramePosition (LiveSRRF_CL.java:955-960). */
    kernelResetFramePosition(cur);

    for (int start = 0; start < n_frames; start += frames_per_load) {
        int nLoad = std::min(frames_per_load, n_frames - start);
        std::memcpy(px.data(), frames_interp + (size_t)start * wh, sizeof(float) * nLoad * wh);
        refcommon::range3d(widthM, heightM, nLoad,
                           [&] { calculateGradientRobX(px.data(), gx.data(), gy.data(), cur); });
        for (int f = 0; f < nLoad; ++f) {
            refcommon::range1d(wh, [&] {
                calculateRadialGradientConvergence(px.data(), gx.data(), gy.data(), prev.data(),
                                                   outbuf.data(), driftXY.data(), cur);
            });
            for (int i = 0; i < 2; ++i) {
                clshim::gid[0] = i;
                kernelIncrementFramePosition(cur);
            }
        }
    }
    refcommon::range1d(wh, [&] { kernelCalculateVar(outbuf.data()); });
    refcommon::nan_to_zero(outbuf.data(), 4 * wh);
    std::memcpy(out, outbuf.data(), sizeof(float) * 4 * wh);
    return 0;
}

/* Debug read-back of the Roberts-cross gradient of one interpolated frame
 * (readGradientBuffers, LiveSRRF_CL.java:797-879). */
extern "C" int ref_fht_gradient(const float* frame, int widthM, int heightM, float* gx_out,
                                float* gy_out) {
    using namespace ref_fht;
    $WIDTH$ = widthM;
    $HEIGHT$ = heightM;
    $WH$ = widthM * heightM;
    int cur[2] = {0, 0};
    refcommon::range3d(widthM, heightM, 1, [&] {
        calculateGradientRobX(const_cast<float*>(frame), gx_out, gy_out, cur);
    });
    return 0;
}
