/*
 * esrrf_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference eSRRF hot path (NanoJ-eSRRF), written from the
 * mathematics of the reference's kernels and host code.  It is the checker used by tests/,
 * __graft_entry__.smoke() and the bench's CPU-baseline leg; the product library never links it.
 *
 * Every routine exists twice: `_f32` follows the reference's FP32 expression order (the parity
 * target), `_f64` evaluates the same algorithm in double precision (the error statements).
 * All output images are [4][planes][HM][WM] float slices in the reference's order
 * AVG, VAR, TAC2, INT with NaN replaced by 0 (LiveSRRF_CL.java:775-793).
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

/* Fourier interpolation of one stack, restating FourierInterpolation.java:12-73 and
 * mirrorPaddingEvenSquare (:118-172) with the 2-D discrete Hartley transform evaluated from
 * its definition in double precision.  scale_mode 0: mean preserving (inverse scaled by
 * 1/(N*N) of the padded input size); 1: inverse scaled by 1/(N'*N') of the magnified size. */
int orc_fht_interpolate(const float* raw, int n_frames, int width, int height, int magnification,
                        int scale_mode, float* out /* [n][H*M][W*M] */);

/* Roberts-cross gradient of one frame (liveSRRF_noInterpolation.cl:138-159). */
void orc_robx_f32(const float* img, int width, int height, float* gx, float* gy);

/* One SR block of the FHT path on already-interpolated frames
 * (liveSRRF_noInterpolation.cl:245-428, LiveSRRF_CL.java:462-794). */
int orc_fht_block_f32(const float* interp, int n_frames, int widthM, int heightM,
                      int magnification, float fwhm, int sensitivity, int int_weighting,
                      const float* drift_x, const float* drift_y, float* out);
int orc_fht_block_f64(const float* interp, int n_frames, int widthM, int heightM,
                      int magnification, float fwhm, int sensitivity, int int_weighting,
                      const float* drift_x, const float* drift_y, float* out);

/* One SR block of the 2-D bicubic path (liveSRRF.cl:26-505, LiveSRRF_CL.java:266-794). */
int orc_bic_block_f32(const float* frames, int n_frames, int width, int height,
                      int magnification, float fwhm, int sensitivity, int int_weighting,
                      int mp_correction, const float* drift_x, const float* drift_y, float* out);
int orc_bic_block_f64(const float* frames, int n_frames, int width, int height,
                      int magnification, float fwhm, int sensitivity, int int_weighting,
                      int mp_correction, const float* drift_x, const float* drift_y, float* out);

/* One SR block of the 3-D path on reshaped planes [n][planes][h][w]
 * (live3DSRRF.cl:42-611, LiveSRRF_CL.java:159-264, 636-794). */
int orc_3d_block_f32(const float* planes, int n_frames, int n_planes, int width, int height,
                     int magnification, float fwhm, int sensitivity, int int_weighting,
                     int mp_correction, const float* theta_deg, const float* shift_x,
                     const float* shift_y, const float* drift_x, const float* drift_y, float* out);
int orc_3d_block_f64(const float* planes, int n_frames, int n_planes, int width, int height,
                     int magnification, float fwhm, int sensitivity, int int_weighting,
                     int mp_correction, const float* theta_deg, const float* shift_x,
                     const float* shift_y, const float* drift_x, const float* drift_y, float* out);

/* Host-side MFM split of camera frames into planes (reshapeImageStack3D,
 * LiveSRRF_CL.java:963-994): crop the 3x3 tile named by roi[p], then (p - background)/coeff. */
int orc_mfm_reshape(const float* frames, int n_frames, int width, int height, int n_planes,
                    const float* roi, const float* intensity_coeff, float background,
                    float* planes /* [n][planes][height/3][width/3] */);

#ifdef __cplusplus
}
#endif
