// esrrf_internal.h -- shared declarations of the libesrrf CUDA kernels and host engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace esrrf {

// ------------------------------------------------------------------------------------------
// Fourier interpolation plan.
//
// FourierInterpolation.fhtSpaceInterpolation (FourierInterpolation.java:12-58) mirror-pads a
// frame to an N x N square (N a power of two), takes its 2-D Hartley transform, moves every
// spectral index p >= N/2 to p + (M-1) N on an NM x NM canvas, inverts, and crops.  The whole
// map is linear in the frame and, written out, equals
//     I' = s [ Dy X Dx^T + P (x) c_x + c_y (x) Q - u_y (x) R - T (x) u_x ]
// where X is the padded frame, D the N-1-term Dirichlet kernel sampled at
// 2 pi (m M - n)/(N M), c(n) = cos(pi n / M), u(n) = sin(pi n / M), and P, Q, R, T are per-frame
// vectors built from the alternating row/column sums of X (the unpaired Nyquist row/column of
// the Hartley spectrum).  The dense part runs as two batched GEMMs; the rank-one part is
// folded into the second GEMM's epilogue.
// ------------------------------------------------------------------------------------------
struct InterpPlan {
    int w = 0, h = 0, M = 0;  // raw frame size and magnification
    int N = 0;                // padded square size
    int WM = 0, HM = 0;       // output size
    int xroi = 0, yroi = 0;   // crop offsets on the NM canvas
    bool identity_pad = true; // no mirror padding needed (power-of-two square input)
    double s_axis = 0;        // per-axis scale folded into Dx, Dy
    double s = 0;             // total scale
    // device arrays
    float* dxT = nullptr;     // [N][WM]   (Dx transposed, scaled)
    float* dy = nullptr;      // [HM][N]   (scaled)
    float* dyT = nullptr;     // [N][HM]   (scaled, transposed copy for the vector kernel)
    float* cx = nullptr;      // [WM]
    float* ux = nullptr;      // [WM]
    float* cy = nullptr;      // [HM]
    float* uy = nullptr;      // [HM]
    int* srcx = nullptr;      // [N] source column of padded column
    int* srcy = nullptr;      // [N] source row of padded row
    // tensor-core passes (tc): Dx and Dy as split operand panels, and a device flag set when a
    // bounded wait gave up
    bool tc = false;
    float* dxp = nullptr;     // pass 1 B panels [WM/256][N/16] (hi, lo)
    float* dyp = nullptr;     // pass 2 A panels [HM/128][N/16] (hi, lo)
    int* tc_err = nullptr;
};

// Per-frame interpolation scratch for a chunk of F frames.
struct InterpScratch {
    int capacity = 0;
    float* rowT = nullptr;    // [F][interp_rowT_floats]  first-pass output
    float* xs = nullptr;      // [F][interp_xs_floats]  padded frame as operand panels (tc)
    float* alt = nullptr;     // [F][interp_alt_floats(N)]  alternating row/column sums, row sums
    float* vec = nullptr;     // [F][interp_vec_floats(HM, WM)]  P, T, Q, R and the frame mean
};
inline size_t interp_alt_floats(int N) { return 3 * (size_t)N + 1; }
inline size_t interp_vec_floats(int HM, int WM) { return 2 * (size_t)HM + 2 * (size_t)WM + 1; }

cudaError_t interp_plan_create(InterpPlan& plan, int w, int h, int M, int scale_mode);
void interp_plan_destroy(InterpPlan& plan);

// Adjoint of the interpolation: graw[F][h][w] += L^T gI[F][HM][WM].  dx: Dx row-major [WM][N]
// (scaled like dxT); scratch T1 [F][N][WM], gX [F][N][N], proj [F][2HM+2WM], dvec [F][2N+1].
cudaError_t interp_adjoint_run(const InterpPlan& p, const float* dx, const float* gI, int F,
                               float* T1, float* gX, float* proj, float* dvec, float* graw,
                               cudaStream_t stream);

// Tensor-core (tcgen05, three-term TF32) form of the two dense passes; needs N % 128 == 0.
// Writes the first-pass rows into scratch.rowT as pass 2's operand panels.
bool tc_interp_supported(const InterpPlan& plan);
cudaError_t tc_plan_tables(InterpPlan& plan, const std::vector<float>& dxT, const std::vector<float>& dy);
// Scratch floats per frame: first-pass rows (either form) and the frame's operand panels.
size_t interp_rowT_floats(const InterpPlan& plan);
size_t interp_xs_floats(const InterpPlan& plan);
cudaError_t tc_interp_passes(const InterpPlan& plan, InterpScratch& scratch, const void* raw,
                             bool is_u16, int F, float* out, cudaStream_t stream);
// Reads (and clears) the plan's tensor-core failure flag; synchronises `stream`.
cudaError_t interp_tc_check(const InterpPlan& plan, cudaStream_t stream, bool* failed);

// raw: [F][h][w] uint16 (is_u16) or float; out: [F][HM][WM]
cudaError_t interp_run(const InterpPlan& plan, InterpScratch& scratch, const void* raw,
                       bool is_u16, int F, float* out, cudaStream_t stream, int* launches);

// ------------------------------------------------------------------------------------------
// RGC geometry of the FHT path (liveSRRF_noInterpolation.cl:245-393, constants from
// LiveSRRF_CL.java:491-500).  Taps are integer offsets (i, j) in [r0, r1]^2.
// ------------------------------------------------------------------------------------------
constexpr int kMaxBox = 48;  // max tap box side r1 - r0 + 1 supported by the fused kernel

struct FhtGeometry {
    float sigma = 0, tSS = 0, tSO = 0, radius = 0;
    int r0 = 0, r1 = 0, S = 0;   // S = r1 - r0 + 1
    float sensitivity = 1;
    // host tables [S][S] indexed [(j - r0) * S + (i - r0)]
    std::vector<float> w, wd;    // weight and weight / distance (0 outside the tap disc)
    std::vector<int> jlo, jhi;   // per column i: valid j range (jlo > jhi if none)
    float wsum_interior = 0;     // sum of weights in the reference's (j, i) order
};
FhtGeometry fht_geometry(int M, float fwhm, int sensitivity);

// Accumulator state for one SR block on the device.
struct BlockState {
    long pixels = 0;
    double* acc = nullptr;  // [4][pixels]: sum X, sum X^2, sum X_t X_{t-1}, sum v
    float* prev = nullptr;  // [pixels]
};

struct FhtRgcArgs {
    const float* interp;   // [F][H][W]
    const float* gx;       // plain path: [F][H][W] Roberts-cross gradients
    const float* gy;
    int W, H, F;
    int t0;                // frame index within the block of the first frame
    const float* shift;    // [2][F] drift in magnified pixels (plain path)
    int int_weighting;
    BlockState st;
    float* cg_out = nullptr;  // fused kernel only: if set, write CGLH / sum of weights per frame
                              // [F][H][W] (before the sensitivity power) instead of accumulating
    float* prev_out = nullptr;  // fused kernel: [H][W] scratch that lets a launch split its frames
                                // into groups across CTAs (the last group's values land here and
                                // are copied to st.prev after the launch, so no group overwrites a
                                // value another group still reads); null: one group
};

cudaError_t fht_robx(const float* interp, int W, int H, int F, float* gx, float* gy,
                     cudaStream_t stream);
cudaError_t fht_rgc_plain(const FhtGeometry& g, const FhtRgcArgs& a, cudaStream_t stream);

struct FhtFusedTables {
    float* wtab = nullptr;     // device [S*S] weights
    float* wdtab = nullptr;    // device [S*S] weight / distance
    int* jrange = nullptr;     // device [2*S]
    float* wsum = nullptr;     // device [H*W] per-pixel weight sums
};
cudaError_t fht_fused_tables(const FhtGeometry& g, int W, int H, FhtFusedTables& t,
                             cudaStream_t stream);
void fht_fused_tables_free(FhtFusedTables& t);
cudaError_t fht_rgc_fused(const FhtGeometry& g, const FhtFusedTables& t, const FhtRgcArgs& a,
                          cudaStream_t stream);
bool fht_fused_supported(const FhtGeometry& g);
// Multiprocessor count of a device (cached per device).
int sm_count(int dev);

// Frames with drift on the fused kernel.  A frame's shift (sx, sy) in magnified pixels is
// uniform over the frame, so the tap geometry of every output pixel is the same: source offsets
// (floor(sx) + i, floor(sy) + j) and centre offsets (i - frac(sx), j - frac(sy)), i, j in
// [r0, r1].  Per frame of a launch: the integer shift, the offsets of tap (0, 0), the sum of the
// weights over the whole disc in the reference's (j, i) order, the weight tables, each column's
// disc chord and 2-D prefix sums of the weights (for output pixels whose tap box leaves the
// image).
struct alignas(16) FhtDriftFrame {  // 48 bytes: copied to shared memory in 16-byte pieces
    int ix, iy;         // floor of the shift
    float fi0, fj0;     // r0 - frac(sx), r0 - frac(sy)
    float wsum_int;     // sum of w over the disc, (j, i) order
    float fx, fy;       // frac(sx), frac(sy)
    int zero;           // 1: sx == sy == 0 (the interpolated pixel is the intensity)
    float sx, sy;       // the shift itself (magnified pixels)
    int pad[2];
};
struct FhtDriftTables {
    int capacity = 0, S = 0;
    FhtDriftFrame* fr = nullptr;  // [F]
    float2* wt = nullptr;         // [F][S][S] (w, w/d), [ii][jj - lo_ii]: each column from its chord's first row
    int* jr = nullptr;            // [F][2S] per column: first and last tap row of the disc
    double* pre = nullptr;        // [F][S+1][S+1] prefix sums: pre[jj][ii] = sum over rows < jj, cols < ii
    float* v = nullptr;           // [F][H][W] intensity at the shifted position
};
// Buffers for F frames of tap boxes up to S wide and `pixels` output pixels per frame (0: no
// intensity planes).
cudaError_t fht_drift_tables_alloc(int S, int F, long pixels, FhtDriftTables& t);
// Tables of F frames with shifts sx[f], sy[f] (device, magnified pixels).
cudaError_t fht_drift_tables_build(const FhtGeometry& g, const float* sx, const float* sy, int F,
                                   FhtDriftTables& t, cudaStream_t stream);
// The intensity of every pixel of F frames at the frame's shift, into v [F][H][W]:
// getInterpolatedValue(xM + sx, yM + sy) (bicubic, bilinear near the border; the pixel itself for a
// frame with sx == sy == 0).  The sweep's per-frame mode needs these planes; the engine's launches
// sample in the tile kernel.
cudaError_t fht_shift_sample(const float* interp, int W, int H, int F, const float* sx, const float* sy,
                             float* v, cudaStream_t stream);
void fht_drift_tables_free(FhtDriftTables& t);
// The fused kernel on a launch whose frames have the tables of `t` (built for this launch).
cudaError_t fht_rgc_fused_drift(const FhtGeometry& g, const FhtDriftTables& t, const FhtRgcArgs& a,
                                cudaStream_t stream);
// Per-pixel sum of a [S][S] tap table over the in-image taps, (j, i) order.
cudaError_t tap_table_sum(const float* tab, int r0, int S, int W, int H, float* out,
                          cudaStream_t stream);

// AVG/VAR/TAC2/INT from the block accumulators (kernelCalculateVar and the readback's NaN->0).
// tac_div2: the 2-D bicubic path's double division of TAC2 by (n-1).
cudaError_t finalize_block(const BlockState& st, int n, int tac_div2, float* out,
                           cudaStream_t stream);
cudaError_t zero_block(BlockState& st, cudaStream_t stream);

// ------------------------------------------------------------------------------------------
// 2-D bicubic path (liveSRRF.cl) and 3-D path (live3DSRRF.cl): constants as
// prepareBuffersBICinterpolation computes them (LiveSRRF_CL.java:301-342).
// ------------------------------------------------------------------------------------------
struct BicGeometry {
    float sigma = 0, tSS = 0, tSO = 0, radius = 0;
    float sensitivity = 1;
};
BicGeometry bic_geometry(float fwhm, int sensitivity);

struct BicRgcArgs {
    const float* fraw;   // [F][h][w] raw frames as float (intensity source)
    const float* gxi;    // [F][2h][2w] 2x-resampled 2-point gradient
    const float* gyi;
    int w, h, M, F, t0;
    float tSS, tSO, radius, sens;
    const float* shift;  // [2][F] drift x magnification (used in raw pixels, as the reference)
    int int_weighting;
    BlockState st;
};

cudaError_t bic_prepare(const void* raw, int is_u16, int w, int h, int F, float* fraw, float* gx,
                        float* gy, float* gxi, float* gyi, cudaStream_t stream);
cudaError_t grad2x(const float* g, int w, int h, int planes, float* gi, cudaStream_t stream);
cudaError_t bic_rgc(const BicRgcArgs& a, cudaStream_t stream);

// Tabulated 2-D bicubic-path RGC for launches without drift.  With zero shift the tap geometry
// of an output pixel depends only on its sub-pixel phase (xM % M, yM % M), so each phase's taps
// inside the disc (reference loop order j, i) are listed once; a CTA of 32 x 8 input cells of one
// phase stages its slab of the unit-gradient field in shared memory per frame.
struct BicTables {
    float4* tab = nullptr;   // [taps] (offset in a CTA's slab as int bits, dx, dy, w / d)
    float* tw = nullptr;     // [taps] w
    int2* node = nullptr;    // [taps] 2x-grid node offset (sx, sy) from (2 qx, 2 qy)
    int* start = nullptr;    // [M^2 + 1] first tap of each phase
    float* wsum = nullptr;   // [h M][w M] sum of w over each pixel's in-range taps
    int max_taps = 0;
    // zero halo of the field (2x-grid columns, even, and rows); padded width and height
    int padx = 0, pady = 0, W2p = 0, H2p = 0;
    // slab of a CTA: rows 2 qy + sy - sl_symin, per parity columns qx + (sx >> 1) - sl_fxmin,
    // both parities side by side in a row of 2 sl_nx float2s
    int sl_symin = 0, sl_fxmin = 0, sl_rows = 0, sl_nx = 0;
    size_t smem = 0;         // dynamic shared memory of one CTA
};
// Tables for frames of w x h pixels; false in `built` when a CTA's shared memory would not fit
// (the per-pixel kernel runs instead).  The per-pixel sums of weights are computed on `stream`
// (synchronised before returning).
cudaError_t bic_tables_build(const BicGeometry& g, int M, int w, int h, BicTables& t, bool& built,
                             cudaStream_t stream);
void bic_tables_free(BicTables& t);
size_t bic_field_float2s(const BicTables& t, int F);
struct BicTabArgs {
    const float2* U;     // [F][H2p][W2p] padded unit gradient, columns split by parity
    const float* fraw;   // [F][h][w] raw frames as float (intensity source)
    int w, h, M, F, t0;
    float sens;
    int int_weighting;
    BicTables tab;
    BlockState st;
    // per-frame mode (the sweep): CGLH / sum of weights and the intensity of every frame,
    // [F][hM][wM] each, instead of the block's cumulants
    float* cg_out;
    float* v_out;
};
// unit gradient (Gx read at x + 1, Gy at y + 1 of the 2x grid) into the interior of the padded
// field; zero at the last column and row, which no tap reads.  The halo is zeroed once, when the
// field is allocated.
cudaError_t unit_grad2d(const float* gxi, const float* gyi, int w, int h, int F, const BicTables& t,
                        float2* U, cudaStream_t stream);
cudaError_t bic_rgc_tab(const BicTabArgs& a, cudaStream_t stream);
// MP map of AVG/VAR/TAC2 and division (then NaN->0) on a finalized output [4][PM][HM][WM].
cudaError_t mp_correct(float* out, int w, int h, int P, int M, int is3d, float* map,
                       cudaStream_t stream);

struct Rgc3dArgs {
    const float* apx;    // [F][P][h][w] aligned planes
    const float* gxi;    // [F][P][2h][2w]
    const float* gyi;
    const float* gzi;
    int w, h, P, M, F, t0;
    float tSS, tSO, radius, sens;
    const float* shift;  // [2][F] drift x magnification (used in raw pixels, as the reference)
    int int_weighting;
    BlockState st;
};
struct Mfm3dTables {
    int* tile_x0 = nullptr;   // [P] crop origin of each plane in the camera frame
    int* tile_y0 = nullptr;
    float* coeff = nullptr;   // [P] intensity scaling
    float* cos_t = nullptr;   // [P] cos / sin of -theta (radians, float)
    float* sin_t = nullptr;
    float* shx = nullptr;     // [P]
    float* shy = nullptr;
};
// Tabulated 3-D RGC for launches without drift.  With zero shift the tap geometry of an output
// voxel depends only on its sub-pixel phase (xM % M, yM % M, zM % M), so each phase's taps inside
// the disc (reference loop order j, i, k) are listed once: source offset into the unit-gradient
// field, (dx, dy, dz), d^2, w, w/d, and the phase's interior sum of weights.
struct Rgc3dTables {
    float4* taba = nullptr;   // [taps] (offset into the padded field as int bits, dx, dy, dz)
    float4* tabb = nullptr;   // [taps] (d^2, w, w/d, packed (sx, sy, sz) as int bits)
    int* start = nullptr;     // [M^3 + 1] first tap of each phase
    float* wsum = nullptr;    // [P M][h M][w M] sum of w over each voxel's in-range taps
    int max_taps = 0;
    // zero halo of the unit-gradient field: 2x-grid columns (even) and rows, planes below/above
    int padx = 0, pady = 0, padz_lo = 0, padz_hi = 0;
    int W2p = 0, H2p = 0, Pp = 0;  // padded 2x-grid width, height and plane count
    // z-blocked form (M <= 5): per lateral phase the union over z-phases of the taps, each entry
    // [offset, dx, dy, then (dz, w, w/d) per z-phase (w = 0: not a tap of that z-phase)], padded
    // to whole float4s
    float4* ztab = nullptr;
    int* zstart = nullptr;    // [M^2 + 1] first entry of each lateral phase
    int zmax_taps = 0, zes = 0;  // largest entry count of a phase; float4s per entry
    // slab-staged form: a phase's entries are ordered by plane offset sz = zk0 .. zk0 + znz - 1;
    // zseg[lp (znz + 1) + s] is the first entry of plane s; zsoff[entry] the entry's offset in a
    // CTA's slab of the field (rows 2 qy + sy - sl_symin, per parity columns qx + (sx >> 1) -
    // sl_fxmin, both parities side by side in a row of 2 sl_nx float4s)
    int* zseg = nullptr;
    int* zsoff = nullptr;
    int zk0 = 0, znz = 0;
    // Within a plane offset the entries are grouped by the range [a, b] of z-phases they are taps
    // of (a contiguous range: dz is monotonic in the z-phase), the full range first, then the
    // others in (a, b) order (z3d_class_range); zcseg[lp (znz zncls + 1) + s zncls + c] is the
    // first entry of class c of plane s, the last value the phase's entry count.
    int* zcseg = nullptr;
    int zncls = 0;             // M (M + 1) / 2 classes
    int sl_symin = 0, sl_fxmin = 0, sl_rows = 0, sl_nx = 0;
};
// Tables for planes of w x h pixels, P planes; the per-voxel sums of weights are computed on
// `stream` (synchronised before returning).
cudaError_t rgc3d_tables_build(const BicGeometry& g, int M, int w, int h, int P, Rgc3dTables& t,
                               cudaStream_t stream);
size_t rgc3d_field_float4s(const Rgc3dTables& t, int F);
bool rgc3d_one_voxel();
void rgc3d_tables_free(Rgc3dTables& t);
struct Rgc3dTabArgs {
    const float4* U;     // [F][Pp][H2p][W2p] padded unit gradient, columns split by parity
    const float* apx;    // [F][P][h][w] aligned planes
    int w, h, P, M, F, t0;
    float sens;
    int int_weighting;
    Rgc3dTables tab;
    BlockState st;
    int form = 0;        // kRgc3dForm*: which tabulated kernel (0: the default choice)
};
// Forms of the tabulated 3-D RGC (rgc_3d_tab); a form whose shared memory does not fit falls
// back to the next one.
constexpr int kRgc3dAuto = 0, kRgc3dTwoCells = 1, kRgc3dSlab = 2, kRgc3dL1 = 3;
// unit gradient field from the 2x-resampled components (Gx read at x+1, Gy at y+1, Gz in place)
// into the interior of the padded field; zero where no tap may read (plane 0, last column and
// row).  The halo is zeroed once, when the field is allocated.
cudaError_t unit_grad3d(const float* gxi, const float* gyi, const float* gzi, int w, int h, int P,
                        int F, const Rgc3dTables& t, float4* U, cudaStream_t stream);
cudaError_t rgc_3d_tab(const Rgc3dTabArgs& a, cudaStream_t stream);

// camera frames [F][H][W] -> planes [F][P][hs][ws] ((p - background) / coeff), aligned planes,
// 3-D 2-point gradient and its 2x lateral resampling.
cudaError_t mfm_prepare(const void* raw, int is_u16, int W, int H, int P, int ws, int hs, int F,
                        const Mfm3dTables& t, float background, float* planes, float* apx,
                        float* gx, float* gy, float* gz, float* gxi, float* gyi, float* gzi,
                        cudaStream_t stream);
cudaError_t rgc_3d(const Rgc3dArgs& a, cudaStream_t stream);

// Variants of the table set-up that place their tables in caller-provided device memory (no
// allocation); used by the allocation-free entry point.
cudaError_t interp_plan_place(InterpPlan& plan, int w, int h, int M, int scale_mode,
                              unsigned char* base, size_t* bytes, cudaStream_t stream);
cudaError_t fht_fused_tables_place(const FhtGeometry& g, int W, int H, FhtFusedTables& t,
                                   unsigned char* base, size_t* bytes, cudaStream_t stream);

}  // namespace esrrf
