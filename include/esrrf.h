/*
 * esrrf.h -- C ABI of libesrrf, a B200 (sm_100a) engine for the eSRRF hot path of
 * NanoJ-eSRRF: Fourier interpolation of each frame, gradient field, radial gradient
 * convergence (RGC) with Gaussian distance weighting and a sensitivity exponent, intensity
 * weighting, and AVG/VAR/TAC2 temporal cumulants over frame blocks, in 2-D and 3-D.
 *
 * The entry points replace the members of the reference's device-engine class
 * nanoj.liveSRRF.LiveSRRF_CL (src/nanoj/liveSRRF/LiveSRRF_CL.java); each declaration cites
 * the member it replaces.  Conventions:
 *   - plain pointers and sizes only; images are row-major float32 or uint16, frames contiguous;
 *   - every call returns an esrrf_status; esrrf_last_error() gives the message of the last
 *     failure on a handle (the reference logs and carries on, or throws RuntimeException on
 *     device-initialisation failure, LiveSRRF_CL.java:115-119);
 *   - one handle owns one CUDA stream and its device buffers; handles are independent (the
 *     reference keeps its OpenCL context in static fields, LiveSRRF_CL.java:70-88, so it has
 *     one engine per JVM); calls on one handle must not overlap, except
 *     esrrf_request_cancel(), which is thread-safe;
 *   - host buffers may be pageable or pinned; the *_device variants take device pointers.
 */
#ifndef ESRRF_H
#define ESRRF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ESRRF_VERSION_MAJOR 0
#define ESRRF_VERSION_MINOR 2

typedef enum {
    ESRRF_OK = 0,
    ESRRF_CANCELLED = 1,       /* calculateSRRF returned true (user pressed Escape) */
    ESRRF_ERR_INVALID = -1,    /* bad argument or inconsistent parameters */
    ESRRF_ERR_CUDA = -2,       /* a CUDA runtime call failed; see esrrf_last_error() */
    ESRRF_ERR_NOMEM = -3,      /* device or pinned-host allocation failed */
    ESRRF_ERR_STATE = -4,      /* call out of order (e.g. frames pushed past the block) */
    ESRRF_ERR_TIMEOUT = -5,    /* a bounded device wait gave up */
    ESRRF_ERR_NODEVICE = -6    /* no CUDA device */
} esrrf_status;

/* Interpolation mode of the 2-D path (LiveSRRF_CL.java:159-264): FHT loads
 * liveSRRF_noInterpolation.cl on Fourier-interpolated frames, BIC loads liveSRRF.cl. */
typedef enum { ESRRF_INTERP_FHT = 0, ESRRF_INTERP_BIC = 1 } esrrf_interp;

/* Scale of the inverse Hartley transform in the Fourier interpolation.  The reference's
 * transform (nanoj.core2.NanoJFHT, not vendored) does not say which it uses. */
typedef enum {
    ESRRF_FHT_SCALE_MEAN_PRESERVING = 0, /* interpolated mean equals the raw mean */
    ESRRF_FHT_SCALE_UNITARY_BIG = 1      /* inverse scaled by 1/(N*M)^2: mean divided by M^2 */
} esrrf_fht_scale;

/* Parameters of LiveSRRF_CL.initialise (LiveSRRF_CL.java:159) as a POD struct.
 * width/height: raw frame size (3-D: the full MFM camera frame, split 3x3 into planes).
 * fwhm: the GUI's "Radius" (sigma = fwhm / 2.354).  n_frames_on_gpu: frames per push.
 * n_frame_for_srrf: frames per SR block.  block_length: accepted for API fidelity; the CUDA
 * kernels do not need the reference's 1-D work splitting (LiveSRRF_CL.java:707-742).
 * 3-D (n_planes > 0): per-plane calibration of the .njt table the reference loads
 * (LiveSRRF_CL.java:210-227): roi index, theta (degrees), x/y shift, intensity scaling,
 * background; axial_offset_nm and pixel_size_um give the (unused by the kernel) dimRatio. */
typedef struct {
    int width, height;
    int magnification;
    float fwhm;
    int sensitivity;
    int n_frames_on_gpu;
    int n_frame_for_srrf;
    int block_length;
    int device;           /* CUDA ordinal; -1 = the device with most SMs x clock */
    int int_weighting;    /* 1: weight CGLH by the interpolated intensity */
    int mp_correction;    /* 1: macro-pixel correction (BIC and 3-D paths only, as in the reference) */
    int interp;           /* esrrf_interp; forced to BIC in 3-D (LiveSRRF_CL.java:166-168) */
    int fht_scale;        /* esrrf_fht_scale */
    int kernel;           /* 0: fused tile kernel where applicable, 1: plain per-pixel kernel */
    int frames_per_launch;/* frames per interpolation + RGC launch; 0: the block in equal launches of
                             at most 50 frames (FHT path, within ~4 GB of frame buffers) or 32
                             (2-D bicubic path, within ~2 GB), 8 timepoints in 3-D;
                             ESRRF_FRAMES_PER_LAUNCH_TUNED: measured by the autotuner (below) */
    /* 3-D calibration, all arrays of length n_planes (NULL in 2-D). */
    int n_planes;
    const float* roi;
    const float* theta_deg;
    const float* shift_x;
    const float* shift_y;
    const float* intensity_coeff;
    float background;
    float axial_offset_nm;
    float pixel_size_um;
} esrrf_params;

typedef struct esrrf_handle esrrf_handle;

/* Library version "major.minor". */
const char* esrrf_get_version(void);

/* Number of CUDA devices; replaces the platform scan of LiveSRRF_CL.checkDevices
 * (LiveSRRF_CL.java:111-155). */
esrrf_status esrrf_device_count(int* count);

/* Name, SM count and max clock (MHz) of one device (checkDevices' per-device log). */
esrrf_status esrrf_device_info(int device, char* name, size_t name_len, int* sm_count,
                               int* clock_mhz);

/* Fill *p with the reference GUI defaults (LiveSRRF_optimised_.java:128-134): M 5,
 * radius 2, sensitivity 1, 100 frames/block, 20000 block length, FHT on, intensity weighting
 * on, MP correction off. */
void esrrf_default_params(esrrf_params* p);

/* Replaces LiveSRRF_CL.initialise (LiveSRRF_CL.java:159-264) and its buffer/program set-up
 * (prepareBuffersFHTinterpolation :462-579, prepareBuffersBICinterpolation :266-459).  Sizes:
 * width, height >= 4; one output slice (widthM x heightM, in 3-D times planes x M) below 2^31
 * pixels. */
esrrf_status esrrf_create(const esrrf_params* params, esrrf_handle** out);

/* Replaces LiveSRRF_CL.release (LiveSRRF_CL.java:939-951). */
esrrf_status esrrf_destroy(esrrf_handle* h);

/* Replaces LiveSRRF_CL.loadDriftXYGPUbuffer (LiveSRRF_CL.java:583-595): per-frame drift of
 * the current block in raw pixels, n = n_frame_for_srrf values each (NULL = zero drift). */
esrrf_status esrrf_set_drift(esrrf_handle* h, const float* drift_x, const float* drift_y, int n);

/* Replaces LiveSRRF_CL.resetFramePosition (LiveSRRF_CL.java:955-960): starts a new block. */
esrrf_status esrrf_reset_frame_position(esrrf_handle* h);

/* Replaces LiveSRRF_CL.calculateSRRF (LiveSRRF_CL.java:636-746): accumulates n_frames
 * consecutive frames (host memory, [n][height][width]) into the current block.  Returns
 * ESRRF_CANCELLED if esrrf_request_cancel() was called. */
esrrf_status esrrf_calculate_srrf_u16(esrrf_handle* h, const uint16_t* frames, int n_frames);
esrrf_status esrrf_calculate_srrf_f32(esrrf_handle* h, const float* frames, int n_frames);
/* Same, frames already in device memory of the handle's device. */
esrrf_status esrrf_calculate_srrf_u16_device(esrrf_handle* h, const uint16_t* d_frames,
                                             int n_frames);
esrrf_status esrrf_calculate_srrf_f32_device(esrrf_handle* h, const float* d_frames,
                                             int n_frames);

/* Replaces LiveSRRF_CL.readSRRFbuffer (LiveSRRF_CL.java:749-794): finalises VAR/TAC2 (and the
 * MP correction on the BIC/3-D paths) and copies [4][planesM][heightM][widthM] float slices,
 * in the order AVG, VAR, TAC2, INT, NaN replaced by 0, to host memory `out`. */
esrrf_status esrrf_read_srrf(esrrf_handle* h, float* out);
/* Same into device memory. */
esrrf_status esrrf_read_srrf_device(esrrf_handle* h, float* d_out);
/* Queued form of esrrf_read_srrf (no reference counterpart; the reference reads synchronously):
 * finalises the block into one of two device output slots and queues the copy to host `out` on
 * its own stream, returning at once, so that the next block's frames (reset + push) overlap the
 * copy.  `out` must stay valid (and should be pinned for the copy to overlap) until
 * esrrf_finish_queue returns; a third read waits for the first one's copy. */
esrrf_status esrrf_read_srrf_async(esrrf_handle* h, float* out);

/* Frames (timepoints in 3-D) per interpolation + RGC launch: esrrf_params.frames_per_launch, or
 * the value chosen when that is 0 or ESRRF_FRAMES_PER_LAUNCH_TUNED (no reference counterpart: the
 * reference launches per frame). */
esrrf_status esrrf_frames_per_launch(const esrrf_handle* h, int* frames);

/* Autotuner.  The reference sizes its GPU loads from a memory model (calculatenFrameOnGPU /
 * predictMemoryUsed, gui/LiveSRRF_optimised_.java:763-877); here esrrf_create with
 * frames_per_launch = ESRRF_FRAMES_PER_LAUNCH_TUNED measures instead: for the parameter set's
 * frame size, magnification, tap box, path and block length it times one block of synthetic frames
 * through a temporary engine for each candidate frames-per-launch value (every way to cut the
 * block into equal launches of 8 to 64 frames that fits ~4 GB; in 3-D also the tabulated kernel's
 * forms: two cells per thread, one cell per thread with the slab in shared memory, the field read
 * through L1), keeps the fastest, and caches the choice in a text file keyed by the device name
 * and those parameters (ESRRF_TUNE_CACHE, else esrrf_tune.txt beside libesrrf.so), so later
 * handles with the same key are created without measuring.  esrrf_tune_report gives the choice,
 * its source ("measured", "cache" or "off") and the candidates' times as JSON text. */
#define ESRRF_FRAMES_PER_LAUNCH_TUNED (-1)
esrrf_status esrrf_tune_report(const esrrf_handle* h, char* buf, size_t len);

/* Output geometry (public fields widthS/heightS/nPlanes/nPlanesM, LiveSRRF_CL.java:41-45). */
esrrf_status esrrf_output_shape(const esrrf_handle* h, int* width_m, int* height_m,
                                int* planes_m);

/* Replaces readGradientBuffers (LiveSRRF_CL.java:797-879): gradient components of the first
 * frame of the last push ([2 or 3][planes][h'][w'] float, h'/w' as in the reference). */
esrrf_status esrrf_read_gradients(esrrf_handle* h, float* out, size_t out_len);

/* Replaces LiveSRRF_CL.readAlignedPixels (LiveSRRF_CL.java:881-906): the 3-D path's aligned planes
 * (split, background-subtracted, scaled, rotated and shifted) of the first frame of the last group
 * of frames on the device (a push of at most esrrf_frames_per_launch frames is one group),
 * [n_planes][height / 3][width / 3] float, NaN -> 0.  ESRRF_ERR_STATE on the 2-D paths. */
esrrf_status esrrf_read_aligned_pixels(esrrf_handle* h, float* out, size_t out_len);

/* Replaces LiveSRRF_CL.readMPmaps (LiveSRRF_CL.java:909-935): the macro-pixel maps of the last read
 * (each cumulant's mean over the image of every sub-pixel phase), [3][M][M] on the bicubic path,
 * [3][M][M][M] (per cumulant M z-phase slices of M x M) in 3-D, NaN -> 0.  ESRRF_ERR_STATE without
 * MP correction or on the FHT path (the reference builds the map on the bicubic paths only). */
esrrf_status esrrf_read_mp_maps(esrrf_handle* h, float* out, size_t out_len);

/* Replaces finishQueue (LiveSRRF_CL.java:1009-1015): waits for every queued kernel, input copy
 * and read-back of the handle; ESRRF_ERR_TIMEOUT if a bounded tensor-core wait gave up.  The
 * pushes (esrrf_calculate_srrf_*) from host memory return once their frames are copied; the
 * kernels of the last frames may still run until a read or this call. */
esrrf_status esrrf_finish_queue(esrrf_handle* h);

/* Thread-safe cancellation (replaces the IJ.escapePressed() polling, LiveSRRF_CL.java:731-734). */
esrrf_status esrrf_request_cancel(esrrf_handle* h);

/* Diagnostic of the device-side failure detection (no counterpart in the reference, whose
 * OpenCL waits are host-side queue.finish() calls): runs the tensor-core passes' bounded
 * mbarrier wait, with a limit of `cycles` SM clock cycles (1 .. 1e9), on a barrier that receives
 * its one arrival (arrive = 1: ESRRF_OK) or none (arrive = 0: the wait gives up, records it in a
 * device flag as the passes do, and the host reads ESRRF_ERR_TIMEOUT).  The context stays usable. */
esrrf_status esrrf_check_bounded_wait(int device, int arrive, long long cycles);

/* Message of the last failure on h (or of the last failed esrrf_create when h is NULL). */
const char* esrrf_last_error(const esrrf_handle* h);

/* Runs the handle's kernels on a caller-owned CUDA stream (cudaStream_t passed as void*; NULL
 * restores a private stream).  Calls still return only when their work on it is done. */
esrrf_status esrrf_set_stream(esrrf_handle* h, void* stream);

/* Enables per-launch CUDA-event timing of the interpolation and RGC kernels (off by default).  The reference's NanoJProfiler timings
 * (LiveSRRF_CL.java:67, 609-631, 727-741) are the counterpart.  Events are read back once,
 * after the call's final stream synchronisation, so timing adds no intermediate waits. */
esrrf_status esrrf_set_timing(esrrf_handle* h, int enable);

/* Device time (ms) of the last calculate call's interpolation and RGC kernels (timing on) and
 * the number of kernels it launched (always). */
esrrf_status esrrf_last_timing(const esrrf_handle* h, float* interp_ms, float* rgc_ms,
                               int* launches);

/* ---- Batched parameter sweep and rolling analysis over uneven blocks -----------------------
 * Replaces the per-combination loop of ParametersSweep_.run (gui/ParametersSweep_.java:328-519:
 * initialise + resetFramePosition + loadDriftXYGPUbuffer + calculateSRRF + readSRRFbuffer for
 * every radius x sensitivity) and the block loop of LiveSRRF_optimised_.run
 * (gui/LiveSRRF_optimised_.java:276-389), on the 2-D FHT path or the 2-D bicubic path (the
 * sweep's "Use FHT interpolation" option, gui/ParametersSweep_.java:879).  All frames are
 * interpolated (FHT) or their gradients resampled (bicubic) once, and the RGC tap loop runs once
 * per (magnification, radius) for all sensitivities and blocks; the whole sweep is one captured
 * CUDA graph per device replayed per run.  Blocks are arbitrary [start, start + length) frame
 * ranges (uneven and overlapping allowed).  The bicubic sweep applies the MP correction to every
 * output, as the reference's sweep initialises the engine with it on
 * (gui/ParametersSweep_.java:410).
 * Drift (FHT sweep): one shift per frame of the stack in raw pixels, the array the sweep computes
 * once and loads into every combination's engine (gui/ParametersSweep_.java:282-290, 452-454);
 * NULL = zero drift.  A rolling analysis whose blocks each have their own shift array (relative to
 * the block's first frame, gui/LiveSRRF_optimised_.java:283-305) passes non-overlapping blocks
 * with the arrays laid end to end.
 * Devices: n_devices > 1 splits the sweep across those CUDA ordinals (esrrf_sweep_plan says how);
 * each device keeps its own copy of the frames it needs, nothing is exchanged between devices, and
 * esrrf_sweep_run gathers every output into the host buffer.  n_devices = 0 uses `device`.  A
 * device listed k times takes up to k shards, which run concurrently on it (each with its own
 * stream, frame copy and graph). */
typedef struct {
    int width, height, n_frames;
    int n_mag;
    const int* magnifications;
    int n_radius;
    const float* radii;        /* the GUI's "Radius" (fwhm) values */
    int n_sens;
    const int* sensitivities;
    int n_blocks;
    const int* block_start;
    const int* block_length;
    int int_weighting;
    int device;                /* CUDA ordinal; -1 = device 0 */
    int interp;                /* esrrf_interp: ESRRF_INTERP_FHT or ESRRF_INTERP_BIC */
    const float* drift_x;      /* [n_frames] per-frame shift in raw pixels, or NULL (FHT only) */
    const float* drift_y;
    int n_devices;             /* 0: one device (`device`); > 1: shard across `devices` */
    const int* devices;
} esrrf_sweep_params;

typedef struct esrrf_sweep esrrf_sweep;

esrrf_status esrrf_sweep_create(const esrrf_sweep_params* params, esrrf_sweep** out);
/* How esrrf_sweep_create splits a sweep across its devices (host arithmetic, no device work; the
 * reference runs one device).  Units are the (magnification, radius) pairs, costed by tap count x
 * output pixels x frame span, assigned longest first to the least-loaded device, or -- when that
 * leaves devices idle or unbalanced -- the blocks, cut by start into contiguous runs of balanced
 * frame span, every pair on every device; the split with the smaller largest cost is used.
 * pair_device[m * n_radius + r] / block_device[b]: the device ordinal, -1 = every device of the
 * split, -2 = none.  device_cost[d] (per entry of the device list, so per shard where a device is
 * listed twice): the relative cost.  Each may be NULL. */
esrrf_status esrrf_sweep_plan(const esrrf_sweep_params* params, int* pair_device, int* block_device,
                              double* device_cost);
/* Output layout: for magnification m, radius r the floats from offsets[m * n_radius + r] hold
 * [n_sens][n_blocks][4][HM_m][WM_m] (AVG, VAR, TAC2, INT; NaN -> 0), HM_m = height * M_m. */
esrrf_status esrrf_sweep_output_layout(const esrrf_sweep* s, size_t* total_floats, size_t* offsets);
/* frames: [n_frames][height][width] uint16 (is_u16 = 1) or float; device pointers here (a sweep on
 * one device only), host pointers in esrrf_sweep_run.  The first run with given pointers captures
 * the graph.  esrrf_sweep_run with a pinned `out` (page-locked, e.g. cudaHostAlloc) on a one-device
 * sweep copies each (magnification, radius) pair's outputs while the later pairs compute. */
esrrf_status esrrf_sweep_run_device(esrrf_sweep* s, const void* d_frames, int is_u16, float* d_out);
esrrf_status esrrf_sweep_run(esrrf_sweep* s, const void* frames, int is_u16, float* out);
/* Kernels in one run (the graphs' node count over all devices). */
esrrf_status esrrf_sweep_launch_count(const esrrf_sweep* s, int* launches);
/* Devices the sweep runs on (1 unless it was split). */
esrrf_status esrrf_sweep_shard_count(const esrrf_sweep* s, int* shards);
const char* esrrf_sweep_last_error(const esrrf_sweep* s);
esrrf_status esrrf_sweep_destroy(esrrf_sweep* s);

/* ---- SQUIRREL metrics ----------------------------------------------------------------------------
 * Replaces ErrorMapLiveSRRF.optimise + calculateErrorMap (ErrorMapLiveSRRF.java:81-193) as the
 * parameter sweep applies them to every reconstruction (gui/ParametersSweep_.java:468-519): for
 * each super-resolved image and its reference (the INT slice of the same block), the blur sigma in
 * [0, 4 / 2.35482 M] pixels minimising the RMSE of the blurred, intensity-fitted image (Brent
 * search), the fit's alpha and beta, RSE (that RMSE), RSP (its Pearson coefficient) and optionally
 * the error map |ref - blur(alpha SR + beta)|. */
typedef struct {
    int width, height;     /* super-resolved image size in pixels */
    int magnification;     /* M: sigma bound 4 / 2.35482 M pixels; fixed sigma and crop x M */
    int fix_sigma;         /* 1: sigma = fixed_sigma x M, no search */
    float fixed_sigma;     /* input pixels */
    int crop;              /* border of this many input pixels (x M) left out of everything */
    void* stream;          /* cudaStream_t for the work (NULL: the default stream) */
} esrrf_squirrel_params;

/* d_base: device floats; image i is [height][width] at d_base + sr_offsets[i], its reference at
 * d_base + ref_offsets[i] (host arrays; references may repeat).  Host outputs (each may be NULL):
 * sigma, alpha, beta, rse, rsp [n].  d_error_maps (device, may be NULL): [n][h'][w'], the cropped
 * size.  Returns when the results are on the host. */
esrrf_status esrrf_squirrel(const esrrf_squirrel_params* p, int n, const float* d_base,
                            const size_t* sr_offsets, const size_t* ref_offsets, float* sigma,
                            float* alpha, float* beta, float* rse, float* rsp, float* d_error_maps);
const char* esrrf_squirrel_last_error(void);

/* ---- Drift (vibration) estimation ---------------------------------------------------------------
 * Replaces XYShiftCalculator.calculateShiftArray (XYShiftCalculator.java:26-48), whose shifts the
 * plugins hand to loadDriftXYGPUbuffer (gui/ParametersSweep_.java:282-290,
 * gui/LiveSRRF_optimised_.java:283-305), i.e. to esrrf_set_drift.  For each frame f, the circular
 * cross-correlation C_f(s) = sum_p (ref(p) - mean ref) frame_f(p + s) over the lags |sx|, |sy| <= R,
 * its arg-max and the stationary point of the least-squares quadratic through the 3 x 3 samples
 * around it.  shift_x/shift_y[f] is the displacement of frame f's content relative to the reference
 * frame, the value esrrf_set_drift takes for that frame.  The reference searches the whole map;
 * here R = max_shift (<= 0: 31), at most (min(width, height) - 1) / 2 (the whole map). */
esrrf_status esrrf_drift_window(int width, int height, int max_shift, int* radius);
/* d_frames: device, n_frames x height x width (uint16 if is_u16, else float32); ref_frame indexes
 * into them.  shift_x, shift_y: host [n_frames].  d_ccm (device, may be NULL): [n_frames][2R+1][2R+1],
 * C_f at lag (sy, sx) in row sy + R, column sx + R.  Returns when the shifts are on the host.
 * Scratch (the partial maps, about n_frames (2R+1)^2 x 8 B x row tiles, at most ~1 GB) is one
 * workspace per device, grown on demand and kept until the process exits; calls on one device
 * are serialised on it.  Errors: esrrf_drift_last_error(). */
esrrf_status esrrf_estimate_drift(const void* d_frames, int is_u16, int n_frames, int width, int height,
                                  int ref_frame, int max_shift, float* shift_x, float* shift_y,
                                  float* d_ccm, void* stream);
const char* esrrf_drift_last_error(void);

/* ---- Fourier ring correlation ------------------------------------------------------------------
 * Replaces the FRC resolution of the parameter sweep (gui/ParametersSweep_.java:403-447:
 * FRC.calculateFireNumber(odd, even, FIXED_1_OVER_7) x the reconstruction's pixel size) for a batch
 * of image pairs.  NanoJ-Core's FRC is not in the reference tree; the method restated: each image
 * minus its mean times a Tukey window (tapers over the outer eighth of each axis), zero-padded to
 * N x N (N the next power of two >= max(width, height, 32)); FRC(r) = sum Re(F1 conj F2) /
 * sqrt(sum |F1|^2 sum |F2|^2) over rings r = round(|(u, v)|) = 0 .. N/2; FIRE = N / q x pixel_size,
 * q the first crossing of 1/7 (linear between rings, r >= 2); NaN if FRC(1) < 1/7 or no crossing. */
typedef struct {
    int width, height;  /* image size in pixels */
    float pixel_size;   /* the resolution's unit per pixel (1: pixels) */
    void* stream;       /* cudaStream_t (NULL: the default stream) */
} esrrf_frc_params;

esrrf_status esrrf_frc_size(int width, int height, int* padded_size, int* n_rings);
/* d_base: device floats; pair i is the [height][width] images at d_base + a_offsets[i] and
 * d_base + b_offsets[i] (host arrays).  fire: host [n].  curves (host, may be NULL): [n][n_rings]. */
esrrf_status esrrf_frc(const esrrf_frc_params* p, int n, const float* d_base, const size_t* a_offsets,
                       const size_t* b_offsets, float* fire, float* curves);
const char* esrrf_frc_last_error(void);

/* ---- Differentiable eSRRF ---------------------------------------------------------------------
 * A fidelity loss of the 2-D FHT-path AVG reconstruction and its hand-written adjoint; there is
 * no counterpart in the reference's OpenCL path (the closest is the post-hoc error map of
 * ErrorMapLiveSRRF.java:81-233).  With R = (1/T) sum_t I_t C_t^S (S real), B = Gaussian(sigma) * R,
 * D = M x M box average of B and F the frame average of the input,
 *   loss = mean((alpha D + beta - F)^2),  alpha, beta the least-squares fit of F on D.
 * esrrf_loss_and_grad gives the loss and d loss / d(radius, S, sigma) in grads[0..2] and, if
 * d_grad_frames is non-NULL, d loss / d frames ([T][height][width] float, device).  Zero drift,
 * intensity weighting on, mean-preserving interpolation; tap boxes 6..26 pixels wide. */
typedef struct esrrf_adjoint esrrf_adjoint;
esrrf_status esrrf_adjoint_create(int width, int height, int n_frames, int magnification, int device,
                                  esrrf_adjoint** out);
esrrf_status esrrf_adjoint_forward(esrrf_adjoint* a, const float* d_frames, float fwhm,
                                   float sensitivity, float sigma_b, double* loss);
esrrf_status esrrf_loss_and_grad(esrrf_adjoint* a, const float* d_frames, float fwhm,
                                 float sensitivity, float sigma_b, double* loss, double* grads,
                                 float* d_grad_frames);
const char* esrrf_adjoint_last_error(const esrrf_adjoint* a);
esrrf_status esrrf_adjoint_destroy(esrrf_adjoint* a);

/* Allocation-free variant of one FHT-path SR block; it has no counterpart in the reference.
 * For callers that must not allocate device memory when they reconstruct -- e.g. a
 * live-acquisition callback, where cudaMalloc/cudaFree can synchronise the device and stall
 * the camera stream, or a host that owns every device byte through its own pool.  It computes
 * what esrrf_create + esrrf_calculate_srrf_*_device + esrrf_read_srrf_device compute for one
 * block (FHT interpolation, mean-preserving scale, zero drift, fused RGC, FP64 cumulants) and
 * takes every temporary buffer from one 64 MiB static device array that each GPU loading the
 * library holds until exit; frame sizes whose tables, buffers and accumulators need more than
 * that (roughly widthM x heightM above 1.2 M pixels) are rejected with ESRRF_ERR_INVALID, as
 * are radii whose tap box exceeds 32 magnified pixels.  The interpolation's dense passes run on
 * the FP32 SIMT kernels (the handle uses tensor cores on large frames): the results agree with
 * the handle's to ~1e-6 of each slice's range.
 * d_frames: device [n_frames][height][width], uint16 (is_u16 = 1) or float.  d_out: device
 * [4][height*M][width*M] float (AVG, VAR, TAC2, INT).  stream: cudaStream_t or NULL.
 * err/err_len: optional buffer for a message on failure.
 * The tables (interpolation, tap weights) are kept in the array between calls: a call with the
 * same frame size, magnification, radius and sensitivity as the previous call on its device only
 * enqueues kernels; a call that changes them first builds them on the host and uploads them with
 * pageable copies (which wait for the stream's earlier work), so make one such call at set-up.
 * The first call on a device also looks up the array's address (cudaGetSymbolAddress, with that
 * device current) -- make it before any stream capture.  Calls share the array and it keeps
 * the last call's contents (the accumulators are cleared at the start of each call); calls
 * whose work overlaps on the GPU race on it. */
esrrf_status esrrf_fht_block_noalloc(const void* d_frames, int is_u16, int n_frames, int width,
                                     int height, int magnification, float fwhm, int sensitivity,
                                     int int_weighting, float* d_out, void* stream, char* err,
                                     size_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* ESRRF_H */
