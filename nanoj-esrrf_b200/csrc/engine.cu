// engine.cu -- host engine behind the C ABI (include/esrrf.h).  One handle mirrors one
// nanoj.liveSRRF.LiveSRRF_CL instance (src/nanoj/liveSRRF/LiveSRRF_CL.java): it owns a CUDA
// stream, the device buffers and the block bookkeeping that the reference keeps in the
// two-int nCurrentFrame buffer (LiveSRRF_CL.java:296-299, 738-741, 955-960).
#include <string.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/esrrf.h"
#include "engine.h"
#include "esrrf_internal.h"

using namespace esrrf;

namespace {
std::mutex g_err_mu;
std::string g_create_error;

const char* kVersion = "0.2";
}  // namespace

#define CK(call)                                                                     \
    do {                                                                             \
        cudaError_t _e = (call);                                                     \
        if (_e != cudaSuccess) return h->fail_cuda(_e, #call, __LINE__);             \
    } while (0)

esrrf_status esrrf_handle::fail(esrrf_status s, const std::string& msg) {
    err = msg;
    return s;
}

esrrf_status esrrf_handle::fail_cuda(cudaError_t e, const char* what, int line) {
    err = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) +
          ") in " + what + " at engine.cu:" + std::to_string(line);
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? ESRRF_ERR_NOMEM : ESRRF_ERR_CUDA;
}

namespace {

esrrf_status validate(const esrrf_params& p, std::string& msg) {
    if (p.width < 4 || p.height < 4) return msg = "width and height must be >= 4", ESRRF_ERR_INVALID;
    if (p.magnification < 1 || p.magnification > 16)
        return msg = "magnification must be in [1, 16]", ESRRF_ERR_INVALID;
    if (!(p.fwhm > 0.f) || p.fwhm > 20.f) return msg = "fwhm (radius) must be in (0, 20]", ESRRF_ERR_INVALID;
    if (p.sensitivity < 0 || p.sensitivity > 64) return msg = "sensitivity must be in [0, 64]", ESRRF_ERR_INVALID;
    if (p.n_frame_for_srrf < 1) return msg = "n_frame_for_srrf must be >= 1", ESRRF_ERR_INVALID;
    if (p.n_frames_on_gpu < 1) return msg = "n_frames_on_gpu must be >= 1", ESRRF_ERR_INVALID;
    if (p.frames_per_launch < ESRRF_FRAMES_PER_LAUNCH_TUNED)
        return msg = "frames_per_launch must be >= 0, or ESRRF_FRAMES_PER_LAUNCH_TUNED", ESRRF_ERR_INVALID;
    if (p.n_planes < 0) return msg = "n_planes must be >= 0", ESRRF_ERR_INVALID;
    if (p.n_planes > 0) {
        if (!p.roi || !p.theta_deg || !p.shift_x || !p.shift_y || !p.intensity_coeff)
            return msg = "3-D calibration arrays must all be given", ESRRF_ERR_INVALID;
        if (p.n_planes < 2 || p.n_planes > 9) return msg = "n_planes must be in [2, 9]", ESRRF_ERR_INVALID;
    }
    if (p.interp != ESRRF_INTERP_FHT && p.interp != ESRRF_INTERP_BIC)
        return msg = "interp must be ESRRF_INTERP_FHT or ESRRF_INTERP_BIC", ESRRF_ERR_INVALID;
    // one output slice (2-D frame, or 3-D volume of the 3 x 3 camera tiles' planes) must index in
    // 32 bits: the kernels' per-slice offsets are ints
    const long long M = p.magnification;
    const long long slice = p.n_planes > 0 ? (p.width / 3) * M * ((p.height / 3) * M) * (p.n_planes * M)
                                           : p.width * M * (p.height * M);
    if (slice > 2147483647LL)
        return msg = "output too large: width x height x magnification^2 (x planes x magnification in 3-D) "
                     "must stay below 2^31 pixels per slice",
               ESRRF_ERR_INVALID;
    return ESRRF_OK;
}

int pick_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return -1;
    int best = 0;
    double best_score = -1;
    for (int d = 0; d < n; ++d) {
        int sms = 0, clk = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d);
        cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, d);
        const double score = (double)sms * clk;  // checkDevices' CU x clock rule
        if (score > best_score) {
            best_score = score;
            best = d;
        }
    }
    return best;
}

}  // namespace

esrrf_status esrrf_handle::init(const esrrf_params& params) {
    esrrf_handle* h = this;
    p = params;
    if (p.n_planes > 0) {
        mode = Mode::k3D;
        roi.assign(p.roi, p.roi + p.n_planes);
        theta.assign(p.theta_deg, p.theta_deg + p.n_planes);
        shx.assign(p.shift_x, p.shift_x + p.n_planes);
        shy.assign(p.shift_y, p.shift_y + p.n_planes);
        coeff.assign(p.intensity_coeff, p.intensity_coeff + p.n_planes);
        p.roi = p.theta_deg = p.shift_x = p.shift_y = p.intensity_coeff = nullptr;
    } else {
        mode = p.interp == ESRRF_INTERP_FHT ? Mode::kFHT : Mode::kBIC;
    }
    device = p.device >= 0 ? p.device : pick_device();
    if (device < 0) return fail(ESRRF_ERR_NODEVICE, "no CUDA device");
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&read_stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ev_a));
    CK(cudaEventCreate(&ev_b));
    CK(cudaEventCreate(&ev_c));
    for (int b = 0; b < 2; ++b) {
        CK(cudaEventCreateWithFlags(&ev_host_free[b], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_copied[b], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_dev_free[b], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_fin[b], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_read_done[b], cudaEventDisableTiming));
    }
    drift_x.assign(p.n_frame_for_srrf, 0.f);
    drift_y.assign(p.n_frame_for_srrf, 0.f);
    F = p.frames_per_launch > 0 ? p.frames_per_launch : 8;
    if (p.frames_per_launch == 0 && mode == Mode::kFHT) {
        // FHT path: the block in equal launches of at most 50 frames (fewer launches amortise the
        // per-launch fold of the block accumulators and the last, partial launch: 100-frame blocks
        // of 512 x 512 at M4 run 4 % faster than with 8), within ~4 GB of per-frame buffers
        // (interpolated frames, their gradients, the interpolation scratch: ~5 output planes)
        const double per_frame = 5.0 * sizeof(float) * (double)p.width * p.magnification * p.height * p.magnification;
        const int fmax = (int)std::max(1.0, std::min(50.0, 4e9 / per_frame));
        const int nb = std::max(1, p.n_frame_for_srrf);
        const int launches = (nb + fmax - 1) / fmax;
        F = (nb + launches - 1) / launches;
    } else if (p.frames_per_launch == 0 && mode == Mode::kBIC) {
        // 2-D bicubic path: likewise at most 32 frames (100-frame blocks of 512 x 512 at M4: 4 %
        // faster than 8), within ~2 GB of per-frame buffers (raw frame and its gradients, the 2x
        // gradients and the padded unit-gradient field: ~19 input planes)
        const double per_frame = 19.0 * sizeof(float) * (double)p.width * p.height;
        const int fmax = (int)std::max(1.0, std::min(32.0, 2e9 / per_frame));
        const int nb = std::max(1, p.n_frame_for_srrf);
        const int launches = (nb + fmax - 1) / fmax;
        F = (nb + launches - 1) / launches;
    } else if (p.frames_per_launch == 0 && mode == Mode::k3D) {
        // 3-D path: equal launches of at most 32 timepoints (fewer launches amortise loading the
        // tap tables and the previous values and folding the sums; 9 x 128^2 planes at M3, 200
        // timepoints: 264 Mpx.frames/s against 258 with 8), within ~2 GB of per-timepoint buffers
        // (the camera frame's planes, their 2x gradients and the padded unit-gradient field: ~40
        // camera-frame planes)
        const double per_frame = 40.0 * sizeof(float) * (double)p.width * p.height;
        const int fmax = (int)std::max(1.0, std::min(32.0, 2e9 / per_frame));
        const int nb = std::max(1, p.n_frame_for_srrf);
        const int launches = (nb + fmax - 1) / fmax;
        F = (nb + launches - 1) / launches;
    }

    if (mode == Mode::kFHT) return init_fht();
    return init_bic3d();
}

// Staging buffers, block accumulators and output, shared by the three paths.
esrrf_status esrrf_handle::alloc_common(size_t frame_bytes, long out_pixels) {
    esrrf_handle* h = this;
    raw_frame_bytes = frame_bytes;
    for (int b = 0; b < 2; ++b) {
        CK(cudaMalloc(&d_raw[b], raw_frame_bytes * F));
        CK(cudaMallocHost(&h_stage[b], raw_frame_bytes * F));
    }
    st.pixels = out_pixels;
    CK(cudaMalloc(&st.acc, sizeof(double) * 4 * out_pixels));
    CK(cudaMalloc(&st.prev, sizeof(float) * out_pixels));
    CK(cudaMalloc(&d_out, sizeof(float) * 4 * out_pixels));
    CK(zero_block(st, stream));
    CK(cudaMalloc(&d_shift, sizeof(float) * 2 * (size_t)F));
    CK(cudaStreamSynchronize(stream));
    frame_in_block = 0;
    return ESRRF_OK;
}

esrrf_status esrrf_handle::init_bic3d() {
    esrrf_handle* h = this;
    const int M = p.magnification;
    W = p.width;
    H = p.height;
    bgeo = bic_geometry(p.fwhm, p.sensitivity);
    if (mode == Mode::k3D) {
        P = p.n_planes;
        ws = W / 3;  // nSplits = 3 (LiveSRRF_CL.java:37, 229-230)
        hs = H / 3;
        if (ws < 4 || hs < 4) return fail(ESRRF_ERR_INVALID, "MFM planes must be at least 4x4 pixels");
        std::vector<int> tx0(P), ty0(P);
        std::vector<float> ct(P), sn(P);
        for (int z = 0; z < P; ++z) {
            // ROI index -> tile origin, Math.round((float) W / 3 * i) (LiveSRRF_CL.java:973-978)
            const int i = ((int)roi[z]) % 3;
            const int j = ((int)(roi[z] - (float)i)) / 3;
            tx0[z] = (int)floorf((float)W / 3 * i + 0.5f);
            ty0[z] = (int)floorf((float)H / 3 * j + 0.5f);
            if (roi[z] < 0 || roi[z] > 8 || tx0[z] + ws > W || ty0[z] + hs > H)
                return fail(ESRRF_ERR_INVALID, "calibration ROI outside the camera frame");
            if (!(coeff[z] != 0.f)) return fail(ESRRF_ERR_INVALID, "intensity scaling must be non-zero");
            // -theta in radians as the Java host uploads it (LiveSRRF_CL.java:441)
            const float th = (float)(-(double)theta[z] * M_PI / 180.0);
            ct[z] = cosf(th);
            sn[z] = sinf(th);
        }
        auto up = [&](auto** d, const auto& v) -> cudaError_t {
            cudaError_t e = cudaMalloc((void**)d, sizeof(v[0]) * v.size());
            if (e != cudaSuccess) return e;
            return cudaMemcpy(*d, v.data(), sizeof(v[0]) * v.size(), cudaMemcpyHostToDevice);
        };
        CK(up(&mfm.tile_x0, tx0));
        CK(up(&mfm.tile_y0, ty0));
        CK(up(&mfm.coeff, coeff));
        CK(up(&mfm.cos_t, ct));
        CK(up(&mfm.sin_t, sn));
        CK(up(&mfm.shx, shx));
        CK(up(&mfm.shy, shy));
        PM = P * M;
    } else {
        P = 1;
        ws = W;
        hs = H;
        PM = 1;
    }
    WM = ws * M;
    HM = hs * M;
    const size_t plane = (size_t)ws * hs;
    CK(cudaMalloc(&d_fraw, sizeof(float) * F * P * plane));
    CK(cudaMalloc(&d_gx, sizeof(float) * F * P * plane));
    CK(cudaMalloc(&d_gy, sizeof(float) * F * P * plane));
    CK(cudaMalloc(&d_gxi, sizeof(float) * F * P * 4 * plane));
    CK(cudaMalloc(&d_gyi, sizeof(float) * F * P * 4 * plane));
    if (mode == Mode::k3D) {
        CK(cudaMalloc(&d_planes, sizeof(float) * F * P * plane));
        CK(cudaMalloc(&d_gz, sizeof(float) * F * P * plane));
        CK(cudaMalloc(&d_gzi, sizeof(float) * F * P * 4 * plane));
        CK(rgc3d_tables_build(bgeo, M, ws, hs, P, t3d, stream));
        CK(cudaMalloc(&d_u3, sizeof(float4) * rgc3d_field_float4s(t3d, F)));
        CK(cudaMemsetAsync(d_u3, 0, sizeof(float4) * rgc3d_field_float4s(t3d, F), stream));  // zero halo
    } else {
        CK(bic_tables_build(bgeo, M, ws, hs, tbic, tbic_built, stream));
        if (tbic_built) {
            CK(cudaMalloc(&d_u2, sizeof(float2) * bic_field_float2s(tbic, F)));
            CK(cudaMemsetAsync(d_u2, 0, sizeof(float2) * bic_field_float2s(tbic, F), stream));  // zero halo
        }
    }
    CK(cudaMalloc(&d_mpmap, sizeof(float) * 3 * M * M * M));
    return alloc_common(sizeof(float) * (size_t)W * H, (long)WM * HM * PM);
}

esrrf_status esrrf_handle::init_fht() {
    esrrf_handle* h = this;
    const int M = p.magnification;
    W = p.width;
    H = p.height;
    WM = W * M;
    HM = H * M;
    PM = 1;
    CK(interp_plan_create(plan, W, H, M, p.fht_scale));
    geo = fht_geometry(M, p.fwhm, p.sensitivity);
    use_fused = (p.kernel == 0) && fht_fused_supported(geo);
    if (use_fused) CK(fht_fused_tables(geo, WM, HM, tables, stream));
    const long whM = (long)WM * HM;
    scratch.capacity = F;
    CK(cudaMalloc(&scratch.rowT, sizeof(float) * (size_t)F * interp_rowT_floats(plan)));
    if (plan.tc) CK(cudaMalloc(&scratch.xs, sizeof(float) * (size_t)F * interp_xs_floats(plan)));
    CK(cudaMalloc(&scratch.alt, sizeof(float) * (size_t)F * interp_alt_floats(plan.N)));
    CK(cudaMalloc(&scratch.vec, sizeof(float) * (size_t)F * interp_vec_floats(HM, WM)));
    CK(cudaMalloc(&d_prev_out, sizeof(float) * (size_t)WM * HM));
    CK(cudaMalloc(&d_interp, sizeof(float) * (size_t)F * whM));
    CK(cudaMalloc(&d_gx, sizeof(float) * (size_t)F * whM));
    CK(cudaMalloc(&d_gy, sizeof(float) * (size_t)F * whM));
    return alloc_common(sizeof(float) * (size_t)W * H, whM);  // a float or a uint16 frame
}

void esrrf_handle::release() {
    if (device >= 0) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    if (read_stream) cudaStreamSynchronize(read_stream);
    interp_plan_destroy(plan);
    fht_fused_tables_free(tables);
    fht_drift_tables_free(dtab);
    cudaFree(d_drift);
    d_drift = nullptr;
    if (h_drift_pin) cudaFreeHost(h_drift_pin);
    h_drift_pin = nullptr;
    if (ev_drift) cudaEventDestroy(ev_drift);
    ev_drift = nullptr;
    cudaFree(scratch.rowT);
    cudaFree(scratch.xs);
    cudaFree(scratch.alt);
    cudaFree(scratch.vec);
    cudaFree(d_interp);
    cudaFree(d_gx);
    cudaFree(d_gy);
    cudaFree(d_shift);
    for (int b = 0; b < 2; ++b) {
        cudaFree(d_raw[b]);
        cudaFreeHost(h_stage[b]);
        if (ev_host_free[b]) cudaEventDestroy(ev_host_free[b]);
        if (ev_copied[b]) cudaEventDestroy(ev_copied[b]);
        if (ev_dev_free[b]) cudaEventDestroy(ev_dev_free[b]);
        if (ev_fin[b]) cudaEventDestroy(ev_fin[b]);
        if (ev_read_done[b]) cudaEventDestroy(ev_read_done[b]);
        ev_fin[b] = ev_read_done[b] = nullptr;
        read_pending[b] = false;
    }
    cudaFree(st.acc);
    cudaFree(st.prev);
    cudaFree(d_prev_out);
    cudaFree(d_out);
    cudaFree(d_out2);
    d_out2 = nullptr;
    rgc3d_tables_free(t3d);
    cudaFree(d_u3);
    bic_tables_free(tbic);
    cudaFree(d_u2);
    for (float* b : {d_fraw, d_planes, d_gz, d_gxi, d_gyi, d_gzi, d_mpmap, mfm.coeff, mfm.cos_t,
                     mfm.sin_t, mfm.shx, mfm.shy})
        cudaFree(b);
    cudaFree(mfm.tile_x0);
    cudaFree(mfm.tile_y0);
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    ev_pool.clear();
    if (ev_a) cudaEventDestroy(ev_a);
    if (ev_b) cudaEventDestroy(ev_b);
    if (ev_c) cudaEventDestroy(ev_c);
    if (stream && own_stream) cudaStreamDestroy(stream);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (read_stream) cudaStreamDestroy(read_stream);
    stream = copy_stream = read_stream = nullptr;
}

// loadDriftXYGPUbuffer (LiveSRRF_CL.java:583-595): the block's shifts, stored x M.  On the fused
// FHT path they also go to the device (stream-ordered after the kernels already queued, so a
// later block's shifts never reach an earlier block's launches); the pinned copy is rewritten only
// once its previous upload has been read.
esrrf_status esrrf_handle::set_drift(const float* dx, const float* dy) {
    esrrf_handle* h = this;
    const int n = p.n_frame_for_srrf;
    bool any = false;
    for (int i = 0; i < n; ++i) {
        drift_x[i] = dx ? dx[i] : 0.f;
        drift_y[i] = dy ? dy[i] : 0.f;
        any |= drift_x[i] != 0.f || drift_y[i] != 0.f;
    }
    if (mode != Mode::kFHT || !use_fused || (!any && !d_drift)) return ESRRF_OK;
    CK(cudaSetDevice(device));
    if (!d_drift) {
        CK(cudaMalloc(&d_drift, sizeof(float) * 2 * (size_t)n));
        CK(cudaMallocHost(&h_drift_pin, sizeof(float) * 2 * (size_t)n));
        CK(cudaEventCreateWithFlags(&ev_drift, cudaEventDisableTiming));
    } else {
        CK(cudaEventSynchronize(ev_drift));
    }
    const int M = p.magnification;
    for (int i = 0; i < n; ++i) {
        h_drift_pin[i] = M * drift_x[i];
        h_drift_pin[n + i] = M * drift_y[i];
    }
    CK(cudaMemcpyAsync(d_drift, h_drift_pin, sizeof(float) * 2 * (size_t)n, cudaMemcpyHostToDevice, stream));
    CK(cudaEventRecord(ev_drift, stream));
    return ESRRF_OK;
}

esrrf_status esrrf_handle::reset_block() {
    esrrf_handle* h = this;
    CK(cudaSetDevice(device));
    CK(zero_block(st, stream));
    frame_in_block = 0;
    return ESRRF_OK;
}

// Runs interpolation + RGC for F_now frames that are already in device memory at `src`.
esrrf_status esrrf_handle::process_chunk(const void* src, bool is_u16, int F_now) {
    esrrf_handle* h = this;
    const int M = p.magnification;
    // per-frame drift of this chunk, x magnification (loadDriftXYGPUbuffer, LiveSRRF_CL.java:586-589)
    std::vector<float> sh(2 * F_now);
    bool any_drift = false;
    for (int f = 0; f < F_now; ++f) {
        sh[f] = M * drift_x[frame_in_block + f];
        sh[F_now + f] = M * drift_y[frame_in_block + f];
        any_drift |= (sh[f] != 0.f || sh[F_now + f] != 0.f);
    }
    if (mode != Mode::kFHT) return process_chunk_bic3d(src, is_u16, F_now, sh);
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
    if (timing) {
        esrrf_status r;
        if ((r = timing_event(&e0)) != ESRRF_OK || (r = timing_event(&e1)) != ESRRF_OK ||
            (r = timing_event(&e2)) != ESRRF_OK)
            return r;
        CK(cudaEventRecord(e0, stream));
    }
    CK(interp_run(plan, scratch, src, is_u16, F_now, d_interp, stream, &launches));
    if (timing) CK(cudaEventRecord(e1, stream));
    FhtRgcArgs a{};
    a.interp = d_interp;
    a.W = WM;
    a.H = HM;
    a.F = F_now;
    a.t0 = frame_in_block;
    a.int_weighting = p.int_weighting;
    a.st = st;
    a.prev_out = d_prev_out;
    if (use_fused && !any_drift) {
        CK(fht_rgc_fused(geo, tables, a, stream));
        launches += 1;
    } else if (use_fused && d_drift) {
        // frames with drift: per-frame tap tables and shifted intensities, then the fused kernel
        // (the kernel samples the shifted intensities from its own tiles: no intensity planes)
        if (!dtab.fr) CK(fht_drift_tables_alloc(geo.S, F, 0, dtab));
        const int n = p.n_frame_for_srrf;
        CK(fht_drift_tables_build(geo, d_drift + frame_in_block, d_drift + n + frame_in_block, F_now, dtab,
                                  stream));
        CK(fht_rgc_fused_drift(geo, dtab, a, stream));
        launches += 2;
    } else {
        CK(cudaMemcpyAsync(d_shift, sh.data(), sizeof(float) * 2 * F_now, cudaMemcpyHostToDevice, stream));
        CK(fht_robx(d_interp, WM, HM, F_now, d_gx, d_gy, stream));
        a.gx = d_gx;
        a.gy = d_gy;
        a.shift = d_shift;
        CK(fht_rgc_plain(geo, a, stream));
        launches += 2;
        CK(cudaStreamSynchronize(stream));  // `sh` is a host temporary
    }
    if (timing) CK(cudaEventRecord(e2, stream));
    frame_in_block += F_now;
    return ESRRF_OK;
}

// Events come from a pool so per-launch timing needs no synchronisation until the end of the
// calculate call; triples (interp start, RGC start, RGC end) are read back by collect_timing().
esrrf_status esrrf_handle::timing_event(cudaEvent_t* out) {
    esrrf_handle* h = this;
    if (ev_used == (int)ev_pool.size()) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        ev_pool.push_back(e);
    }
    *out = ev_pool[ev_used++];
    return ESRRF_OK;
}

void esrrf_handle::collect_timing() {
    for (int i = 0; i + 2 < ev_used; i += 3) {
        float t1 = 0.f, t2 = 0.f;
        if (cudaEventElapsedTime(&t1, ev_pool[i], ev_pool[i + 1]) == cudaSuccess) t_interp += t1;
        if (cudaEventElapsedTime(&t2, ev_pool[i + 1], ev_pool[i + 2]) == cudaSuccess) t_rgc += t2;
        ++n_rgc_launches;
    }
    cudaGetLastError();
    ev_used = 0;
}

esrrf_status esrrf_handle::process_chunk_bic3d(const void* src, bool is_u16, int F_now,
                                               const std::vector<float>& sh) {
    esrrf_handle* h = this;
    CK(cudaMemcpyAsync(d_shift, sh.data(), sizeof(float) * 2 * F_now, cudaMemcpyHostToDevice, stream));
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
    if (timing) {
        esrrf_status r;
        if ((r = timing_event(&e0)) != ESRRF_OK || (r = timing_event(&e1)) != ESRRF_OK ||
            (r = timing_event(&e2)) != ESRRF_OK)
            return r;
        CK(cudaEventRecord(e0, stream));
    }
    if (mode == Mode::kBIC) {
        CK(bic_prepare(src, is_u16 ? 1 : 0, W, H, F_now, d_fraw, d_gx, d_gy, d_gxi, d_gyi, stream));
        launches += 3;
    } else {
        CK(mfm_prepare(src, is_u16 ? 1 : 0, W, H, P, ws, hs, F_now, mfm, p.background, d_planes,
                       d_fraw, d_gx, d_gy, d_gz, d_gxi, d_gyi, d_gzi, stream));
        launches += 6;
    }
    if (timing) CK(cudaEventRecord(e1, stream));
    // tabulated taps unless a frame of this launch has drift or the plain kernel was asked for
    bool no_drift = p.kernel == 0;
    for (int i = 0; i < 2 * F_now; ++i) no_drift = no_drift && sh[i] == 0.f;
    if (mode == Mode::kBIC && no_drift && tbic_built) {
        CK(unit_grad2d(d_gxi, d_gyi, ws, hs, F_now, tbic, d_u2, stream));
        BicTabArgs ta{};
        ta.U = d_u2;
        ta.fraw = d_fraw;
        ta.w = ws;
        ta.h = hs;
        ta.M = p.magnification;
        ta.F = F_now;
        ta.t0 = frame_in_block;
        ta.sens = bgeo.sensitivity;
        ta.int_weighting = p.int_weighting;
        ta.tab = tbic;
        ta.st = st;
        CK(bic_rgc_tab(ta, stream));
        launches += 1;
    } else if (mode == Mode::kBIC) {
        BicRgcArgs a{};
        a.fraw = d_fraw;
        a.gxi = d_gxi;
        a.gyi = d_gyi;
        a.w = ws;
        a.h = hs;
        a.M = p.magnification;
        a.F = F_now;
        a.t0 = frame_in_block;
        a.tSS = bgeo.tSS;
        a.tSO = bgeo.tSO;
        a.radius = bgeo.radius;
        a.sens = bgeo.sensitivity;
        a.shift = d_shift;
        a.int_weighting = p.int_weighting;
        a.st = st;
        CK(bic_rgc(a, stream));
    } else {
        if (no_drift) {
            CK(unit_grad3d(d_gxi, d_gyi, d_gzi, ws, hs, P, F_now, t3d, d_u3, stream));
            Rgc3dTabArgs ta{};
            ta.U = d_u3;
            ta.apx = d_fraw;
            ta.w = ws;
            ta.h = hs;
            ta.P = P;
            ta.M = p.magnification;
            ta.F = F_now;
            ta.t0 = frame_in_block;
            ta.sens = bgeo.sensitivity;
            ta.int_weighting = p.int_weighting;
            ta.tab = t3d;
            ta.st = st;
            ta.form = form3d;
            CK(rgc_3d_tab(ta, stream));
            launches += 1;
        }
        Rgc3dArgs a{};
        a.apx = d_fraw;
        a.gxi = d_gxi;
        a.gyi = d_gyi;
        a.gzi = d_gzi;
        a.w = ws;
        a.h = hs;
        a.P = P;
        a.M = p.magnification;
        a.F = F_now;
        a.t0 = frame_in_block;
        a.tSS = bgeo.tSS;
        a.tSO = bgeo.tSO;
        a.radius = bgeo.radius;
        a.sens = bgeo.sensitivity;
        a.shift = d_shift;
        a.int_weighting = p.int_weighting;
        a.st = st;
        if (!no_drift) CK(rgc_3d(a, stream));
    }
    launches += 1;
    if (timing) CK(cudaEventRecord(e2, stream));
    CK(cudaStreamSynchronize(stream));  // `sh` is a host temporary
    frame_in_block += F_now;
    return ESRRF_OK;
}

esrrf_status esrrf_handle::calculate(const void* frames, bool is_u16, int n, bool on_device) {
    esrrf_handle* h = this;
    if (n < 0 || (n > 0 && !frames)) return fail(ESRRF_ERR_INVALID, "frames must be non-null");
    if (frame_in_block + n > p.n_frame_for_srrf)
        return fail(ESRRF_ERR_STATE, "more frames pushed than n_frame_for_srrf in this block");
    CK(cudaSetDevice(device));
    launches = 0;
    t_interp = t_rgc = 0.f;
    n_rgc_launches = 0;
    ev_used = 0;
    const size_t fbytes = is_u16 ? sizeof(uint16_t) * (size_t)W * H : sizeof(float) * (size_t)W * H;
    if (on_device) {
        for (int s = 0; s < n; s += F) {
            if (cancel.exchange(0)) return ESRRF_CANCELLED;
            const int F_now = std::min(F, n - s);
            esrrf_status r = process_chunk((const char*)frames + fbytes * s, is_u16, F_now);
            if (r != ESRRF_OK) return r;
        }
        CK(cudaStreamSynchronize(stream));
        if (timing) collect_timing();
        return ESRRF_OK;
    }
    // Host frames: double-buffered pinned staging; the copy of chunk s+1 overlaps the kernels of
    // chunk s (copy stream + events).
    cudaPointerAttributes attr{};
    const bool pinned = cudaPointerGetAttributes(&attr, frames) == cudaSuccess &&
                        attr.type == cudaMemoryTypeHost;
    cudaGetLastError();
    for (int s = 0; s < n; s += F, ++chunk_seq) {
        if (cancel.exchange(0)) {
            cudaStreamSynchronize(copy_stream);
            cudaStreamSynchronize(stream);
            return ESRRF_CANCELLED;
        }
        const int b = (int)(chunk_seq & 1);
        const int F_now = std::min(F, n - s);
        const char* src = (const char*)frames + fbytes * s;
        if (chunk_seq >= 2) CK(cudaStreamWaitEvent(copy_stream, ev_dev_free[b], 0));
        if (pinned) {
            CK(cudaMemcpyAsync(d_raw[b], src, fbytes * F_now, cudaMemcpyHostToDevice, copy_stream));
        } else {
            if (chunk_seq >= 2) CK(cudaEventSynchronize(ev_host_free[b]));
            memcpy(h_stage[b], src, fbytes * F_now);
            CK(cudaMemcpyAsync(d_raw[b], h_stage[b], fbytes * F_now, cudaMemcpyHostToDevice, copy_stream));
            CK(cudaEventRecord(ev_host_free[b], copy_stream));
        }
        CK(cudaEventRecord(ev_copied[b], copy_stream));
        CK(cudaStreamWaitEvent(stream, ev_copied[b], 0));
        esrrf_status r = process_chunk(d_raw[b], is_u16, F_now);
        if (r != ESRRF_OK) return r;
        CK(cudaEventRecord(ev_dev_free[b], stream));
    }
    // The caller's frames are consumed once their copies are done; the last chunks' kernels may
    // still run (reads, resets and drift uploads queue behind them on the same stream).
    if (timing) {
        CK(cudaStreamSynchronize(stream));
        collect_timing();
    } else {
        CK(cudaStreamSynchronize(copy_stream));
    }
    return ESRRF_OK;
}

esrrf_status esrrf_handle::read(float* out, bool on_device) {
    esrrf_handle* h = this;
    CK(cudaSetDevice(device));
    if (frame_in_block == 0) return fail(ESRRF_ERR_STATE, "no frames accumulated in this block");
    // slot 0 may still be the source of a queued read-back
    if (read_pending[0]) CK(cudaStreamWaitEvent(stream, ev_read_done[0], 0));
    // kernelCalculateVar + NaN->0 (LiveSRRF_CL.java:749-794) on the block accumulated so far.
    CK(finalize_block(st, p.n_frame_for_srrf, mode == Mode::kBIC ? 1 : 0, d_out, stream));
    // MP map correction runs on the bicubic and 3-D paths only (LiveSRRF_CL.java:762-770)
    if (p.mp_correction && mode != Mode::kFHT)
        CK(mp_correct(d_out, ws, hs, P, p.magnification, mode == Mode::k3D ? 1 : 0, d_mpmap, stream));
    const size_t bytes = sizeof(float) * 4 * (size_t)st.pixels;
    CK(cudaMemcpyAsync(out, d_out, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       stream));
    bool tc_failed = false;
    CK(interp_tc_check(plan, stream, &tc_failed));  // synchronises the stream
    if (tc_failed)
        return fail(ESRRF_ERR_TIMEOUT, "interpolation tensor-core pass: a bounded wait gave up");
    return ESRRF_OK;
}

// The block's cumulants into one of two output slots and a device-to-host copy of it queued on
// read_stream; returns at once.  The next block's frames can be pushed while the copy runs.
esrrf_status esrrf_handle::read_async(float* out) {
    esrrf_handle* h = this;
    CK(cudaSetDevice(device));
    if (frame_in_block == 0) return fail(ESRRF_ERR_STATE, "no frames accumulated in this block");
    const size_t bytes = sizeof(float) * 4 * (size_t)st.pixels;
    if (!d_out2) CK(cudaMalloc(&d_out2, bytes));
    const int s = read_slot;
    read_slot ^= 1;
    float* dst = s ? d_out2 : d_out;
    if (read_pending[s]) CK(cudaStreamWaitEvent(stream, ev_read_done[s], 0));
    CK(finalize_block(st, p.n_frame_for_srrf, mode == Mode::kBIC ? 1 : 0, dst, stream));
    if (p.mp_correction && mode != Mode::kFHT)
        CK(mp_correct(dst, ws, hs, P, p.magnification, mode == Mode::k3D ? 1 : 0, d_mpmap, stream));
    CK(cudaEventRecord(ev_fin[s], stream));
    CK(cudaStreamWaitEvent(read_stream, ev_fin[s], 0));
    CK(cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, read_stream));
    CK(cudaEventRecord(ev_read_done[s], read_stream));
    read_pending[s] = true;
    return ESRRF_OK;
}

esrrf_status esrrf_handle::drain() {
    esrrf_handle* h = this;
    CK(cudaSetDevice(device));
    CK(cudaStreamSynchronize(copy_stream));
    CK(cudaStreamSynchronize(stream));
    CK(cudaStreamSynchronize(read_stream));
    read_pending[0] = read_pending[1] = false;
    bool tc_failed = false;
    CK(interp_tc_check(plan, stream, &tc_failed));
    if (tc_failed)
        return fail(ESRRF_ERR_TIMEOUT, "interpolation tensor-core pass: a bounded wait gave up");
    return ESRRF_OK;
}

// ------------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------------
extern "C" {

const char* esrrf_get_version(void) { return kVersion; }

esrrf_status esrrf_device_count(int* count) {
    if (!count) return ESRRF_ERR_INVALID;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
        return ESRRF_ERR_NODEVICE;
    }
    *count = n;
    return ESRRF_OK;
}

esrrf_status esrrf_device_info(int device, char* name, size_t name_len, int* sm_count,
                               int* clock_mhz) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        cudaGetLastError();
        return ESRRF_ERR_INVALID;
    }
    if (name && name_len) {
        strncpy(name, prop.name, name_len - 1);
        name[name_len - 1] = 0;
    }
    int clk = 0;
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, device);
    if (sm_count) *sm_count = prop.multiProcessorCount;
    if (clock_mhz) *clock_mhz = clk / 1000;
    return ESRRF_OK;
}

void esrrf_default_params(esrrf_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->magnification = 5;
    p->fwhm = 2.0f;
    p->sensitivity = 1;
    p->n_frames_on_gpu = 100;
    p->n_frame_for_srrf = 100;
    p->block_length = 20000;
    p->device = -1;
    p->int_weighting = 1;
    p->mp_correction = 0;
    p->interp = ESRRF_INTERP_FHT;
    p->fht_scale = ESRRF_FHT_SCALE_MEAN_PRESERVING;
    p->kernel = 0;
    p->frames_per_launch = 0;
    p->pixel_size_um = 0.1f;
}

esrrf_status esrrf_create(const esrrf_params* params, esrrf_handle** out) {
    if (!params || !out) return ESRRF_ERR_INVALID;
    *out = nullptr;
    std::string msg;
    esrrf_status s = validate(*params, msg);
    if (s != ESRRF_OK) {
        std::lock_guard<std::mutex> lk(g_err_mu);
        g_create_error = msg;
        return s;
    }
    esrrf_params prm = *params;
    TuneChoice tuned;
    if (prm.frames_per_launch == ESRRF_FRAMES_PER_LAUNCH_TUNED) {
        // measured (or cached) frames per launch and kernel form, then the handle proper
        s = tune_engine(prm, tuned, msg);
        if (s != ESRRF_OK) {
            std::lock_guard<std::mutex> lk(g_err_mu);
            g_create_error = msg;
            return s;
        }
        prm.frames_per_launch = tuned.frames_per_launch;
    }
    esrrf_handle* h = new (std::nothrow) esrrf_handle();
    if (!h) return ESRRF_ERR_NOMEM;
    h->form3d = tuned.form;
    h->tune_report = tuned.report;
    s = h->init(prm);
    if (s != ESRRF_OK) {
        {
            std::lock_guard<std::mutex> lk(g_err_mu);
            g_create_error = h->err;
        }
        h->release();
        delete h;
        return s;
    }
    *out = h;
    return ESRRF_OK;
}

esrrf_status esrrf_destroy(esrrf_handle* h) {
    if (!h) return ESRRF_ERR_INVALID;
    h->release();
    delete h;
    return ESRRF_OK;
}

esrrf_status esrrf_set_drift(esrrf_handle* h, const float* dx, const float* dy, int n) {
    if (!h) return ESRRF_ERR_INVALID;
    if (n != h->p.n_frame_for_srrf && !(n == 0 && !dx && !dy))
        return h->fail(ESRRF_ERR_INVALID, "drift arrays must hold n_frame_for_srrf values");
    // the kernels turn shifts x M into integer tile offsets: finite and at most 1e6 raw pixels
    for (int i = 0; i < n; ++i)
        if ((dx && !(std::fabs(dx[i]) <= 1e6f)) || (dy && !(std::fabs(dy[i]) <= 1e6f)))
            return h->fail(ESRRF_ERR_INVALID, "drift shifts must be finite and at most 1e6 pixels");
    return h->set_drift(dx, dy);
}

esrrf_status esrrf_reset_frame_position(esrrf_handle* h) {
    if (!h) return ESRRF_ERR_INVALID;
    return h->reset_block();
}

esrrf_status esrrf_calculate_srrf_u16(esrrf_handle* h, const uint16_t* frames, int n) {
    if (!h) return ESRRF_ERR_INVALID;
    return h->calculate(frames, true, n, false);
}
esrrf_status esrrf_calculate_srrf_f32(esrrf_handle* h, const float* frames, int n) {
    if (!h) return ESRRF_ERR_INVALID;
    return h->calculate(frames, false, n, false);
}
esrrf_status esrrf_calculate_srrf_u16_device(esrrf_handle* h, const uint16_t* frames, int n) {
    if (!h) return ESRRF_ERR_INVALID;
    return h->calculate(frames, true, n, true);
}
esrrf_status esrrf_calculate_srrf_f32_device(esrrf_handle* h, const float* frames, int n) {
    if (!h) return ESRRF_ERR_INVALID;
    return h->calculate(frames, false, n, true);
}

esrrf_status esrrf_read_srrf(esrrf_handle* h, float* out) {
    if (!h || !out) return ESRRF_ERR_INVALID;
    return h->read(out, false);
}
esrrf_status esrrf_read_srrf_device(esrrf_handle* h, float* out) {
    if (!h || !out) return ESRRF_ERR_INVALID;
    return h->read(out, true);
}

esrrf_status esrrf_tune_report(const esrrf_handle* h, char* buf, size_t len) {
    if (!h || !buf || len == 0) return ESRRF_ERR_INVALID;
    const std::string& r = h->tune_report.empty() ? std::string("{\"source\": \"off\"}") : h->tune_report;
    strncpy(buf, r.c_str(), len - 1);
    buf[len - 1] = 0;
    return r.size() < len ? ESRRF_OK : ESRRF_ERR_INVALID;
}

esrrf_status esrrf_frames_per_launch(const esrrf_handle* h, int* frames) {
    if (!h || !frames) return ESRRF_ERR_INVALID;
    *frames = h->F;
    return ESRRF_OK;
}

esrrf_status esrrf_output_shape(const esrrf_handle* h, int* wm, int* hm, int* pm) {
    if (!h) return ESRRF_ERR_INVALID;
    if (wm) *wm = h->WM;
    if (hm) *hm = h->HM;
    if (pm) *pm = h->PM;
    return ESRRF_OK;
}

esrrf_status esrrf_read_gradients(esrrf_handle* h, float* out, size_t out_len) {
    if (!h || !out) return ESRRF_ERR_INVALID;
    if (cudaSetDevice(h->device) != cudaSuccess) return ESRRF_ERR_CUDA;
    if (h->mode != esrrf_handle::Mode::kFHT) {
        // 2x-resampled gradient components of the first frame of the last push
        const size_t plane = (size_t)4 * h->ws * h->hs * h->P;
        const int nc = h->mode == esrrf_handle::Mode::k3D ? 3 : 2;
        if (out_len < nc * plane) return h->fail(ESRRF_ERR_INVALID, "output buffer too small");
        const float* src[3] = {h->d_gxi, h->d_gyi, h->d_gzi};
        for (int c = 0; c < nc; ++c)
            if (cudaMemcpyAsync(out + c * plane, src[c], sizeof(float) * plane, cudaMemcpyDeviceToHost,
                                h->stream) != cudaSuccess) {
                cudaGetLastError();
                return h->fail(ESRRF_ERR_CUDA, "gradient read-back failed");
            }
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) return h->fail(ESRRF_ERR_CUDA, "sync failed");
        return ESRRF_OK;
    }
    const size_t plane = (size_t)h->WM * h->HM;
    if (out_len < 2 * plane) return h->fail(ESRRF_ERR_INVALID, "output buffer too small");
    // The interpolated frames of the last chunk are still resident: recompute the gradient of
    // the first one (readGradientBuffers reads frame 0 of the last load).
    if (fht_robx(h->d_interp, h->WM, h->HM, 1, h->d_gx, h->d_gy, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(out, h->d_gx, sizeof(float) * plane, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(out + plane, h->d_gy, sizeof(float) * plane, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
        cudaGetLastError();
        return h->fail(ESRRF_ERR_CUDA, "gradient read-back failed");
    }
    return ESRRF_OK;
}

esrrf_status esrrf_read_aligned_pixels(esrrf_handle* h, float* out, size_t out_len) {
    if (!h || !out) return ESRRF_ERR_INVALID;
    if (h->mode != esrrf_handle::Mode::k3D) return h->fail(ESRRF_ERR_STATE, "aligned pixels exist on the 3-D path only");
    if (cudaSetDevice(h->device) != cudaSuccess) return ESRRF_ERR_CUDA;
    const size_t n = (size_t)h->P * h->ws * h->hs;  // first frame of the last push
    if (out_len < n) return h->fail(ESRRF_ERR_INVALID, "output buffer too small");
    if (cudaMemcpyAsync(out, h->d_fraw, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
        cudaGetLastError();
        return h->fail(ESRRF_ERR_CUDA, "aligned-pixel read-back failed");
    }
    for (size_t i = 0; i < n; ++i)
        if (std::isnan(out[i])) out[i] = 0.f;
    return ESRRF_OK;
}

esrrf_status esrrf_read_mp_maps(esrrf_handle* h, float* out, size_t out_len) {
    if (!h || !out) return ESRRF_ERR_INVALID;
    if (h->mode == esrrf_handle::Mode::kFHT || !h->p.mp_correction)
        return h->fail(ESRRF_ERR_STATE, "MP maps exist on the bicubic and 3-D paths with MP correction only");
    if (cudaSetDevice(h->device) != cudaSuccess) return ESRRF_ERR_CUDA;
    const int M = h->p.magnification;
    const size_t n = (size_t)3 * M * M * (h->mode == esrrf_handle::Mode::k3D ? M : 1);
    if (out_len < n) return h->fail(ESRRF_ERR_INVALID, "output buffer too small");
    if (cudaMemcpyAsync(out, h->d_mpmap, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
        cudaGetLastError();
        return h->fail(ESRRF_ERR_CUDA, "MP map read-back failed");
    }
    for (size_t i = 0; i < n; ++i)
        if (std::isnan(out[i])) out[i] = 0.f;
    return ESRRF_OK;
}

esrrf_status esrrf_finish_queue(esrrf_handle* h) {
    if (!h) return ESRRF_ERR_INVALID;
    return h->drain();
}

esrrf_status esrrf_read_srrf_async(esrrf_handle* h, float* out) {
    if (!h || !out) return ESRRF_ERR_INVALID;
    return h->read_async(out);
}

esrrf_status esrrf_request_cancel(esrrf_handle* h) {
    if (!h) return ESRRF_ERR_INVALID;
    h->cancel.store(1);
    return ESRRF_OK;
}

const char* esrrf_last_error(const esrrf_handle* h) {
    if (!h) {
        std::lock_guard<std::mutex> lk(g_err_mu);
        return g_create_error.c_str();
    }
    return h->err.c_str();
}

esrrf_status esrrf_last_timing(const esrrf_handle* h, float* interp_ms, float* rgc_ms, int* launches) {
    if (!h) return ESRRF_ERR_INVALID;
    if (interp_ms) *interp_ms = h->t_interp;
    if (rgc_ms) *rgc_ms = h->t_rgc;
    if (launches) *launches = h->launches;
    return ESRRF_OK;
}

esrrf_status esrrf_set_stream(esrrf_handle* h, void* stream) {
    if (!h) return ESRRF_ERR_INVALID;
    if (cudaSetDevice(h->device) != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess) {
        cudaGetLastError();
        return h->fail(ESRRF_ERR_CUDA, "could not drain the current stream");
    }
    if (h->own_stream) cudaStreamDestroy(h->stream);
    if (stream) {
        h->stream = (cudaStream_t)stream;
        h->own_stream = false;
    } else {
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            return h->fail(ESRRF_ERR_CUDA, "stream creation failed");
        }
        h->own_stream = true;
    }
    return ESRRF_OK;
}

esrrf_status esrrf_set_timing(esrrf_handle* h, int enable) {
    if (!h) return ESRRF_ERR_INVALID;
    h->timing = enable != 0;
    return ESRRF_OK;
}

}  // extern "C"
