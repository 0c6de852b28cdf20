// engine.h -- the esrrf_handle behind the C ABI: one per LiveSRRF_CL-equivalent engine.
#pragma once
#include <atomic>
#include <string>
#include <vector>

#include "../../include/esrrf.h"
#include "esrrf_internal.h"

// Choice of the autotuner (tune.cu) for one parameter set.
struct TuneChoice {
    int frames_per_launch = 0;
    int form = 0;
    std::string report;
};
// Times candidate frames-per-launch values (and, in 3-D, kernel forms) on synthetic frames of the
// parameters' size, or reads an earlier result from the cache file; fills `out`.
esrrf_status tune_engine(const esrrf_params& p, TuneChoice& out, std::string& msg);

struct esrrf_handle {
    enum class Mode { kFHT, kBIC, k3D };

    esrrf_params p{};
    Mode mode = Mode::kFHT;
    std::vector<float> roi, theta, shx, shy, coeff;  // 3-D calibration copies
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;

    int W = 0, H = 0;           // raw frame size handled by the kernels
    int WM = 0, HM = 0, PM = 1; // output plane size and number of output planes
    int F = 8;                  // frames per interpolation + RGC launch

    // FHT path
    esrrf::InterpPlan plan;
    esrrf::InterpScratch scratch;
    esrrf::FhtGeometry geo;
    esrrf::FhtFusedTables tables;
    bool use_fused = false;
    float* d_interp = nullptr;
    float* d_gx = nullptr;
    float* d_gy = nullptr;
    float* d_shift = nullptr;
    // drift on the fused kernel: the block's shifts x M on the device ([2][n_frame_for_srrf],
    // uploaded by esrrf_set_drift from a pinned copy on the compute stream), per-launch tables
    float* d_drift = nullptr;
    float* h_drift_pin = nullptr;
    cudaEvent_t ev_drift = nullptr;   // the last upload of h_drift_pin has been read
    esrrf::FhtDriftTables dtab;

    // 2-D bicubic and 3-D paths
    esrrf::BicGeometry bgeo;
    esrrf::Mfm3dTables mfm;
    int P = 1, ws = 0, hs = 0;  // planes and per-plane size (3-D); ws = W, hs = H in 2-D
    float* d_fraw = nullptr;    // [F][P][hs][ws] float frames / aligned planes
    float* d_planes = nullptr;  // [F][P][hs][ws] split planes before alignment (3-D)
    float* d_gz = nullptr;
    float* d_gxi = nullptr;     // [F][P][2hs][2ws]
    float* d_gyi = nullptr;
    float* d_gzi = nullptr;
    float* d_mpmap = nullptr;   // [3][M^2 or M^3]
    esrrf::Rgc3dTables t3d;     // 3-D tap tables per sub-pixel phase (launches without drift)
    float4* d_u3 = nullptr;     // [F][P][2hs][2ws] unit gradient field
    esrrf::BicTables tbic;      // 2-D bicubic tap tables per sub-pixel phase (launches without drift)
    bool tbic_built = false;
    float2* d_u2 = nullptr;     // [F][2hs][2ws] padded unit gradient field (2-D bicubic)

    // input staging (double-buffered)
    size_t raw_frame_bytes = 0;
    void* d_raw[2] = {nullptr, nullptr};
    void* h_stage[2] = {nullptr, nullptr};
    cudaEvent_t ev_host_free[2] = {nullptr, nullptr};
    cudaEvent_t ev_copied[2] = {nullptr, nullptr};
    cudaEvent_t ev_dev_free[2] = {nullptr, nullptr};

    long chunk_seq = 0;  // host chunks staged so far: a staging buffer is reused only after the
                         // kernels of its previous chunk (possibly from an earlier call) are done

    // block accumulators and output
    esrrf::BlockState st;
    float* d_prev_out = nullptr;  // [HM][WM] lets a fused launch split its frames into groups (FHT)
    float* d_out = nullptr;
    // queued read-back (esrrf_read_srrf_async): two output slots, slot 0 = d_out; the
    // device-to-host copies run on read_stream and overlap the next block's kernels
    float* d_out2 = nullptr;
    cudaStream_t read_stream = nullptr;
    cudaEvent_t ev_fin[2] = {nullptr, nullptr};
    cudaEvent_t ev_read_done[2] = {nullptr, nullptr};
    bool read_pending[2] = {false, false};
    int read_slot = 0;
    int frame_in_block = 0;     // nCurrentFrame[0] of the reference
    std::vector<float> drift_x, drift_y;

    // control, errors, timing
    std::atomic<int> cancel{0};
    std::string err;
    bool timing = false;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_c = nullptr;
    std::vector<cudaEvent_t> ev_pool;  // [3 per chunk] interp start, RGC start, RGC end
    int ev_used = 0;
    float t_interp = 0.f, t_rgc = 0.f;
    int launches = 0, n_rgc_launches = 0;
    bool own_stream = true;
    int form3d = 0;             // tabulated 3-D kernel form (kRgc3d*; 0: default choice)
    std::string tune_report;    // what the autotuner measured or read (empty: not tuned)

    esrrf_status timing_event(cudaEvent_t* out);
    void collect_timing();

    esrrf_status init(const esrrf_params& params);
    esrrf_status init_fht();
    esrrf_status init_bic3d();
    esrrf_status alloc_common(size_t raw_frame_bytes, long out_pixels);
    void release();
    esrrf_status reset_block();
    esrrf_status set_drift(const float* dx, const float* dy);
    esrrf_status calculate(const void* frames, bool is_u16, int n, bool on_device);
    esrrf_status process_chunk(const void* src, bool is_u16, int F_now);
    esrrf_status process_chunk_bic3d(const void* src, bool is_u16, int F_now,
                                     const std::vector<float>& sh);
    esrrf_status read(float* out, bool on_device);
    esrrf_status read_async(float* host_out);
    esrrf_status drain();  // every queued kernel and copy done, tensor-core wait flag checked
    esrrf_status fail(esrrf_status s, const std::string& msg);
    esrrf_status fail_cuda(cudaError_t e, const char* what, int line);
};
