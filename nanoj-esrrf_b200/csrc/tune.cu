// tune.cu -- the engine's autotuner: frames per launch (and the 3-D kernel form) measured per
// parameter set and cached on disk.
//
// The reference sizes its GPU loads from a memory model (calculatenFrameOnGPU / predictMemoryUsed,
// gui/LiveSRRF_optimised_.java:763-877) and launches one kernel per frame.  Here a block is cut into
// equal launches of F frames; F trades the per-launch costs (the fold of the FP32 launch sums into
// the FP64 block accumulators, the interpolation's tile quantisation, the partial last launch of a
// block, the first launch's upload that cannot overlap) against the buffers it needs.  The tuner
// times one block of synthetic frames through a temporary engine for each candidate, keeps the
// fastest, and caches the choice in a text file keyed by the device and the parameters that set
// the cost (path, frame size, magnification, tap box, block length, intensity weighting, planes).
#include <dlfcn.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/esrrf.h"
#include "engine.h"
#include "esrrf_internal.h"

using namespace esrrf;

namespace {

std::mutex g_tune_mu;

// Synthetic camera frames: background, shot-noise-like hash noise and a smooth pattern whose
// gradients point in every direction, so the RGC's inward test takes both branches.
__global__ void synth_frames_kernel(float* __restrict__ f, int W, int H, int n) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long total = (long)W * H * n;
    if (i >= total) return;
    const int x = (int)(i % W), y = (int)((i / W) % H), t = (int)(i / ((long)W * H));
    unsigned h = (unsigned)i * 2654435761u ^ (unsigned)t * 40503u;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    const float noise = (float)(h & 0xFFFF) * (1.0f / 65536.0f);
    const float pattern = __sinf(0.37f * x + 0.5f * t) * __cosf(0.23f * y - 0.3f * t);
    f[i] = 100.f + 20.f * noise + 200.f * fmaxf(pattern, 0.f);
}

const char* form_name(int form) {
    switch (form) {
        case kRgc3dTwoCells: return "two-cells";
        case kRgc3dSlab: return "slab";
        case kRgc3dL1: return "l1";
        default: return "default";
    }
}

std::string cache_path() {
    const char* env = std::getenv("ESRRF_TUNE_CACHE");
    if (env && *env) return env;
    Dl_info info;
    if (dladdr((void*)&synth_frames_kernel, &info) && info.dli_fname) {
        std::string lib = info.dli_fname;
        const size_t slash = lib.find_last_of('/');
        return (slash == std::string::npos ? std::string(".") : lib.substr(0, slash)) + "/esrrf_tune.txt";
    }
    return "esrrf_tune.txt";
}

std::string key_of(const esrrf_params& p, const std::string& devname) {
    std::ostringstream k;
    const bool fht = p.n_planes == 0 && p.interp == ESRRF_INTERP_FHT;
    k << "v1|" << devname << "|" << (p.n_planes > 0 ? "3d" : fht ? "fht" : "bic") << "|" << p.width << "x"
      << p.height << "|M" << p.magnification << "|";
    if (fht) k << "box" << fht_geometry(p.magnification, p.fwhm, 1).S;
    else k << "r" << p.fwhm;
    k << "|n" << p.n_frame_for_srrf << "|iw" << p.int_weighting << "|planes" << p.n_planes << "|k" << p.kernel;
    std::string s = k.str();
    for (char& c : s)
        if (c == ' ' || c == '\t' || c == '\n') c = '_';
    return s;
}

bool cache_get(const std::string& path, const std::string& key, TuneChoice& out, double& ms) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    bool found = false;
    while (std::getline(f, line)) {
        std::istringstream ls(line);
        std::string k;
        int F = 0, form = 0;
        double t = 0;
        if (!(ls >> k >> F >> form >> t) || k != key || F < 1) continue;
        out.frames_per_launch = F;
        out.form = form;
        ms = t;
        found = true;  // the last entry of a key wins
    }
    return found;
}

void cache_put(const std::string& path, const std::string& key, const TuneChoice& c, double ms) {
    std::ofstream f(path, std::ios::app);
    if (f) f << key << " " << c.frames_per_launch << " " << c.form << " " << ms << "\n";
}

// Candidate frames per launch for blocks of n frames: every equal cut of the block into launches
// of about 8 .. 64 frames (3-D: 4 .. 32 timepoints) that fits the per-frame buffer budget.
std::vector<int> candidates(const esrrf_params& p, int n) {
    std::vector<int> targets;
    double per_frame = 0, budget = 4e9;
    if (p.n_planes > 0) {
        targets = {4, 8, 16, 32};
        per_frame = 40.0 * sizeof(float) * (double)p.width * p.height;
        budget = 2e9;
    } else if (p.interp == ESRRF_INTERP_FHT) {
        targets = {8, 12, 16, 25, 34, 50, 64};
        per_frame = 5.0 * sizeof(float) * (double)p.width * p.magnification * p.height * p.magnification;
    } else {
        targets = {8, 16, 25, 32, 50, 64};
        per_frame = 19.0 * sizeof(float) * (double)p.width * p.height;
        budget = 2e9;
    }
    const int fcap = (int)std::max(1.0, std::floor(budget / per_frame));
    std::vector<int> out;
    for (int f : targets) {
        f = std::min({f, fcap, n});
        const int launches = (n + f - 1) / f;
        const int F = (n + launches - 1) / launches;
        if (std::find(out.begin(), out.end(), F) == out.end()) out.push_back(F);
    }
    std::sort(out.begin(), out.end());
    return out;
}

// Device time of one block (reset, all frames, read) through a temporary engine; min of `reps`.
esrrf_status time_candidate(const esrrf_params& base, int F, int form, const float* d_frames, int n,
                            float* d_out, int reps, double& ms, std::string& msg) {
    esrrf_params p = base;
    p.frames_per_launch = F;
    p.n_frame_for_srrf = n;
    p.n_frames_on_gpu = n;
    esrrf_handle* h = new esrrf_handle();
    h->form3d = form;
    esrrf_status s = h->init(p);
    if (s != ESRRF_OK) {
        msg = "autotuner: " + h->err;
        h->release();
        delete h;
        return s;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    ms = 1e30;
    for (int r = 0; r <= reps && s == ESRRF_OK; ++r) {  // run 0 warms up
        cudaEventRecord(e0, h->stream);
        if ((s = h->reset_block()) == ESRRF_OK && (s = h->calculate(d_frames, false, n, true)) == ESRRF_OK)
            s = h->read(d_out, true);
        cudaEventRecord(e1, h->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) s = ESRRF_ERR_CUDA;
        float t = 0.f;
        if (s == ESRRF_OK && r > 0 && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess) ms = std::min(ms, (double)t);
    }
    if (s != ESRRF_OK) msg = "autotuner: " + h->err;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->release();
    delete h;
    return s;
}

}  // namespace

esrrf_status tune_engine(const esrrf_params& params, TuneChoice& out, std::string& msg) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    esrrf_params p = params;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        msg = "no CUDA device";
        return ESRRF_ERR_NODEVICE;
    }
    int dev = p.device;
    if (dev < 0) {  // the device the engine itself picks: most SMs x clock
        double best = -1;
        for (int d = 0; d < ndev; ++d) {
            int sms = 0, clk = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d);
            cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, d);
            if ((double)sms * clk > best) best = (double)sms * clk, dev = d;
        }
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        msg = "autotuner: device query failed";
        return ESRRF_ERR_CUDA;
    }
    p.device = dev;
    const std::string key = key_of(p, std::string(prop.name) + "_sm" + std::to_string(prop.multiProcessorCount));
    const std::string path = cache_path();
    double ms = 0;
    if (cache_get(path, key, out, ms)) {
        std::ostringstream r;
        r << "{\"source\": \"cache\", \"key\": \"" << key << "\", \"frames_per_launch\": " << out.frames_per_launch
          << ", \"form\": \"" << form_name(out.form) << "\", \"ms_per_frame\": " << ms << ", \"file\": \"" << path
          << "\"}";
        out.report = r.str();
        return ESRRF_OK;
    }
    // one block of synthetic frames (at most 200: the per-launch costs show within that)
    const int n = std::min(p.n_frame_for_srrf, 200);
    const std::vector<int> Fs = candidates(p, n);
    std::vector<int> forms = {kRgc3dAuto};
    if (p.n_planes > 0 && p.kernel == 0) forms = {kRgc3dTwoCells, kRgc3dSlab, kRgc3dL1};
    if (cudaSetDevice(dev) != cudaSuccess) {
        cudaGetLastError();
        msg = "autotuner: cudaSetDevice failed";
        return ESRRF_ERR_CUDA;
    }
    float* d_frames = nullptr;
    float* d_out = nullptr;
    const long planes_out = p.n_planes > 0 ? (long)p.n_planes * p.magnification : 1;
    const long ws = p.n_planes > 0 ? p.width / 3 : p.width, hs = p.n_planes > 0 ? p.height / 3 : p.height;
    const size_t nin = (size_t)n * p.width * p.height;
    const size_t nout = 4 * (size_t)planes_out * ws * p.magnification * hs * p.magnification;
    if (cudaMalloc(&d_frames, sizeof(float) * nin) != cudaSuccess ||
        cudaMalloc(&d_out, sizeof(float) * nout) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d_frames);
        msg = "autotuner: no memory for the trial block";
        return ESRRF_ERR_NOMEM;
    }
    synth_frames_kernel<<<(unsigned)((nin + 255) / 256), 256>>>(d_frames, p.width, p.height, n);
    esrrf_status s = cudaDeviceSynchronize() == cudaSuccess ? ESRRF_OK : ESRRF_ERR_CUDA;
    std::ostringstream cand;
    double best = 1e30;
    for (int form : forms)
        for (int F : Fs) {
            if (s != ESRRF_OK) break;
            double t = 0;
            s = time_candidate(p, F, form, d_frames, n, d_out, 2, t, msg);
            if (s != ESRRF_OK) break;
            const double per_frame = t / n;
            cand << (cand.tellp() > 0 ? ", " : "") << "{\"frames_per_launch\": " << F << ", \"form\": \""
                 << form_name(form) << "\", \"ms_per_frame\": " << per_frame << "}";
            if (per_frame < best) {
                best = per_frame;
                out.frames_per_launch = F;
                out.form = form;
            }
        }
    cudaFree(d_frames);
    cudaFree(d_out);
    if (s != ESRRF_OK) return s;
    // the choice for blocks of n frames is used as the launch size of the caller's blocks; recut
    // the caller's block length into equal launches of at most that many frames
    const int nb = std::max(1, params.n_frame_for_srrf);
    const int launches = (nb + out.frames_per_launch - 1) / out.frames_per_launch;
    out.frames_per_launch = (nb + launches - 1) / launches;
    cache_put(path, key, out, best);
    std::ostringstream r;
    r << "{\"source\": \"measured\", \"key\": \"" << key << "\", \"frames_per_launch\": " << out.frames_per_launch
      << ", \"form\": \"" << form_name(out.form) << "\", \"ms_per_frame\": " << best << ", \"file\": \"" << path
      << "\", \"trial_frames\": " << n << ", \"candidates\": [" << cand.str() << "]}";
    out.report = r.str();
    return ESRRF_OK;
}
